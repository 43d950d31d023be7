// Time-invariant all-pole filter (one coefficient set per signal), parallel in
// time.  The time-varying chunked scan pays N basis filters per sample to
// learn each chunk's transition; with constant coefficients every chunk of a
// signal has the same transition P = C^L (C the companion matrix), so:
//
//  1. power    one CTA per signal: P = C^L by square-and-multiply in FP64.
//  2. zero     one thread per (signal, chunk): the chunk filtered from zero
//              state; its exit state z_c is stored.
//  3. combine  one warp per signal: entry states s_{c+1} = P s_c + z_c in
//              FP64, lane r holding row r of P.
//  4. fix      one thread per (signal, chunk): the chunk filtered again from
//              its exact entry state; outputs written.
//
// The backward is the same filter over reversed time on grad_y (for constant
// coefficients the adjoint's coefficient diagonal A[t+1+i, i] is just a[i]),
// followed by the per-tap reduction grad_a[i] = -sum_t grad_x[t] y[t-1-i] and
// grad_zi[k] = -sum_{i>=k} a[i] grad_x[i-k] (torchlpc/core.py:186-229 with a
// stride-0 A).  Coefficients and history live in registers; the history is a
// ring indexed by compile-time positions (steps unrolled by the padded order).
#include "lpc_ti.cuh"

namespace lpcb {

namespace {

constexpr int kTiChunk = 1024;  // target chunk length, rounded to a multiple of the padded order

inline int ti_chunk_len(int NP) { return NP * ((kTiChunk + NP - 1) / NP); }
inline size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

struct TiLayout {
    int NP, Lc;
    int64_t nc;
    size_t P, zst, est, total;
};

inline TiLayout ti_layout(size_t esz, int64_t B, int64_t T, int64_t N) {
    TiLayout l;
    l.NP = padded_order(N);
    l.Lc = ti_chunk_len(l.NP);
    l.nc = (T + l.Lc - 1) / l.Lc;
    size_t off = 0;
    l.P = off;  // [B][NP][NP] FP64 chunk transitions
    off = al256(off + (size_t)B * l.NP * l.NP * sizeof(double));
    l.zst = off;  // [B][nc][NP] zero-state exit states
    off = al256(off + (size_t)B * l.nc * l.NP * esz);
    l.est = off;  // [B][nc][NP] exact entry states
    off = al256(off + (size_t)B * l.nc * l.NP * esz);
    l.total = off;
    return l;
}

template <typename F>
struct TiArgs {
    const F *in;   // forward x, backward grad_y: (B,T)
    const F *a;    // a[b,i] = a[b*as_b + i]
    const F *zi;   // forward initial state (B,N) or nullptr
    F *out;        // forward y, backward grad_x
    int64_t as_b, B, T, nc;
    int N, Lc;
    double *P;
    F *zst, *est;
};

// acc - sum_i a[i] * h[(u-1-i) mod NP]: four partial chains over the older
// taps, the newest tap last (one FMA on the loop-carried path).
template <typename T, int NP>
__device__ __forceinline__ T ti_step(const T (&a)[NP], const T (&h)[NP], int u, T acc) {
    if constexpr (NP == 1) {
        return fma(-a[0], h[0], acc);
    } else {
        T q[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
        for (int i = 1; i < NP; ++i) q[i & 3] = fma(a[i], h[(u - 1 - i + 2 * NP) % NP], q[i & 3]);
        acc = acc - ((q[0] + q[1]) + (q[2] + q[3]));
        return fma(-a[0], h[(u - 1 + NP) % NP], acc);
    }
}

// State vector of the direct form: s[i] = y[t0-1-i] sits at ring slot NP-1-i
// at a block boundary.
template <int NP>
__device__ __forceinline__ constexpr int ti_slot(int i) {
    return NP - 1 - i;
}

// ---------------------------------------------------------------- power
// P = C^Lc, C the companion matrix of the padded order: row 0 is -a, row j
// (j >= 1) is the unit vector e_{j-1}.  Square-and-multiply in shared memory,
// one CTA per signal; each thread keeps a 4x4 tile of the product in
// registers, so a step of the inner product loads 8 operands for 16 FMAs (one
// output per thread loaded 2 per FMA and bound the kernel on shared-memory
// bandwidth: 276 us of a 1.03 ms forward at 2048 x 65536, order 32, on B200).
constexpr int kTiPowerThreads = 64;

template <typename T, int NP>
__global__ void __launch_bounds__(kTiPowerThreads) ti_power_kernel(const T *a, int64_t as_b, int N, int Lc, double *P) {
    __shared__ double M[NP][NP + 1], R[NP][NP + 1];
    constexpr int RB = NP % 4 == 0 ? 4 : NP;  // tile edge
    constexpr int NB = NP / RB;               // tiles per matrix edge
    static_assert(NB * NB <= kTiPowerThreads, "one tile per thread");
    const int64_t b = blockIdx.x;
    const int tid = threadIdx.x;
    for (int e = tid; e < NP * NP; e += blockDim.x) {
        const int r = e / NP, c = e - (e / NP) * NP;
        double m = 0.0;
        if (r == 0)
            m = c < N ? -(double)a[b * as_b + c] : 0.0;
        else
            m = (c == r - 1) ? 1.0 : 0.0;
        M[r][c] = m;
        R[r][c] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    const bool act = tid < NB * NB;
    const int r0 = act ? (tid / NB) * RB : 0;
    const int c0 = act ? (tid % NB) * RB : 0;
    // X <- X * Y (X may equal Y): the tile is computed in registers, written
    // back after every thread has read its operands
    auto mul_into = [&](double (*X)[NP + 1], double (*Y)[NP + 1]) {
        double acc[RB][RB];
#pragma unroll
        for (int i = 0; i < RB; ++i)
#pragma unroll
            for (int j = 0; j < RB; ++j) acc[i][j] = 0.0;
        if (act) {
#pragma unroll 4
            for (int k = 0; k < NP; ++k) {
                double xv[RB], yv[RB];
#pragma unroll
                for (int i = 0; i < RB; ++i) xv[i] = X[r0 + i][k];
#pragma unroll
                for (int j = 0; j < RB; ++j) yv[j] = Y[k][c0 + j];
#pragma unroll
                for (int i = 0; i < RB; ++i)
#pragma unroll
                    for (int j = 0; j < RB; ++j) acc[i][j] = fma(xv[i], yv[j], acc[i][j]);
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int i = 0; i < RB; ++i)
#pragma unroll
                for (int j = 0; j < RB; ++j) X[r0 + i][c0 + j] = acc[i][j];
        }
        __syncthreads();
    };
    for (int e = Lc; e > 0; e >>= 1) {
        if (e & 1) mul_into(R, M);
        if (e > 1) mul_into(M, M);
    }
    for (int e = tid; e < NP * NP; e += blockDim.x) P[(size_t)b * NP * NP + e] = R[e / NP][e % NP];
}

// ---------------------------------------------------------------- zero / fix
// FIX = false: chunk from zero state, exit state to zst.  FIX = true: chunk
// from its entry state est, outputs written.  REV: time runs backwards
// (index T-1-s of in/out for step s).  VEC (T a multiple of 4 floats, 16-byte
// aligned rows): each thread's input and output stream moves in 16-byte
// groups of 4 steps, the next group's load issued one group ahead.
template <typename T, int NP, bool REV, bool FIX, bool VEC>
__global__ void __launch_bounds__(256) ti_chunk_kernel(TiArgs<T> p) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p.B * p.nc) return;
    const int64_t b = idx / p.nc;
    const int64_t c = idx - b * p.nc;
    const int N = p.N;
    T a[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) a[i] = i < N ? p.a[b * p.as_b + i] : T(0);
    T h[NP];
    if constexpr (FIX) {
        const T *e = p.est + (size_t)idx * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) h[ti_slot<NP>(i)] = e[i];
    } else {
#pragma unroll
        for (int i = 0; i < NP; ++i) h[i] = T(0);
    }
    const T *inb = p.in + b * p.T;
    T *outb = p.out + b * p.T;
    const int64_t s0 = c * p.Lc;
    const int64_t send = min64(s0 + p.Lc, p.T);  // steps holding samples end here
    const int nblk = (int)((send - s0 + NP - 1) / NP);
    if constexpr (VEC && sizeof(T) == 4 && NP % 4 == 0) {
        // groups of 4 steps s..s+3: forward elements t..t+3, backward t-3..t
        auto gload = [&](int64_t s) -> float4 {
            if (s >= send) return make_float4(0.f, 0.f, 0.f, 0.f);
            const int64_t t = REV ? p.T - 4 - s : s;
            return *reinterpret_cast<const float4 *>(inb + t);
        };
        float4 nxt = gload(s0);
#pragma unroll 1
        for (int blk = 0; blk < nblk; ++blk) {
            const int64_t sb = s0 + (int64_t)blk * NP;
#pragma unroll
            for (int g = 0; g < NP / 4; ++g) {
                const float4 cur = nxt;
                nxt = gload(sb + 4 * g + 4);
                const float xin[4] = {REV ? cur.w : cur.x, REV ? cur.z : cur.y, REV ? cur.y : cur.z,
                                      REV ? cur.x : cur.w};
                float o[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int u = 4 * g + k;
                    h[u] = ti_step<T, NP>(a, h, u, xin[k]);
                    o[k] = h[u];
                }
                const int64_t s = sb + 4 * g;
                if (FIX && s < send) {
                    const int64_t t = REV ? p.T - 4 - s : s;
                    *reinterpret_cast<float4 *>(outb + t) =
                        REV ? make_float4(o[3], o[2], o[1], o[0]) : make_float4(o[0], o[1], o[2], o[3]);
                }
            }
        }
    } else {
#pragma unroll 1
        for (int blk = 0; blk < nblk; ++blk) {
            const int64_t sb = s0 + (int64_t)blk * NP;
#pragma unroll
            for (int u = 0; u < NP; ++u) {
                const int64_t s = sb + u;
                const bool in_range = s < send;
                const int64_t t = REV ? p.T - 1 - s : s;
                const T xv = in_range ? inb[t] : T(0);
                h[u] = ti_step<T, NP>(a, h, u, xv);
                if (FIX && in_range) outb[t] = h[u];
            }
        }
    }
    if constexpr (!FIX) {
        // exit state after the chunk's blocks (a partial last chunk has no successor)
        T *z = p.zst + (size_t)idx * NP;
#pragma unroll
        for (int i = 0; i < NP; ++i) z[i] = h[ti_slot<NP>(i)];
    }
}

// ---------------------------------------------------------------- combine
// One warp per signal: lane r keeps row r of P; s_{c+1} = P s_c + z_c (FP64).
// The zero-state exit states of 8 chunks are loaded ahead of the chain (a
// load per chunk inside it waited out a DRAM latency every chunk), and the
// matrix-vector product runs as four partial chains.
template <typename T, int NP, bool REV>
__global__ void __launch_bounds__(256) ti_combine_kernel(TiArgs<T> p) {
    const int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (b >= p.B) return;  // whole warps: b is uniform across a warp
    const bool row = lane < NP;
    double Pr[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) Pr[q] = row ? p.P[((size_t)b * NP + lane) * NP + q] : 0.0;
    double s = 0.0;
    if (!REV && row && p.zi && lane < p.N) s = (double)p.zi[b * p.N + lane];
    constexpr int AHEAD = 8;
    for (int64_t c0 = 0; c0 < p.nc; c0 += AHEAD) {
        double zv[AHEAD];
#pragma unroll
        for (int k = 0; k < AHEAD; ++k) {
            const int64_t c = c0 + k;
            zv[k] = (row && c + 1 < p.nc) ? (double)p.zst[((size_t)b * p.nc + c) * NP + lane] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < AHEAD; ++k) {
            const int64_t c = c0 + k;
            if (c >= p.nc) break;  // uniform across the warp
            if (row) p.est[((size_t)b * p.nc + c) * NP + lane] = (T)s;
            if (c + 1 == p.nc) break;
            double v[4] = {zv[k], 0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < NP; ++q) v[q & 3] = fma(Pr[q], __shfl_sync(0xffffffffu, s, q), v[q & 3]);
            s = (v[0] + v[1]) + (v[2] + v[3]);
        }
    }
}

// ---------------------------------------------------------------- gradients
// grad_a[b,i] = sgn * sum_t grad_x[b,t] * ypad[b,t-1-i], ypad(-1-k) = zi[b,k].
// One thread per segment of a signal keeps the last NP outputs in a register
// ring (slot (i - j) mod NP holds y[t_j - 1 - i] at step j), so each sample
// costs one load of grad_x, one of y and NP FMAs; warps whose lanes share a
// signal reduce with shuffles and add once per tap.  VEC: 16-byte loads.
template <typename T, int NP, bool VEC>
__global__ void __launch_bounds__(256) ti_grad_a_kernel(const T *gx, const T *y, const T *zi, T *ga, int64_t B,
                                                       int64_t T_, int N, int seg, int64_t nseg, T sgn) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = idx < B * nseg;
    const int64_t b = on ? idx / nseg : -1;
    T acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = T(0);
    if (on) {
        const int64_t t0 = (idx - b * nseg) * seg;
        const int64_t tend = min64(t0 + seg, T_);
        const T *gb = gx + b * T_;
        const T *yb = y + b * T_;
        const T *zb = zi ? zi + b * N : nullptr;
        T yr[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            const int64_t j = t0 - 1 - i;
            yr[i] = j >= 0 ? yb[j] : ((zb && -1 - j < N) ? zb[-1 - j] : T(0));
        }
        const int nblk = (int)((tend - t0 + NP - 1) / NP);
#pragma unroll 1
        for (int blk = 0; blk < nblk; ++blk) {
            const int64_t tb = t0 + (int64_t)blk * NP;
            if constexpr (VEC && sizeof(T) == 4 && NP % 4 == 0) {
#pragma unroll
                for (int q = 0; q < NP / 4; ++q) {
                    const int64_t t = tb + 4 * q;
                    float4 g4 = make_float4(0.f, 0.f, 0.f, 0.f), y4 = g4;
                    if (t < tend) {
                        g4 = *reinterpret_cast<const float4 *>(gb + t);
                        y4 = *reinterpret_cast<const float4 *>(yb + t);
                    }
                    const float gv[4] = {g4.x, g4.y, g4.z, g4.w};
                    const float yv[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const int u = 4 * q + k;
#pragma unroll
                        for (int i = 0; i < NP; ++i) acc[i] = fma(gv[k], yr[(i - u + NP) % NP], acc[i]);
                        yr[NP - 1 - u] = yv[k];
                    }
                }
            } else {
#pragma unroll
                for (int u = 0; u < NP; ++u) {
                    const int64_t t = tb + u;
                    const T g = t < tend ? gb[t] : T(0);
#pragma unroll
                    for (int i = 0; i < NP; ++i) acc[i] = fma(g, yr[(i - u + NP) % NP], acc[i]);
                    yr[NP - 1 - u] = t < T_ ? yb[t] : T(0);
                }
            }
        }
    }
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    // every lane takes part in both collectives (idle lanes included)
    const int64_t b0 = __shfl_sync(full, b, 0);
    const bool uniform = __all_sync(full, on && b == b0);
    if (uniform) {
#pragma unroll
        for (int i = 0; i < NP; ++i) {
            T v = acc[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
            if (lane == 0 && i < N && v != T(0)) atomicAdd(ga + b * N + i, sgn * v);
        }
    } else if (on) {
#pragma unroll
        for (int i = 0; i < NP; ++i)
            if (i < N && acc[i] != T(0)) atomicAdd(ga + b * N + i, sgn * acc[i]);
    }
}

// grad_zi[b,k] = -sum_{i=k}^{N-1} a[b,i] grad_x[b,i-k]  (grad_x beyond T is 0)
template <typename T>
__global__ void ti_grad_zi_kernel(const T *gx, const T *a, int64_t as_b, T *gzi, int64_t B, int64_t T_, int N) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= B * N) return;
    const int64_t b = e / N;
    const int k = (int)(e - b * N);
    T v = T(0);
    for (int i = k; i < N; ++i)
        if (i - k < T_) v = fma(-a[b * as_b + i], gx[b * T_ + (i - k)], v);
    gzi[e] = v;
}

template <typename T, int NP, bool REV>
cudaError_t ti_run(TiArgs<T> p, cudaStream_t st) {
    ti_power_kernel<T, NP><<<(unsigned)p.B, kTiPowerThreads, 0, st>>>(p.a, p.as_b, p.N, p.Lc, p.P);
    const int64_t threads = p.B * p.nc;
    const unsigned g1 = (unsigned)((threads + 255) / 256);
    // 16-byte groups need whole groups per signal, aligned rows and an order
    // that is a multiple of the group
    const bool vec = sizeof(T) == 4 && NP % 4 == 0 && p.T % 4 == 0 &&
                     (reinterpret_cast<uintptr_t>(p.in) & 15u) == 0 && (reinterpret_cast<uintptr_t>(p.out) & 15u) == 0;
    if (vec)
        ti_chunk_kernel<T, NP, REV, false, true><<<g1, 256, 0, st>>>(p);
    else
        ti_chunk_kernel<T, NP, REV, false, false><<<g1, 256, 0, st>>>(p);
    ti_combine_kernel<T, NP, REV><<<(unsigned)((p.B * 32 + 255) / 256), 256, 0, st>>>(p);
    if (vec)
        ti_chunk_kernel<T, NP, REV, true, true><<<g1, 256, 0, st>>>(p);
    else
        ti_chunk_kernel<T, NP, REV, true, false><<<g1, 256, 0, st>>>(p);
    return cudaGetLastError();
}

template <typename T, bool REV>
cudaError_t ti_dispatch(const TiArgs<T> &p, int NP, cudaStream_t st) {
    switch (NP) {
#define LPCB_CASE(n) \
    case n: return ti_run<T, n, REV>(p, st);
        LPCB_FOR_EACH_NP(LPCB_CASE)
#undef LPCB_CASE
        default: return cudaErrorNotSupported;
    }
}

template <typename T>
TiArgs<T> ti_args(const TiLayout &l, const T *in, const T *a, int64_t as_b, const T *zi, T *out, int64_t B,
                  int64_t T_, int64_t N, void *ws) {
    unsigned char *w = static_cast<unsigned char *>(ws);
    TiArgs<T> p{};
    p.in = in;
    p.a = a;
    p.as_b = as_b;
    p.zi = zi;
    p.out = out;
    p.B = B;
    p.T = T_;
    p.nc = l.nc;
    p.N = (int)N;
    p.Lc = l.Lc;
    p.P = reinterpret_cast<double *>(w + l.P);
    p.zst = reinterpret_cast<T *>(w + l.zst);
    p.est = reinterpret_cast<T *>(w + l.est);
    return p;
}

template <typename T, int NP>
cudaError_t launch_grad_a(const T *gx, const T *y, const T *zi, T *ga, int64_t B, int64_t T_, int N, T sgn,
                          cudaStream_t st) {
    const int seg = ti_chunk_len(NP);
    const int64_t nseg = (T_ + seg - 1) / seg;
    const int64_t threads = B * nseg;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    const bool vec = sizeof(T) == 4 && NP % 4 == 0 && T_ % 4 == 0 && (reinterpret_cast<uintptr_t>(gx) & 15u) == 0 &&
                     (reinterpret_cast<uintptr_t>(y) & 15u) == 0;
    if (vec)
        ti_grad_a_kernel<T, NP, true><<<grid, 256, 0, st>>>(gx, y, zi, ga, B, T_, N, seg, nseg, sgn);
    else
        ti_grad_a_kernel<T, NP, false><<<grid, 256, 0, st>>>(gx, y, zi, ga, B, T_, N, seg, nseg, sgn);
    return cudaGetLastError();
}

}  // namespace

bool ti_supported(int64_t N) { return N >= 1 && N <= 32; }

size_t ti_workspace(size_t esz, int64_t B, int64_t T, int64_t N) {
    if (!ti_supported(N)) return 0;
    return ti_layout(esz, B, T, N).total;
}

template <typename T>
cudaError_t ti_grad_a(const T *gx, const T *y, const T *zi, T *ga, int64_t B, int64_t T_, int64_t N, bool neg,
                      cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(ga, 0, (size_t)B * N * sizeof(T), st);
    if (e != cudaSuccess) return e;
    const T sgn = neg ? T(1) : T(-1);
    switch (padded_order(N)) {
#define LPCB_CASE(n) \
    case n: return launch_grad_a<T, n>(gx, y, zi, ga, B, T_, (int)N, sgn, st);
        LPCB_FOR_EACH_NP(LPCB_CASE)
#undef LPCB_CASE
        default: return cudaErrorNotSupported;
    }
}

template <typename T>
cudaError_t ti_forward(const FwdArgs<T> &a, void *ws, size_t ws_bytes, cudaStream_t st) {
    const TiLayout l = ti_layout(sizeof(T), a.B, a.T, a.N);
    if (ws_bytes < l.total) return cudaErrorInvalidValue;
    const TiArgs<T> p = ti_args<T>(l, a.x, a.A, a.a_stride_b, a.zi, a.y, a.B, a.T, a.N, ws);
    return ti_dispatch<T, false>(p, l.NP, st);
}

template <typename T>
cudaError_t ti_backward(const BwdArgs<T> &a, void *ws, size_t ws_bytes, cudaStream_t st) {
    const TiLayout l = ti_layout(sizeof(T), a.B, a.T, a.N);
    if (ws_bytes < l.total) return cudaErrorInvalidValue;
    const TiArgs<T> p = ti_args<T>(l, a.gy, a.A, a.a_stride_b, nullptr, a.gx, a.B, a.T, a.N, ws);
    cudaError_t e = ti_dispatch<T, true>(p, l.NP, st);
    if (e != cudaSuccess) return e;
    if (a.gA) {
        e = ti_grad_a<T>(a.gx, a.y, a.zi, a.gA, a.B, a.T, a.N, false, st);
        if (e != cudaSuccess) return e;
    }
    if (a.gzi) {
        const int64_t n = a.B * a.N;
        ti_grad_zi_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.gx, a.A, a.a_stride_b, a.gzi, a.B, a.T,
                                                                          (int)a.N);
        e = cudaGetLastError();
    }
    return e;
}

template cudaError_t ti_grad_a<float>(const float *, const float *, const float *, float *, int64_t, int64_t,
                                      int64_t, bool, cudaStream_t);
template cudaError_t ti_grad_a<double>(const double *, const double *, const double *, double *, int64_t, int64_t,
                                       int64_t, bool, cudaStream_t);
template cudaError_t ti_forward<float>(const FwdArgs<float> &, void *, size_t, cudaStream_t);
template cudaError_t ti_forward<double>(const FwdArgs<double> &, void *, size_t, cudaStream_t);
template cudaError_t ti_backward<float>(const BwdArgs<float> &, void *, size_t, cudaStream_t);
template cudaError_t ti_backward<double>(const BwdArgs<double> &, void *, size_t, cudaStream_t);

}  // namespace lpcb
