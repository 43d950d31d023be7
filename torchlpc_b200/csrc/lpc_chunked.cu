// Chunked linear-recurrence scan for the all-pole filter (parallel in time).
//
// A signal is cut into chunks of L samples.  Over one chunk the filter is an
// affine map of the N-sample state s (s[i] = y[t0-1-i]):
//     s_out = P s_in + z,
// where column k of P is the chunk's response to the unit state e_k and z is
// its response to the input from zero state.  A persistent CTA takes a
// *batch* of G consecutive chunks of one signal from an atomic ticket queue
// (tickets are ordered so that a batch's predecessors always hold earlier
// tickets, which makes every wait below finite) and runs four phases:
//
//  A  "lanes = filters": every chunk gets N+1 lanes, N basis filters and one
//     zero-state filter, each holding its N-tap history in registers.  The
//     coefficient rows of the chunk are staged per window of W steps into
//     shared memory with cp.async (double buffered) and read as broadcasts
//     (one 16-byte shared load feeds every lane of the chunk).
//  B  a Blelloch tree over the G affine maps in shared memory: the batch
//     aggregate (up-sweep) and each chunk's exclusive prefix (down-sweep).
//  C  decoupled look-back over the predecessor batches of the same signal:
//     the aggregate is published, predecessors' aggregates are composed in
//     FP64 until an inclusive state is found, the batch's inclusive state is
//     published (FP64).  Every spin-wait is bounded; on expiry the kernel
//     records LPC_ERR_TIMEOUT in the workspace status word and moves on.
//  D  fix-up: one lane per chunk re-runs its chunk from the exact entry state
//     (the coefficient windows are streamed again; they are L2-resident by
//     then) and the CTA writes the outputs back coalesced.
//
// The backward runs the same machinery over reversed time on grad_y: the
// adjoint recurrence grad_x[t] = grad_y[t] - sum_i A[t+1+i,i] grad_x[t+1+i] in
// transposed (scatter) form, where producing grad_x[t] adds -A[t,i]*grad_x[t]
// to the pending accumulator of output t-1-i.  Its state is the N pending
// accumulators and each step reads one contiguous row A[t,:], so both
// directions stream the same row windows.  grad_A = -grad_x[t] * y[t-1-i] is
// fused into the phase-D epilogue (time-invariant A: per-tap sums added
// atomically); grad_zi is the adjoint carried N steps past t = 0.
#include "lpc_chunked.cuh"

namespace lpcb {

namespace {

// ----------------------------------------------------------------------------
// Workspace layout and flags.
// ----------------------------------------------------------------------------
constexpr unsigned kFlagAgg = 1u;
constexpr unsigned kFlagInc = 2u;
constexpr int kHeaderBytes = 256;  // ticket counter, status word, padding
constexpr int kLookbackChunk = 8;   // predecessor aggregates staged per round of the composition

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

struct WsLayout {
    size_t flags, aggP, aggz, incl, total;
};

inline WsLayout ws_layout(size_t esz, int64_t nbatches, int64_t N) {
    WsLayout l;
    size_t off = kHeaderBytes;
    l.flags = off;
    off = align256(off + (size_t)nbatches * 4);
    l.aggP = off;
    off = align256(off + (size_t)nbatches * N * N * esz);
    l.aggz = off;
    off = align256(off + (size_t)nbatches * N * 8);
    l.incl = off;
    off = align256(off + (size_t)nbatches * N * 8);
    l.total = off;
    return l;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

template <typename F>
struct ChunkParams {
    const F *in;     // forward: x (B,T); backward: grad_y (B,T)
    const F *A;      // A[b,t,i] = A[b*as_b + t*as_t + i]
    const F *zi;     // (B,N) or nullptr
    const F *ysave;  // backward: forward output y (B,T)
    F *out;          // forward: y; backward: grad_x
    F *gA;           // backward: (B,T,N) or (B,N) when as_t == 0, or nullptr
    F *gzi;          // backward: (B,N) or nullptr
    int64_t B, T, as_b, as_t;
    int N;
    int L;           // chunk length (multiple of the window)
    int G;           // chunks per batch
    int64_t nbps;    // batches per signal
    int64_t nbatches;
    unsigned *counter, *status, *flags;
    F *aggP;         // [nbatches][N][N]
    double *aggz;    // [nbatches][N]
    double *incl;    // [nbatches][N]
    unsigned spin_limit;
};

template <int NP>
struct Cfg {
    static constexpr int THREADS = 256;
    static constexpr int W = NP * ((16 + NP - 1) / NP);  // steps per window, multiple of NP
};

// Per-chunk stride of a coefficient window in shared memory: W rows of NP plus
// one 16-byte pad so that the rows different chunks read in the same step
// fall in different banks.
__host__ __device__ constexpr int group_stride(int W, int NP, int esz) { return W * NP + 16 / esz; }
// Row stride of a stored affine map (16-byte aligned, padded against bank conflicts).
__host__ __device__ constexpr int map_row_stride(int NP, int esz) {
    return ((NP + 16 / esz - 1) / (16 / esz)) * (16 / esz) + 16 / esz;
}
__host__ __device__ constexpr int map_stride(int NP, int esz) {
    return NP * map_row_stride(NP, esz) + ((NP + 16 / esz - 1) / (16 / esz)) * (16 / esz);
}

// acc - sum_i a[i] * h[(u-1-i) mod NP] with two partial chains (even/odd taps)
// and the newest tap (i = 0) applied last, so consecutive steps overlap and
// the loop-carried path is one FMA.
template <typename T, int NP>
__device__ __forceinline__ T step_dot(const T (&a)[NP], const T (&h)[NP], int u, T acc) {
    if constexpr (NP == 1) {
        return fma(-a[0], h[(u - 1 + NP) % NP], acc);
    } else {
        T p0 = T(0), p1 = T(0);
#pragma unroll
        for (int i = NP - 1; i >= 1; --i) {
            if ((i & 1) == 0)
                p0 = fma(a[i], h[(u - 1 - i + 2 * NP) % NP], p0);
            else
                p1 = fma(a[i], h[(u - 1 - i + 2 * NP) % NP], p1);
        }
        acc = acc - (p0 + p1);
        return fma(-a[0], h[(u - 1 + NP) % NP], acc);
    }
}

// Transposed (scatter) form for the adjoint recurrence: c[(u+i) mod NP] is the
// pending accumulator of the output i steps ahead; the step's output consumes
// c[u] and scatters -a[i]*out into the rest, so a step reads one contiguous
// coefficient row.
template <typename T, int NP>
__device__ __forceinline__ T step_scatter(const T (&a)[NP], T (&c)[NP], int u, T in) {
    const T g = in + c[u];
    c[u] = T(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) c[(u + 1 + i) % NP] = fma(-a[i], g, c[(u + 1 + i) % NP]);
    return g;
}

// Ring position of logical state element i at a window boundary (u = 0):
// direct form s[i] = y[t0-1-i] at h[NP-1-i]; transposed form c[i] at c[i].
template <bool REV, int NP>
__device__ __forceinline__ constexpr int state_slot(int i) {
    return REV ? i : NP - 1 - i;
}

template <typename T, int NP>
__device__ __forceinline__ void lds_row(T (&dst)[NP], const T *src) {
    if constexpr (sizeof(T) * NP % 16 == 0) {
        constexpr int V = 16 / sizeof(T);
        using V4 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
#pragma unroll
        for (int v = 0; v < NP / V; ++v) {
            V4 q = reinterpret_cast<const V4 *>(src)[v];
            const T *qs = reinterpret_cast<const T *>(&q);
#pragma unroll
            for (int j = 0; j < V; ++j) dst[v * V + j] = qs[j];
        }
    } else {
#pragma unroll
        for (int i = 0; i < NP; ++i) dst[i] = src[i];
    }
}

// Shared-memory plan (bytes), all regions 16-byte aligned.
struct SmemPlan {
    size_t abuf, ibuf, obuf, ybuf, maps, st, sin, lbP, lbz, misc, total;
    __host__ __device__ SmemPlan(size_t esz, int NP, int W, int G, int N, bool rev) {
        auto al = [](size_t v) { return (v + 15) & ~size_t(15); };
        size_t off = 0;
        abuf = off;
        const size_t abytes = al((size_t)2 * G * group_stride(W, NP, (int)esz) * esz);
        // the tree maps alias the window buffers (phases B/C run between the
        // window loops of phases A and D)
        int Gp = 1;
        while (Gp < G) Gp <<= 1;
        const size_t mapbytes = al((size_t)Gp * map_stride(NP, (int)esz) * esz);
        maps = off;
        off += al(abytes > mapbytes ? abytes : mapbytes);
        ibuf = off;
        off += al((size_t)2 * G * W * esz);
        obuf = off;
        off += al((size_t)G * W * esz);
        ybuf = off;
        if (rev) off += al((size_t)2 * G * (W + NP) * esz);
        st = off;  // FP64 entry states of the tree nodes
        off += al((size_t)Gp * NP * sizeof(double));
        sin = off;
        off += al((size_t)NP * sizeof(double));
        lbP = off;  // look-back stages: predecessor aggregates (two stages of kLookbackChunk)
        off += al((size_t)2 * kLookbackChunk * NP * NP * esz);
        lbz = off;
        off += al((size_t)2 * kLookbackChunk * NP * sizeof(double));
        misc = off;
        off += 64;
        total = off;
        (void)N;
    }
};

// ----------------------------------------------------------------------------
// Window loaders.  Window w of chunk g covers steps [w*W, w*W+W) of the chunk.
// Forward: step j is time t = tb + g*L + w*W + j, stored at slot j.
// Backward: step j is time t = top-1-j (top = T - (tb + g*L + w*W)), stored at
// slot t - (top - W) = W-1-j.  Either way a window is a run of W consecutive
// coefficient rows in natural order; rows outside [0, T) read as zero.
// ----------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool is_aligned16(const void *p) {
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

template <typename T, int NP, bool REV>
struct Loader {
    static constexpr int W = Cfg<NP>::W;
    static constexpr int THREADS = Cfg<NP>::THREADS;
    static constexpr int V = 16 / sizeof(T);
    static constexpr int GS = group_stride(W, NP, sizeof(T));

    // Vector fast path: order equals the padded order, rows are dense, 16-byte
    // multiples and 16-byte aligned, so every index below divides by a
    // compile-time constant.
    __device__ static bool fast(const ChunkParams<T> &p) {
        return p.N == NP && p.as_t == NP && NP % V == 0 && (p.as_b * (int64_t)sizeof(T)) % 16 == 0 &&
               is_aligned16<T>(p.A);
    }

    // First row held by slot 0 of chunk g's window w, and the valid slot range.
    __device__ static void rows(const ChunkParams<T> &p, int64_t tb, int g, int w, int64_t &row0, int &lo,
                                int &hi) {
        if (!REV) {
            row0 = tb + (int64_t)g * p.L + (int64_t)w * W;
            lo = 0;
            hi = (int)max64(0, min64(W, p.T - row0));
        } else {
            const int64_t top = p.T - (tb + (int64_t)g * p.L + (int64_t)w * W);
            row0 = top - W;
            lo = (int)min64(W, max64(0, -row0));
            hi = W;
        }
    }

    __device__ static void load(const ChunkParams<T> &p, bool vec, int64_t b, int64_t tb, int Gb, int w,
                                T *As, T *xs, T *ys, bool with_y) {
        const int N = p.N;
        const int tid = threadIdx.x;
        const T *Ab = p.A + b * p.as_b;
        const T *inb = p.in + b * p.T;
        if (vec) {
            constexpr int RV = NP / V;       // vectors per row
            constexpr int VPW = W * RV;      // vectors per chunk window
            for (int e = tid; e < Gb * VPW; e += THREADS) {
                const int g = e / VPW;
                const int v = e - g * VPW;
                const int r = v / RV;
                int64_t row0;
                int lo, hi;
                rows(p, tb, g, w, row0, lo, hi);
                T *dst = As + (size_t)g * GS + v * V;
                if (r >= lo && r < hi) {
                    cp_async<16>(dst, Ab + row0 * NP + v * V);
                } else {
#pragma unroll
                    for (int j = 0; j < V; ++j) dst[j] = T(0);
                }
            }
        } else {
            const int per = W * N;
            for (int e = tid; e < Gb * per; e += THREADS) {
                const int g = e / per;
                const int rem = e - g * per;
                const int r = rem / N;
                const int i = rem - r * N;
                int64_t row0;
                int lo, hi;
                rows(p, tb, g, w, row0, lo, hi);
                T *dst = As + (size_t)g * GS + r * NP + i;
                if (r >= lo && r < hi)
                    cp_async<sizeof(T)>(dst, Ab + (row0 + r) * p.as_t + i);
                else
                    *dst = T(0);
            }
        }
        // inputs (x forward, grad_y backward), slot r <-> index row0 + r
        for (int e = tid; e < Gb * W; e += THREADS) {
            const int g = e / W;
            const int r = e - g * W;
            int64_t row0;
            int lo, hi;
            rows(p, tb, g, w, row0, lo, hi);
            if (r >= lo && r < hi)
                cp_async<sizeof(T)>(xs + e, inb + row0 + r);
            else
                xs[e] = T(0);
        }
        if (REV && with_y) {
            // ys[g][q] = ypad(top - 2 - q), q in [0, W + NP): the lagged outputs
            // y[t-1-i] of the window's steps (y[-1-k] = zi[k])
            const T *yb = p.ysave + b * p.T;
            const T *zib = p.zi ? p.zi + b * N : nullptr;
            constexpr int PY = W + NP;
            for (int e = tid; e < Gb * PY; e += THREADS) {
                const int g = e / PY;
                const int q = e - g * PY;
                const int64_t top = p.T - (tb + (int64_t)g * p.L + (int64_t)w * W);
                const int64_t j = top - 2 - q;
                T *dst = ys + e;
                if (j >= 0 && j < p.T)
                    cp_async<sizeof(T)>(dst, yb + j);
                else if (j < 0 && -1 - j < N && zib)
                    *dst = zib[-1 - j];
                else
                    *dst = T(0);
            }
        }
    }
};

// ----------------------------------------------------------------------------
// The kernel.
// ----------------------------------------------------------------------------
template <typename T, int NP, bool REV, bool NEG>
__global__ void __launch_bounds__(Cfg<NP>::THREADS, NP <= 16 ? 4 : 3) chunked_kernel(ChunkParams<T> p) {
    constexpr int W = Cfg<NP>::W;
    constexpr int THREADS = Cfg<NP>::THREADS;
    constexpr int V = 16 / sizeof(T);
    constexpr int GS = group_stride(W, NP, sizeof(T));
    constexpr int RS = map_row_stride(NP, sizeof(T));
    constexpr int MS = map_stride(NP, sizeof(T));
    extern __shared__ __align__(16) unsigned char smem[];
    const int N = p.N;
    const int G = p.G;
    const int tid = threadIdx.x;
    const SmemPlan S(sizeof(T), NP, W, G, N, REV);
    T *Abuf = reinterpret_cast<T *>(smem + S.abuf);
    T *ibuf = reinterpret_cast<T *>(smem + S.ibuf);
    T *obuf = reinterpret_cast<T *>(smem + S.obuf);
    T *ybuf = reinterpret_cast<T *>(smem + S.ybuf);
    T *maps = reinterpret_cast<T *>(smem + S.maps);  // [Gp][NP rows of RS | z]
    double *st = reinterpret_cast<double *>(smem + S.st);      // [Gp][NP]
    double *s_in = reinterpret_cast<double *>(smem + S.sin);   // [NP]
    int64_t *misc = reinterpret_cast<int64_t *>(smem + S.misc);
    int Gp = 1;
    while (Gp < G) Gp <<= 1;

    const bool vec = Loader<T, NP, REV>::fast(p);
    const int grp = tid / (N + 1);
    const int kk = tid - grp * (N + 1);
    const int nwin = p.L / W;

    for (;;) {
        __syncthreads();
        if (tid == 0) misc[0] = (int64_t)atomicAdd(p.counter, 1u);
        __syncthreads();
        const int64_t ticket = misc[0];
        if (ticket >= p.nbatches) break;
        const int64_t kb = ticket / p.B;  // batch index within the signal
        const int64_t b = ticket - kb * p.B;
        const int64_t tb = kb * (int64_t)G * p.L;  // first step of the batch
        const int64_t rem = p.T - tb;
        const int Gb = (int)min64(G, (rem + p.L - 1) / p.L);

        // ------------------------------------------------------------ phase A
        // chunk maps: N basis filters + one zero-state filter per chunk
        if (N < NP)  // padded coefficient columns must read as zero
            for (int e = tid; e < 2 * G * GS; e += THREADS)
                if ((e % GS) % NP >= N) Abuf[e] = T(0);
        const bool active = grp < Gb;
        const bool xlane = (kk == N);
        T h[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) h[j] = (active && !xlane && j == state_slot<REV, NP>(kk)) ? T(1) : T(0);

        Loader<T, NP, REV>::load(p, vec, b, tb, Gb, 0, Abuf, ibuf, nullptr, false);
        cp_async_commit();
        for (int w = 0; w < nwin; ++w) {
            const T *As = Abuf + (size_t)(w & 1) * G * GS;
            const T *xs = ibuf + (size_t)(w & 1) * G * W;
            if (w + 1 < nwin)
                Loader<T, NP, REV>::load(p, vec, b, tb, Gb, w + 1, Abuf + (size_t)((w + 1) & 1) * G * GS,
                                         ibuf + (size_t)((w + 1) & 1) * G * W, nullptr, false);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            if (active) {
                const T *Ag = As + (size_t)grp * GS;
                const T *xg = xs + (size_t)grp * W;
#pragma unroll 1
                for (int blk = 0; blk < W / NP; ++blk) {
#pragma unroll
                    for (int u = 0; u < NP; ++u) {
                        const int j = blk * NP + u;
                        const int slot = REV ? W - 1 - j : j;
                        T a[NP];
                        lds_row<T, NP>(a, Ag + (size_t)slot * NP);
                        if constexpr (NEG) {
#pragma unroll
                            for (int i = 0; i < NP; ++i) a[i] = -a[i];
                        }
                        const T in = xlane ? xg[slot] : T(0);
                        if constexpr (REV)
                            step_scatter<T, NP>(a, h, u, in);
                        else
                            h[u] = step_dot<T, NP>(a, h, u, in);
                    }
                }
            }
            __syncthreads();
        }
        cp_async_wait<0>();
        __syncthreads();

        // ------------------------------------------------------------ phase B
        // maps (aliasing the window buffers): zero, then column k of chunk g's
        // P from lane k, z from the zero-state lane; identity beyond Gb.
        for (int e = tid; e < Gp * MS; e += THREADS) maps[e] = T(0);
        __syncthreads();
        if (active) {
            T *Mg = maps + (size_t)grp * MS;
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                if (i < N) {
                    const T v = h[state_slot<REV, NP>(i)];
                    if (!xlane)
                        Mg[i * RS + kk] = v;
                    else
                        Mg[NP * RS + i] = v;
                }
            }
        }
        for (int e = tid; e < (Gp - Gb) * N; e += THREADS) {
            const int g = Gb + e / N;
            const int i = e - (g - Gb) * N;
            maps[(size_t)g * MS + i * RS + i] = T(1);
        }
        __syncthreads();
        // up-sweep: M[j] <- M[j] o M[i] (i = j - d: M[i] acts first).  One
        // thread per output row keeps the row in registers.
        for (int d = 1; d < Gp; d <<= 1) {
            const int npairs = Gp / (2 * d);
            const int pslots = THREADS / NP;
            for (int base = 0; base < npairs; base += pslots) {
                const int m = base + tid / NP;
                const int row = tid % NP;
                const bool on = (tid / NP) < pslots && m < npairs;
                T acc[NP];
                T accz = T(0);
                if (on) {
                    const int j = 2 * d * m + 2 * d - 1;
                    const int i = j - d;
                    const T *Pj = maps + (size_t)j * MS + row * RS;
                    const T *Mi = maps + (size_t)i * MS;
#pragma unroll
                    for (int c = 0; c < NP; ++c) acc[c] = T(0);
                    accz = maps[(size_t)j * MS + NP * RS + row];
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        const T pq = Pj[q];
                        T mrow[NP];
                        lds_row<T, NP>(mrow, Mi + q * RS);
#pragma unroll
                        for (int c = 0; c < NP; ++c) acc[c] = fma(pq, mrow[c], acc[c]);
                        accz = fma(pq, Mi[NP * RS + q], accz);
                    }
                }
                __syncthreads();
                if (on) {
                    const int j = 2 * d * m + 2 * d - 1;
                    T *Pj = maps + (size_t)j * MS + row * RS;
#pragma unroll
                    for (int c = 0; c < NP; ++c) Pj[c] = acc[c];
                    maps[(size_t)j * MS + NP * RS + row] = accz;
                }
                __syncthreads();
            }
        }

        // ------------------------------------------------------------ phase C
        // publish the aggregate (root), look back, publish the inclusive state
        const int64_t me = ticket;
        const T *root = maps + (size_t)(Gp - 1) * MS;
        if (kb == 0) {
            if (tid < NP) {
                double v = 0.0;
                if (!REV && p.zi && tid < N) v = (double)p.zi[b * N + tid];
                s_in[tid] = v;
            }
        } else {
            for (int e = tid; e < N * N; e += THREADS) {
                const int r = e / N, c = e - (e / N) * N;
                p.aggP[(size_t)me * N * N + e] = root[r * RS + c];
            }
            for (int e = tid; e < N; e += THREADS) p.aggz[(size_t)me * N + e] = (double)root[NP * RS + e];
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(p.flags + me, kFlagAgg);
            if (tid < 32) {
                // warp 0: parallel look-back.  Lane l watches predecessor
                // kb-1-l-32r; a round ends when every watched batch has
                // published; the nearest inclusive state ends the walk.
                const int lane = tid;
                int64_t found = -1;
                bool timeout = false;
                for (int64_t hi = kb - 1; hi >= 0 && found < 0 && !timeout; hi -= 32) {
                    const int64_t m = hi - lane;
                    unsigned f = kFlagInc;  // batches before 0 do not exist: treat as resolved
                    if (m >= 0) {
                        const unsigned *fp = p.flags + m * p.B + b;
                        f = ld_acquire(fp);
                        unsigned n = 0;
                        while (f == 0u) {
                            if (++n > p.spin_limit || ld_acquire(p.status) != 0u) {
                                atomicOr(p.status, 1u);
                                break;
                            }
                            __nanosleep(32);
                            f = ld_acquire(fp);
                        }
                    }
                    timeout = __any_sync(0xffffffffu, f == 0u);
                    const unsigned inc = __ballot_sync(0xffffffffu, f == kFlagInc && m >= 0);
                    if (inc) found = hi - (__ffs(inc) - 1);
                }
                if (found < 0 && !timeout) {  // cannot happen: batch 0 always publishes an inclusive state
                    if (lane == 0) atomicOr(p.status, 2u);
                    timeout = true;
                }
                // the flags seen above were acquired lane by lane; order every
                // lane's reads of the predecessors' data after them
                __threadfence();
                if (timeout) {
                    if (tid < NP) s_in[tid] = 0.0;
                } else if (tid < NP) {
                    double v = 0.0;
                    if (tid < N) v = p.incl[(size_t)(found * p.B + b) * N + tid];
                    s_in[tid] = v;
                }
                if (tid == 0) misc[1] = timeout ? -1 : found;
            }
            __syncthreads();
            // compose the aggregates found+1 .. kb-1 in order.  The whole CTA
            // streams them into a double-buffered shared stage, kLookbackChunk
            // hops at a time, while warp 0 applies the previous stage.
            const int64_t found = misc[1];
            if (found >= 0) {
                T *lbP = reinterpret_cast<T *>(smem + S.lbP);
                double *lbz = reinterpret_cast<double *>(smem + S.lbz);
                const int64_t m0 = found + 1;
                const int64_t K = kb - m0;
                const int64_t nch = (K + kLookbackChunk - 1) / kLookbackChunk;
                const int per = N * N + N;
                auto issue = [&](int64_t c) {
                    const int64_t h0 = c * kLookbackChunk;
                    const int nh = (int)min64(kLookbackChunk, K - h0);
                    T *dP = lbP + (size_t)(c & 1) * kLookbackChunk * NP * NP;
                    double *dz = lbz + (size_t)(c & 1) * kLookbackChunk * NP;
                    for (int e = tid; e < nh * per; e += THREADS) {
                        const int hh = e / per;
                        const int r = e - hh * per;
                        const int64_t idx = (m0 + h0 + hh) * p.B + b;
                        if (r < N * N) {
                            const int row = r / N, col = r - (r / N) * N;
                            cp_async<sizeof(T)>(dP + (size_t)hh * NP * NP + row * NP + col,
                                                p.aggP + (size_t)idx * N * N + r);
                        } else {
                            cp_async<8>(dz + (size_t)hh * NP + (r - N * N), p.aggz + (size_t)idx * N + (r - N * N));
                        }
                    }
                };
                if (nch > 0) issue(0);
                cp_async_commit();
                for (int64_t c = 0; c < nch; ++c) {
                    if (c + 1 < nch) issue(c + 1);
                    cp_async_commit();
                    cp_async_wait<1>();
                    __syncthreads();
                    if (tid < 32) {
                        const int lane = tid;
                        const int nh = (int)min64(kLookbackChunk, K - c * kLookbackChunk);
                        const T *P0 = lbP + (size_t)(c & 1) * kLookbackChunk * NP * NP;
                        const double *z0 = lbz + (size_t)(c & 1) * kLookbackChunk * NP;
                        for (int hh = 0; hh < nh; ++hh) {
                            double v = 0.0;
                            if (lane < N) {
                                const T *Pr = P0 + (size_t)hh * NP * NP + lane * NP;
                                double v0 = z0[hh * NP + lane], v1 = 0.0;
#pragma unroll
                                for (int q = 0; q < NP; q += 2) {
                                    if (q < N) v0 = fma((double)Pr[q], s_in[q], v0);
                                    if (q + 1 < N) v1 = fma((double)Pr[q + 1], s_in[q + 1], v1);
                                }
                                v = v0 + v1;
                            }
                            __syncwarp();
                            if (lane < N) s_in[lane] = v;
                            __syncwarp();
                        }
                    }
                    __syncthreads();
                }
                cp_async_wait<0>();
            }
        }
        __syncthreads();
        // inclusive state of this batch: root applied to s_in
        if (kb + 1 < p.nbps) {
            if (tid < N) {
                double v = (double)root[NP * RS + tid];
                for (int q = 0; q < N; ++q) v = fma((double)root[tid * RS + q], s_in[q], v);
                p.incl[(size_t)me * N + tid] = v;
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(p.flags + me, kFlagInc);
        }
        // down-sweep on states (FP64): left child <- parent's entry state,
        // right child <- left subtree's aggregate applied to it.
        for (int e = tid; e < Gp * NP; e += THREADS) st[e] = 0.0;
        __syncthreads();
        if (tid < NP) st[(size_t)(Gp - 1) * NP + tid] = s_in[tid];
        __syncthreads();
        for (int d = Gp / 2; d >= 1; d >>= 1) {
            const int npairs = Gp / (2 * d);
            for (int base = 0; base < npairs * NP; base += THREADS) {
                const int e = base + tid;
                const bool on = e < npairs * NP;
                const int m = e / NP;
                const int row = e - m * NP;
                const int j = 2 * d * m + 2 * d - 1;
                const int i = j - d;
                double v = 0.0;
                if (on) {
                    const T *Mi = maps + (size_t)i * MS;
                    const double *par = st + (size_t)j * NP;
                    v = (double)Mi[NP * RS + row];
#pragma unroll
                    for (int q = 0; q < NP; ++q) v = fma((double)Mi[row * RS + q], par[q], v);
                }
                __syncthreads();
                if (on) {
                    st[(size_t)i * NP + row] = st[(size_t)j * NP + row];
                    st[(size_t)j * NP + row] = v;
                }
                __syncthreads();
            }
        }

        // ------------------------------------------------------------ phase D
        // fix-up: one lane per chunk re-runs the chunk from its entry state
        if (N < NP)
            for (int e = tid; e < 2 * G * GS; e += THREADS)
                if ((e % GS) % NP >= N) Abuf[e] = T(0);
        const bool fix = tid < Gb;
#pragma unroll
        for (int i = 0; i < NP; ++i)
            h[state_slot<REV, NP>(i)] = (fix && i < N) ? (T)st[(size_t)tid * NP + i] : T(0);
        const bool ti = REV && p.gA && p.as_t == 0;
        __syncthreads();
        Loader<T, NP, REV>::load(p, vec, b, tb, Gb, 0, Abuf, ibuf, ybuf, REV);
        cp_async_commit();
        for (int w = 0; w < nwin; ++w) {
            const T *As = Abuf + (size_t)(w & 1) * G * GS;
            const T *xs = ibuf + (size_t)(w & 1) * G * W;
            const T *ys = ybuf + (size_t)(w & 1) * G * (W + NP);
            if (w + 1 < nwin)
                Loader<T, NP, REV>::load(p, vec, b, tb, Gb, w + 1, Abuf + (size_t)((w + 1) & 1) * G * GS,
                                         ibuf + (size_t)((w + 1) & 1) * G * W,
                                         ybuf + (size_t)((w + 1) & 1) * G * (W + NP), REV);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            if (fix) {
                const T *Ag = As + (size_t)tid * GS;
                const T *xg = xs + (size_t)tid * W;
                T *og = obuf + (size_t)tid * W;
#pragma unroll 1
                for (int blk = 0; blk < W / NP; ++blk) {
                    T o[NP];
#pragma unroll
                    for (int u = 0; u < NP; ++u) {
                        const int j = blk * NP + u;
                        const int slot = REV ? W - 1 - j : j;
                        T a[NP];
                        lds_row<T, NP>(a, Ag + (size_t)slot * NP);
                        if constexpr (NEG) {
#pragma unroll
                            for (int i = 0; i < NP; ++i) a[i] = -a[i];
                        }
                        if constexpr (REV) {
                            o[u] = step_scatter<T, NP>(a, h, u, xg[slot]);
                        } else {
                            h[u] = step_dot<T, NP>(a, h, u, xg[slot]);
                            o[u] = h[u];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < NP; ++u) og[blk * NP + u] = o[u];
                }
            }
            __syncthreads();
            // flush the window's outputs
            for (int e = tid; e < Gb * W; e += THREADS) {
                const int g = e / W;
                const int j = e - g * W;
                const int64_t pos = tb + (int64_t)g * p.L + (int64_t)w * W + j;  // step index
                if (pos < p.T) {
                    const int64_t t = REV ? p.T - 1 - pos : pos;
                    p.out[b * p.T + t] = obuf[e];
                } else if (REV && p.gzi && pos - p.T < N) {
                    // steps past t = 0 carry the adjoint into the initial conditions
                    p.gzi[b * N + (pos - p.T)] = obuf[e];
                }
            }
            if (REV && p.gA) {
                const T sgn = NEG ? T(1) : T(-1);
                if (!ti && vec && NP % V == 0) {
                    // rows t in [top-W, top-1] are contiguous: one 16-byte vector of
                    // taps per thread and step
                    constexpr int QR = NP / V;     // vectors per row
                    constexpr int QPC = W * QR;    // vectors per chunk window
                    using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
                    for (int e = tid; e < Gb * QPC; e += THREADS) {
                        const int g = e / QPC;
                        const int remg = e - g * QPC;
                        const int rr = remg / QR;  // row offset from the lowest time in the window
                        const int i0 = (remg - rr * QR) * V;
                        const int s = W - 1 - rr;
                        const int64_t pos = tb + (int64_t)g * p.L + (int64_t)w * W + s;
                        if (pos >= p.T) continue;
                        const int64_t t = p.T - 1 - pos;
                        const T gx = sgn * obuf[g * W + s];
                        const T *yq = ys + g * (W + NP) + s + i0;
                        VT o;
                        T *ov = reinterpret_cast<T *>(&o);
#pragma unroll
                        for (int j = 0; j < V; ++j) ov[j] = gx * yq[j];
                        *reinterpret_cast<VT *>(p.gA + (b * p.T + t) * NP + i0) = o;
                    }
                } else if (!ti) {
                    const int per = W * N;
                    for (int e = tid; e < Gb * per; e += THREADS) {
                        const int g = e / per;
                        const int remg = e - g * per;
                        const int rr = remg / N;
                        const int i = remg - rr * N;
                        const int s = W - 1 - rr;
                        const int64_t pos = tb + (int64_t)g * p.L + (int64_t)w * W + s;
                        if (pos >= p.T) continue;
                        const int64_t t = p.T - 1 - pos;
                        p.gA[(b * p.T + t) * N + i] = sgn * obuf[g * W + s] * ys[g * (W + NP) + s + i];
                    }
                } else {
                    // time-invariant coefficients: per-thread partial sums per tap, added atomically
                    for (int i = tid % NP; i < N; i += NP) {
                        T acc = T(0);
                        for (int e = tid / NP; e < Gb * W; e += THREADS / NP) {
                            const int g = e / W;
                            const int sl = e - g * W;
                            const int64_t pos = tb + (int64_t)g * p.L + (int64_t)w * W + sl;
                            if (pos < p.T) acc = fma(obuf[e], ys[g * (W + NP) + sl + i], acc);
                        }
                        if (acc != T(0)) atomicAdd(p.gA + b * N + i, sgn * acc);
                    }
                }
            }
            __syncthreads();
        }
        cp_async_wait<0>();
        // grad_zi entries beyond the padded steps of the signal's last chunk are
        // still pending in that chunk's exit state
        if (REV && p.gzi && kb + 1 == p.nbps && tid == Gb - 1) {
            const int64_t npad = tb + (int64_t)Gb * p.L - p.T;  // steps of the chunk with t < 0
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const int64_t k = npad + i;
                if (i < N && k < N) p.gzi[b * N + k] = h[state_slot<REV, NP>(i)];
            }
        }
    }
}

// ----------------------------------------------------------------------------
// Host side.
// ----------------------------------------------------------------------------
constexpr int kChunkLen = 128;   // target chunk length; rounded to a multiple of the window
constexpr int kMaxChunksPerBatch = 64;

inline int threads_for(int) { return 256; }
inline int window_for(int NP) { return NP * ((16 + NP - 1) / NP); }

struct Plan {
    int NP, G, L;
    int64_t nbps, nbatches;
};

// Chunks per batch: one group of N+1 lanes per chunk, capped so that the
// backward's shared memory fits two CTAs per SM (fp32) or one (fp64).
inline Plan make_plan(size_t esz, int64_t B, int64_t T, int64_t N) {
    Plan pl;
    pl.NP = padded_order(N);
    const int W = window_for(pl.NP);
    pl.L = W * ((kChunkLen + W - 1) / W);
    int G = (int)(threads_for(pl.NP) / (N + 1));
    if (G > kMaxChunksPerBatch) G = kMaxChunksPerBatch;
    const size_t budget = esz == 4 ? 110 * 1024 : 220 * 1024;
    while (G > 1 && SmemPlan(esz, pl.NP, W, G, (int)N, true).total > budget) --G;
    pl.G = G;
    const int64_t span = (int64_t)pl.G * pl.L;
    pl.nbps = (T + span - 1) / span;
    if (pl.nbps < 1) pl.nbps = 1;
    pl.nbatches = B * pl.nbps;
    return pl;
}

template <typename T, int NP, bool REV, bool NEG>
cudaError_t launch_np(ChunkParams<T> p, cudaStream_t st) {
    auto kern = chunked_kernel<T, NP, REV, NEG>;
    const SmemPlan S(sizeof(T), NP, Cfg<NP>::W, p.G, p.N, REV);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S.total);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg<NP>::THREADS, S.total);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > p.nbatches) grid = p.nbatches;
    kern<<<(unsigned)grid, Cfg<NP>::THREADS, S.total, st>>>(p);
    return cudaGetLastError();
}

template <typename T, bool REV, bool NEG>
cudaError_t dispatch(const ChunkParams<T> &p, int NP, cudaStream_t st) {
    if constexpr (NEG) {
        if (NP == 1) return launch_np<T, 1, REV, NEG>(p, st);
        return cudaErrorNotSupported;
    } else {
        switch (NP) {
#define LPCB_CASE(n) \
    case n: return launch_np<T, n, REV, NEG>(p, st);
            LPCB_FOR_EACH_NP(LPCB_CASE)
#undef LPCB_CASE
            default: return cudaErrorNotSupported;
        }
    }
}

template <typename T>
ChunkParams<T> base_params(const Plan &pl, int64_t B, int64_t T_, int64_t N, void *ws) {
    ChunkParams<T> p{};
    p.B = B;
    p.T = T_;
    p.N = (int)N;
    p.L = pl.L;
    p.G = pl.G;
    p.nbps = pl.nbps;
    p.nbatches = pl.nbatches;
    const WsLayout l = ws_layout(sizeof(T), pl.nbatches, N);
    unsigned char *w = static_cast<unsigned char *>(ws);
    p.counter = reinterpret_cast<unsigned *>(w);
    p.status = reinterpret_cast<unsigned *>(w) + 1;
    p.flags = reinterpret_cast<unsigned *>(w + l.flags);
    p.aggP = reinterpret_cast<T *>(w + l.aggP);
    p.aggz = reinterpret_cast<double *>(w + l.aggz);
    p.incl = reinterpret_cast<double *>(w + l.incl);
    p.spin_limit = 1u << 20;  // each poll is an L2 round trip: about a second in total
    return p;
}

}  // namespace

bool chunked_supported(int64_t N) { return N >= 1 && N <= 32; }

bool chunked_preferred(int64_t B, int64_t T, int64_t N, int64_t a_stride_t) {
    if (!chunked_supported(N) || a_stride_t == 0) return false;
    return T >= 4 * kChunkLen && B < 1024;
}

size_t chunked_forward_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t) {
    if (!chunked_supported(N)) return 0;
    const Plan pl = make_plan(esz, B, T, N);
    return ws_layout(esz, pl.nbatches, N).total;
}

size_t chunked_backward_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t a_stride_t) {
    return chunked_forward_workspace(esz, B, T, N, a_stride_t);
}

template <typename T>
cudaError_t chunked_forward(const FwdArgs<T> &a, bool neg, void *ws, size_t ws_bytes, cudaStream_t st) {
    const Plan pl = make_plan(sizeof(T), a.B, a.T, a.N);
    const WsLayout l = ws_layout(sizeof(T), pl.nbatches, a.N);
    if (ws_bytes < l.total) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(ws, 0, l.aggP, st);  // header + flags
    if (e != cudaSuccess) return e;
    ChunkParams<T> p = base_params<T>(pl, a.B, a.T, a.N, ws);
    p.in = a.x;
    p.A = a.A;
    p.as_b = a.a_stride_b;
    p.as_t = a.a_stride_t;
    p.zi = a.zi;
    p.out = a.y;
    return neg ? dispatch<T, false, true>(p, pl.NP, st) : dispatch<T, false, false>(p, pl.NP, st);
}

template <typename T>
cudaError_t chunked_backward(const BwdArgs<T> &a, bool neg, void *ws, size_t ws_bytes, cudaStream_t st) {
    const Plan pl = make_plan(sizeof(T), a.B, a.T, a.N);
    const WsLayout l = ws_layout(sizeof(T), pl.nbatches, a.N);
    if (ws_bytes < l.total) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(ws, 0, l.aggP, st);
    if (e != cudaSuccess) return e;
    if (a.gA && a.a_stride_t == 0) {
        e = cudaMemsetAsync(a.gA, 0, (size_t)a.B * a.N * sizeof(T), st);
        if (e != cudaSuccess) return e;
    }
    ChunkParams<T> p = base_params<T>(pl, a.B, a.T, a.N, ws);
    p.in = a.gy;
    p.A = a.A;
    p.as_b = a.a_stride_b;
    p.as_t = a.a_stride_t;
    p.zi = a.zi;
    p.ysave = a.y;
    p.out = a.gx;
    p.gA = a.gA;
    p.gzi = a.gzi;
    return neg ? dispatch<T, true, true>(p, pl.NP, st) : dispatch<T, true, false>(p, pl.NP, st);
}

template cudaError_t chunked_forward<float>(const FwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_forward<double>(const FwdArgs<double> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<float>(const BwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<double>(const BwdArgs<double> &, bool, void *, size_t, cudaStream_t);

}  // namespace lpcb
