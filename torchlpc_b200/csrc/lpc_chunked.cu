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
// The backward runs the same machinery over reversed time on grad_y with the
// diagonal coefficients A[t+1+i, i] (skewed into shared memory so a step's
// taps are contiguous) and fuses grad_A = -grad_x[t] * y[t-1-i] into the
// phase-D epilogue (time-invariant A: a per-CTA reduction added atomically);
// the CTA that owns t = 0 derives grad_zi from grad_x[0..N-1].
#include "lpc_chunked.cuh"

namespace lpcb {

namespace {

// ----------------------------------------------------------------------------
// Workspace layout and flags.
// ----------------------------------------------------------------------------
constexpr unsigned kFlagAgg = 1u;
constexpr unsigned kFlagInc = 2u;
constexpr int kHeaderBytes = 256;  // ticket counter, status word, padding
constexpr int kLookbackRing = 4;    // predecessor aggregates prefetched ahead of the composition

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
        lbP = off;  // look-back ring: predecessor aggregates in flight
        off += al((size_t)kLookbackRing * NP * NP * esz);
        lbz = off;
        off += al((size_t)kLookbackRing * NP * sizeof(double));
        misc = off;
        off += 64;
        total = off;
        (void)N;
    }
};

// ----------------------------------------------------------------------------
// Window loaders.  Window w of chunk g covers steps [w*W, w*W+W) of the chunk.
// Forward: step j of chunk g is time t = tb + g*L + j (tb: batch start).
// Backward: step j is reversed time tau = tb + g*L + j, i.e. t = T-1-tau.
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

    // Vector fast path: order equals the padded order, rows are dense and
    // 16-byte aligned, so every index below divides by a compile-time constant.
    __device__ static bool fast(const ChunkParams<T> &p) {
        return p.N == NP && p.as_t == NP && NP % V == 0 && (p.as_b * (int64_t)sizeof(T)) % 16 == 0 &&
               is_aligned16<T>(p.A);
    }

    __device__ static void load(const ChunkParams<T> &p, bool vec, int64_t b, int64_t tb, int Gb, int w,
                                T *As, T *xs, T *ys, bool with_y) {
        const int N = p.N;
        const int tid = threadIdx.x;
        const T *Ab = p.A + b * p.as_b;
        const T *inb = p.in + b * p.T;
        if (!REV) {
            if (vec) {
                constexpr int VPW = W * NP / V;  // vectors per chunk window
                for (int e = tid; e < Gb * VPW; e += THREADS) {
                    const int g = e / VPW;
                    const int v = e - g * VPW;
                    const int64_t t0 = tb + (int64_t)g * p.L + (int64_t)w * W;
                    T *dst = As + (size_t)g * GS + v * V;
                    const T *src = Ab + t0 * NP + v * V;
                    if (t0 + W <= p.T) {
                        cp_async<16>(dst, src);
                    } else {
#pragma unroll
                        for (int j = 0; j < V; ++j) {
                            const int64_t t = t0 + (v * V + j) / NP;
                            if (t < p.T)
                                cp_async<sizeof(T)>(dst + j, src + j);
                            else
                                dst[j] = T(0);
                        }
                    }
                }
            } else {
                const int per = W * N;
                for (int e = tid; e < Gb * per; e += THREADS) {
                    const int g = e / per;
                    const int rem = e - g * per;
                    const int r = rem / N;
                    const int i = rem - r * N;
                    const int64_t t = tb + (int64_t)g * p.L + (int64_t)w * W + r;
                    T *dst = As + (size_t)g * GS + r * NP + i;
                    if (t < p.T)
                        cp_async<sizeof(T)>(dst, Ab + t * p.as_t + i);
                    else
                        *dst = T(0);
                }
            }
            for (int e = tid; e < Gb * W; e += THREADS) {
                const int g = e / W;
                const int r = e - g * W;
                const int64_t t = tb + (int64_t)g * p.L + (int64_t)w * W + r;
                if (t < p.T)
                    cp_async<sizeof(T)>(xs + e, inb + t);
                else
                    xs[e] = T(0);
            }
        } else {
            // skewed diagonal: slot (s, i) <- A[top - s + i, i] (zero outside [0, T)),
            // top = T - (first reversed step of the window)
            if (vec) {
                constexpr int RV = NP / V;              // vectors per row
                constexpr int VPC = (W + NP - 1) * RV;  // vectors per chunk window
                for (int e = tid; e < Gb * VPC; e += THREADS) {
                    const int g = e / VPC;
                    const int rem = e - g * VPC;
                    const int q = rem / RV;
                    const int i0 = (rem - q * RV) * V;
                    const int64_t top = p.T - (tb + (int64_t)g * p.L + (int64_t)w * W);
                    const int64_t r = top - (W - 1) + q;
                    T *Ag = As + (size_t)g * GS;
                    const bool in_range = (r >= 0 && r < p.T);
                    const T *src = Ab + r * NP + i0;
#pragma unroll
                    for (int j = 0; j < V; ++j) {
                        const int i = i0 + j;
                        const int s = (int)(top - r) + i;
                        if (s < 0 || s >= W) continue;
                        if (in_range)
                            cp_async<sizeof(T)>(Ag + s * NP + i, src + j);
                        else
                            Ag[s * NP + i] = T(0);
                    }
                }
            } else {
                const int span = W + N - 1;
                const int per = span * N;
                for (int e = tid; e < Gb * per; e += THREADS) {
                    const int g = e / per;
                    const int rem = e - g * per;
                    const int q = rem / N;
                    const int i = rem - q * N;
                    const int64_t top = p.T - (tb + (int64_t)g * p.L + (int64_t)w * W);
                    const int64_t r = top - (W - 1) + q;
                    const int s = (int)(top - r) + i;
                    if (s < 0 || s >= W) continue;
                    T *dst = As + (size_t)g * GS + s * NP + i;
                    if (r >= 0 && r < p.T)
                        cp_async<sizeof(T)>(dst, Ab + r * p.as_t + i);
                    else
                        *dst = T(0);
                }
            }
            for (int e = tid; e < Gb * W; e += THREADS) {
                const int g = e / W;
                const int s = e - g * W;
                const int64_t t = p.T - 1 - (tb + (int64_t)g * p.L + (int64_t)w * W + s);
                if (t >= 0)
                    cp_async<sizeof(T)>(xs + e, inb + t);
                else
                    xs[e] = T(0);
            }
            if (with_y) {
                // ys[g][q] = ypad(top - 2 - q), q in [0, W + NP)
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
    }
};

// ----------------------------------------------------------------------------
// The kernel.
// ----------------------------------------------------------------------------
template <typename T, int NP, bool REV, bool NEG>
__global__ void __launch_bounds__(Cfg<NP>::THREADS, 4) chunked_kernel(ChunkParams<T> p) {
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
        for (int j = 0; j < NP; ++j) h[j] = (active && !xlane && j == NP - 1 - kk) ? T(1) : T(0);

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
                        T a[NP];
                        lds_row<T, NP>(a, Ag + (size_t)j * NP);
                        if constexpr (NEG) {
#pragma unroll
                            for (int i = 0; i < NP; ++i) a[i] = -a[i];
                        }
                        const T in = xlane ? xg[j] : T(0);
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
                    if (!xlane)
                        Mg[i * RS + kk] = h[NP - 1 - i];
                    else
                        Mg[NP * RS + i] = h[NP - 1 - i];
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
                } else {
                    if (tid < NP) {
                        double v = 0.0;
                        if (tid < N) v = p.incl[(size_t)(found * p.B + b) * N + tid];
                        s_in[tid] = v;
                    }
                    __syncwarp();
                    // compose the aggregates found+1 .. kb-1 in order; their data is
                    // pulled into a shared-memory ring kLookbackRing hops ahead
                    T *lbP = reinterpret_cast<T *>(smem + S.lbP);
                    double *lbz = reinterpret_cast<double *>(smem + S.lbz);
                    const int64_t m0 = found + 1;
                    const int64_t K = kb - m0;
                    auto fetch = [&](int64_t hop) {
                        if (hop < K) {
                            const int64_t idx = (m0 + hop) * p.B + b;
                            T *dP = lbP + (size_t)(hop % kLookbackRing) * NP * NP;
                            double *dz = lbz + (size_t)(hop % kLookbackRing) * NP;
                            for (int e = lane; e < N * N; e += 32) {
                                const int r = e / N, c = e - (e / N) * N;
                                cp_async<sizeof(T)>(dP + r * NP + c, p.aggP + (size_t)idx * N * N + e);
                            }
                            if (lane < N) cp_async<8>(dz + lane, p.aggz + (size_t)idx * N + lane);
                        }
                        cp_async_commit();
                    };
#pragma unroll
                    for (int hop = 0; hop < kLookbackRing; ++hop) fetch(hop);
                    for (int64_t hop = 0; hop < K; ++hop) {
                        cp_async_wait<kLookbackRing - 1>();
                        __syncwarp();
                        double v = 0.0;
                        if (lane < N) {
                            const T *Pr = lbP + (size_t)(hop % kLookbackRing) * NP * NP + lane * NP;
                            double v0 = lbz[(hop % kLookbackRing) * NP + lane], v1 = 0.0;
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
                        fetch(hop + kLookbackRing);
                    }
                    cp_async_wait<0>();
                }
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
        for (int i = 0; i < NP; ++i) h[NP - 1 - i] = (fix && i < N) ? (T)st[(size_t)tid * NP + i] : T(0);
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
#pragma unroll
                    for (int u = 0; u < NP; ++u) {
                        const int j = blk * NP + u;
                        T a[NP];
                        lds_row<T, NP>(a, Ag + (size_t)j * NP);
                        if constexpr (NEG) {
#pragma unroll
                            for (int i = 0; i < NP; ++i) a[i] = -a[i];
                        }
                        h[u] = step_dot<T, NP>(a, h, u, xg[j]);
                    }
#pragma unroll
                    for (int u = 0; u < NP; ++u) og[blk * NP + u] = h[u];
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
        // grad_zi from grad_x[0..N-1]: owned by the batch that contains t = 0
        if (REV && p.gzi && tb + (int64_t)Gb * p.L >= p.T) {
            __syncthreads();
            if (tid < N) {
                const int k = tid;
                const T *Ab = p.A + b * p.as_b;
                T acc = T(0);
                // grad_x[j] for j < T - tb was written by this CTA; beyond that
                // it is the batch's entry state (owned by the previous batch)
                const int64_t own = p.T - tb;
                for (int j = 0; j + k < N && j < p.T; ++j) {
                    const T gxj = j < own ? p.out[b * p.T + j] : (T)s_in[j - own];
                    acc = fma(Ab[j * p.as_t + j + k], gxj, acc);
                }
                p.gzi[b * N + k] = NEG ? acc : -acc;
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
