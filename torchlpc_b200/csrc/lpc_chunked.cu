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
//     shared memory with cp.async (double buffered, 16-byte vectors when the
//     rows allow) and read as broadcasts (one 16-byte shared load feeds every
//     lane of the chunk).  Half-way through, the lanes also store the map of
//     the chunk's first half.
//  B  a Blelloch tree over the G affine maps in shared memory: the batch
//     aggregate (up-sweep) and each chunk's exclusive prefix (down-sweep).
//  C  decoupled look-back over the predecessor batches of the same signal:
//     the aggregate is published, predecessors' aggregates are staged into
//     shared memory and composed in FP64 until an inclusive state is found,
//     the batch's inclusive state is published (FP64).  Every wait is
//     bounded; on expiry the kernel records a bit in the workspace status
//     word and moves on.
//  D  fix-up: one lane per half-chunk re-runs it from its exact entry state
//     (second halves start from the first half's map applied to the chunk's
//     entry state, in FP64); the coefficient windows are streamed again (they
//     are L2-resident by then) and the CTA writes the outputs back coalesced.
//
// The backward runs the same machinery over reversed time on grad_y: the
// adjoint recurrence grad_x[t] = grad_y[t] - sum_i A[t+1+i,i] grad_x[t+1+i] in
// transposed (scatter) form, where producing grad_x[t] adds -A[t,i]*grad_x[t]
// to the pending accumulator of output t-1-i.  Its state is the N pending
// accumulators and each step reads one contiguous row A[t,:], so both
// directions stream the same row windows.  grad_A = -grad_x[t] * y[t-1-i] is
// fused into the phase-D epilogue (time-invariant A: a separate reduction
// kernel over the grad_x just written); grad_zi is the adjoint carried N steps
// past t = 0.
#include <atomic>

#include "lpc_chunked.cuh"
#include "lpc_ti.cuh"

namespace lpcb {

namespace {

// ----------------------------------------------------------------------------
// Workspace layout and flags.
// ----------------------------------------------------------------------------
constexpr unsigned kFlagAgg = 1u;
constexpr unsigned kFlagInc = 2u;
constexpr int kHeaderBytes = 256;  // ticket counter, status word, padding
// Predecessor aggregates staged per round of the look-back composition
// (about 4 KB of coefficients per round).
__host__ __device__ constexpr int lookback_hops(int NP, int esz) {
    return 4096 / (NP * NP * esz) < 2 ? 2 : (4096 / (NP * NP * esz) > 8 ? 8 : 4096 / (NP * NP * esz));
}

// Window loaders: per-element cp.async (any layout) or 16-byte cp.async per
// vector (dense rows of the padded order, 16-byte rows and windows, 16-byte
// aligned signal starts).
constexpr int kLoadElem = 0;
constexpr int kLoadVec = 1;

// Status bits a bounded wait records before giving up.
constexpr unsigned kStatusFlagWait = 1u;     // a predecessor's flag never appeared
constexpr unsigned kStatusNoInclusive = 2u;  // look-back ran past batch 0 (cannot happen)

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// A published aggregate is stored padded to the padded order: P as NP rows of
// NP (zeros beyond N), z as NP doubles, each record a multiple of 16 bytes so
// that it can be moved with 16-byte vector loads.
__host__ __device__ constexpr int agg_p_elems(int NP, int esz) {
    return ((NP * NP * esz + 15) / 16) * 16 / esz;
}
__host__ __device__ constexpr int agg_z_elems(int NP) { return ((NP * 8 + 15) / 16) * 2; }

struct WsLayout {
    size_t flags, aggP, aggz, incl, total;
};

inline WsLayout ws_layout(size_t esz, int64_t nbatches, int64_t N) {
    const int NP = padded_order(N);
    WsLayout l;
    size_t off = kHeaderBytes;
    l.flags = off;
    off = align256(off + (size_t)nbatches * 4);
    l.aggP = off;
    off = align256(off + (size_t)nbatches * agg_p_elems(NP, (int)esz) * esz);
    l.aggz = off;
    off = align256(off + (size_t)nbatches * agg_z_elems(NP) * 8);
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
    // Boundary-state checkpointing (forward only).  The exact entry state of
    // every half-chunk (N values, s[i] = y[t0-1-i]) is written to ckpt at
    // ((batch * 2G + half-chunk) * N + i) (batch: physical index, see
    // Sig::pb; half-chunk 2g, 2g+1: the lower and upper half of chunk g).
    // With fixonly set, the kernel instead reads those states and runs only
    // the exact pass (phase D) of every half-chunk: y is recomputed with no
    // map, tree or look-back work and no waits.
    F *ckpt;
    int fixonly;
    int64_t B, T, as_b, as_t;
    int N;
    int L;           // chunk length (multiple of the window)
    int G;           // chunks per batch
    int loader;      // window loader: kLoadElem or kLoadVec
    int64_t nbps;    // batches per signal
    int64_t nbatches;
    const int64_t *roff;  // ragged: signal offsets (nsig+1) into x/y (nullptr: uniform B x T)
    int64_t *bb;          // ragged: first batch of each signal (nsig+1, in the workspace)
    int64_t nsig;
    unsigned *counter, *status, *flags;
    F *aggP;         // [nbatches][agg_p_elems]
    double *aggz;    // [nbatches][agg_z_elems]
    double *incl;    // [nbatches][N]
    unsigned spin_limit;
    // Process-wide error word (device-visible, e.g. mapped pinned host memory)
    // that a CTA finishing with a nonzero status word ORs that status into,
    // so the caller learns of a bounded wait that gave up without reading the
    // workspace; nullptr: not reported beyond the workspace.
    unsigned *err_word;
};

// The signal a batch belongs to.
struct Sig {
    int64_t T;       // samples
    int64_t xo;      // offset of sample 0 in x, y, grad_y, grad_x (grad_A rows: xo * N)
    int64_t ao;      // offset of row 0 in A
    int64_t zo;      // offset in zi and grad_zi
    int64_t kb, nb;  // this batch's index in scan order (backward: from the top), batches of the signal
    int64_t fb, fs;  // workspace index of batch m (scan order) of the signal: fb + m * fs
    int64_t pb;      // physical index of the signal's first batch (checkpoint states)
    int vx;          // input windows move as 16-byte vectors
};

// Steps per phase-A window (phase D: half of it): orders up to 16 stage 32
// steps per barrier, larger orders 16+ steps (measured on B200: the longer
// window shortens the backward by ~11 % at order 16 and slows order 24).
// Two CTAs per SM up to order 24 (fp32), three above.
__host__ __device__ constexpr int window_steps(int NP) {
    return (NP <= 16 ? 2 : 1) * NP * ((16 + NP - 1) / NP);
}
__host__ __device__ constexpr int ctas_per_sm(int NP, int esz) { return esz == 4 && NP > 24 ? 3 : 2; }
// Phase-D (exact pass) windows: half the phase-A window, in fix_stages
// stages (loads issued fix_stages - 1 windows ahead).  Measured on B200 at
// order 16: quarter-length windows in four stages (the same shared memory)
// made the pass 1.45x slower; its time follows the number of windows, not
// the distance the loads run ahead.
__host__ __device__ constexpr int fix_window(int NP) { return window_steps(NP) / 2; }
__host__ __device__ constexpr int fix_stages(int) { return 2; }

template <int NP>
struct Cfg {
    static constexpr int THREADS = 256;
    static constexpr int W = window_steps(NP);  // phase-A window: steps, a multiple of NP
    static constexpr int WD = fix_window(NP);   // phase-D window (half-chunks)
    static constexpr int DS = fix_stages(NP);   // phase-D stages in flight
};

// Per-chunk stride of a coefficient window in shared memory: WC rows of NP
// plus one 16-byte pad so that the rows different chunks read in the same
// step fall in different banks.
__host__ __device__ constexpr int group_stride(int WC, int NP, int esz) { return WC * NP + 16 / esz; }
// Row stride of a stored affine map (16-byte aligned, padded against bank conflicts).
__host__ __device__ constexpr int map_row_stride(int NP, int esz) {
    return ((NP + 16 / esz - 1) / (16 / esz)) * (16 / esz) + 16 / esz;
}
__host__ __device__ constexpr int map_stride(int NP, int esz) {
    return NP * map_row_stride(NP, esz) + ((NP + 16 / esz - 1) / (16 / esz)) * (16 / esz);
}
// Half-chunk map (P rows of NP, then z), padded to 16 bytes.
__host__ __device__ constexpr int half_map_elems(int NP, int esz) {
    return ((NP * NP + NP) * esz + 15) / 16 * 16 / esz;
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

// step_dot with the input selected by a 0/1 factor: xsel * xv - sum, one FMA
// in place of a select and a subtraction (xsel*xv is exact for 0 and 1).
template <typename T, int NP>
__device__ __forceinline__ T step_dot_sel(const T (&a)[NP], const T (&h)[NP], int u, T xsel, T xv) {
    if constexpr (NP == 1) {
        return fma(-a[0], h[(u - 1 + NP) % NP], xsel * xv);
    } else {
        T p0 = T(0), p1 = T(0);
#pragma unroll
        for (int i = NP - 1; i >= 1; --i) {
            if ((i & 1) == 0)
                p0 = fma(a[i], h[(u - 1 - i + 2 * NP) % NP], p0);
            else
                p1 = fma(a[i], h[(u - 1 - i + 2 * NP) % NP], p1);
        }
        const T acc = fma(xsel, xv, -(p0 + p1));
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

// step_scatter with the input selected by a 0/1 factor (one FMA).
template <typename T, int NP>
__device__ __forceinline__ void step_scatter_sel(const T (&a)[NP], T (&c)[NP], int u, T xsel, T xv) {
    const T g = fma(xsel, xv, c[u]);
    c[u] = T(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) c[(u + 1 + i) % NP] = fma(-a[i], g, c[(u + 1 + i) % NP]);
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

// Shared-memory plan (bytes), all regions 16-byte aligned.  The window
// buffers of phases A and D alias the tree maps and the look-back stage:
// phases B and C run between the two window loops.
struct SmemPlan {
    size_t abuf, ibuf, obuf, ybuf, maps, half, st, sin, lbP, lbz, misc, total;
    __host__ __device__ SmemPlan(size_t esz, int NP, int G, bool rev) {
        auto al = [](size_t v) { return (v + 15) & ~size_t(15); };
        const int W = window_steps(NP), WD = fix_window(NP), DS = fix_stages(NP);
        size_t off = 0;
        abuf = off;
        const size_t awin = al((size_t)2 * G * group_stride(W, NP, (int)esz) * esz);
        const size_t dwin = al((size_t)DS * 2 * G * group_stride(WD, NP, (int)esz) * esz);
        int Gp = 1;
        while (Gp < G) Gp <<= 1;
        const size_t mapbytes = al((size_t)Gp * map_stride(NP, (int)esz) * esz);
        const int KL = lookback_hops(NP, (int)esz);
        const size_t lbPbytes = al((size_t)2 * KL * agg_p_elems(NP, (int)esz) * esz);
        const size_t lbzbytes = al((size_t)2 * KL * agg_z_elems(NP) * sizeof(double));
        maps = off;
        lbP = off + mapbytes;
        lbz = lbP + lbPbytes;
        size_t r = mapbytes + lbPbytes + lbzbytes;
        if (awin > r) r = awin;
        if (dwin > r) r = dwin;
        off += al(r);
        ibuf = off;  // inputs: 2 stages x G x W (= DS stages x 2G x WD: DS = 2, WD = W / 2)
        off += al((size_t)2 * G * W * esz);
        obuf = off;  // phase-D outputs of one window
        off += al((size_t)2 * G * WD * esz);
        ybuf = off;  // backward: lagged outputs y of the phase-D windows
        if (rev) off += al((size_t)DS * 2 * G * (WD + NP) * esz);
        half = off;  // map over the first half of each chunk
        off += al((size_t)G * half_map_elems(NP, (int)esz) * esz);
        st = off;  // FP64 entry states of the tree nodes
        off += al((size_t)Gp * NP * sizeof(double));
        sin = off;
        off += al((size_t)NP * sizeof(double));
        misc = off;  // ticket, the batch's signal
        off += 128;
        total = off;
    }
};

// ----------------------------------------------------------------------------
// Window loaders.  Both directions cut a signal on the same grid: chunk g of
// a batch starting at sample tb covers samples [tb + g*Lc, tb + (g+1)*Lc).
// Window w (WC steps) of chunk g holds WC consecutive coefficient rows in
// natural order, slot j <-> row row0 + j:
//   forward traversal (REV false): row0 = tb + g*Lc + w*WC;
//   reverse traversal (REV true):  row0 = tb + (g+1)*Lc - (w+1)*WC, the
//   window w*WC rows below the chunk's top (steps run from slot WC-1 down).
// Rows at or past the end of the signal read as zero (the last chunk of a
// signal may be partial).  Reverse windows also carry the lagged outputs
// ys[g][r] = ypad(row0-NP+r), r in [0, WC+NP), with ypad(-1-k) = zi[k] (zero
// past k = N-1) and zero past the end of the signal.
// ----------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool is_aligned16(const void *p) {
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

template <typename T, int NP, bool REV, int WC>
struct Loader {
    static constexpr int THREADS = Cfg<NP>::THREADS;
    static constexpr int GS = group_stride(WC, NP, sizeof(T));
    static constexpr int PY = WC + NP;
    // rows, input windows and lagged-output windows are whole 16-byte vectors
    static constexpr bool FLAT_OK = (NP * sizeof(T)) % 16 == 0 && (WC * sizeof(T)) % 16 == 0 && (PY * sizeof(T)) % 16 == 0;

    // First row held by slot 0 of chunk g's window w, and the valid slot range.
    __device__ static void rows(const Sig &sg, int64_t tb, int Lc, int g, int w, int64_t &row0, int &lo,
                                int &hi) {
        row0 = REV ? tb + (int64_t)(g + 1) * Lc - (int64_t)(w + 1) * WC : tb + (int64_t)g * Lc + (int64_t)w * WC;
        lo = 0;
        hi = (int)max64(0, min64(WC, sg.T - row0));
    }

    // Vector path: one warp per chunk (chunks warp, warp + 8, ...), so the
    // row range of a chunk's window is computed once per warp; the chunk's
    // rows are one contiguous run in global and shared memory, lane l moving
    // vectors l, l+32, ...  Inputs and lagged outputs follow on the low lanes.
    // The caller commits the group.
    __device__ static void load_vec(const ChunkParams<T> &p, const Sig &sg, int64_t tb, int Gc, int Lc, int w,
                                    T *As, T *xs, T *ys, bool with_y, int lw0, int nlw) {
        constexpr int V = 16 / sizeof(T);
        constexpr int RV = NP / V > 0 ? NP / V : 1;  // vectors per row
        constexpr int AV = WC * RV;                  // coefficient vectors per chunk window
        constexpr int XV = WC / V > 0 ? WC / V : 1;  // input vectors
        constexpr int YV = PY / V;                   // lagged-output vectors
        constexpr int NWARP = THREADS / 32;
        using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
        const int lane = threadIdx.x & 31;
        const int nyv = (xs && REV && with_y) ? YV : 0;
        const int nio = xs ? XV + nyv : 0;  // input-side vectors per chunk
        const T *Ab = p.A + sg.ao;
        const T *inb = p.in + sg.xo;
        const VT zero = {};
        for (int g = (int)(threadIdx.x >> 5) - lw0; g < Gc; g += nlw) {
            int64_t row0;
            int lo, hi;
            rows(sg, tb, Lc, g, w, row0, lo, hi);
            T *dA = As + (size_t)g * GS;
            if (lo == 0 && hi == WC) {
                const T *sA = Ab + row0 * NP;
#pragma unroll
                for (int k = 0; k < (AV + 31) / 32; ++k) {
                    const int v = lane + 32 * k;
                    if (AV % 32 == 0 || v < AV) cp_async<16>(dA + v * V, sA + v * V);
                }
            } else {
                for (int v = lane; v < AV; v += 32) {
                    const int r = v / RV;
                    if (r >= lo && r < hi)
                        cp_async<16>(dA + v * V, Ab + (row0 + r) * NP + (v - r * RV) * V);
                    else
                        *reinterpret_cast<VT *>(dA + v * V) = zero;
                }
            }
            for (int v = lane; v < nio; v += 32) {
                if (v < XV) {
                    const int r = v * V;  // lo, hi and r are multiples of V
                    T *dst = xs + (size_t)g * WC + r;
                    if (r >= lo && r < hi)
                        cp_async<16>(dst, inb + row0 + r);
                    else
                        *reinterpret_cast<VT *>(dst) = zero;
                } else {
                    const int r = (v - XV) * V;
                    T *dst = ys + (size_t)g * PY + r;
                    const int64_t j0 = row0 - NP + r;  // a multiple of V: all or none of the vector is before t = 0
                    if (j0 >= sg.T) {  // T is a multiple of V here: all of the vector is past the end
                        *reinterpret_cast<VT *>(dst) = zero;
                    } else if (j0 >= 0) {
                        cp_async<16>(dst, p.ysave + sg.xo + j0);
                    } else {
                        const T *zib = p.zi ? p.zi + sg.zo : nullptr;
#pragma unroll
                        for (int j = 0; j < V; ++j) {
                            const int64_t k = -1 - (j0 + j);
                            dst[j] = (k >= 0 && k < p.N && zib) ? zib[k] : T(0);
                        }
                    }
                }
            }
        }
    }

    // Flat path for a batch wholly inside its signal with 16-byte vectors
    // (rows, inputs and, backward, lagged outputs that start at or after
    // t = 0): threads lt, lt + nlt, ... take the vectors of the window set in
    // turn, with no per-window range checks.  The caller commits the group.
    __device__ static void load_flat(const ChunkParams<T> &p, const Sig &sg, int64_t tb, int Gc, int Lc, int w,
                                     T *As, T *xs, T *ys, bool with_y, int lt, int nlt) {
        if constexpr (FLAT_OK) {
        constexpr int V = 16 / sizeof(T);
        constexpr int RV = NP / V;   // vectors per row (16-byte rows on this path)
        constexpr int AV = WC * RV;  // coefficient vectors per chunk window
        constexpr int XV = WC / V;   // input vectors per chunk window
        constexpr int YV = PY / V;   // lagged-output vectors per chunk window
        const T *Ab = p.A + sg.ao;
        const T *inb = p.in + sg.xo;
        // first row of chunk g's window: forward tb + g*Lc + w*WC, backward
        // tb + (g+1)*Lc - (w+1)*WC
        const int64_t r00 = REV ? tb + Lc - (int64_t)(w + 1) * WC : tb + (int64_t)w * WC;
        for (int v = lt; v < Gc * AV; v += nlt) {
            const int g = v / AV;
            const int r = v - g * AV;
            cp_async<16>(As + (size_t)g * GS + r * V, Ab + (r00 + (int64_t)g * Lc) * NP + r * V);
        }
        for (int v = lt; v < Gc * XV; v += nlt) {
            const int g = v / XV;
            const int r = v - g * XV;
            cp_async<16>(xs + (size_t)g * WC + r * V, inb + r00 + (int64_t)g * Lc + r * V);
        }
        if (REV && with_y) {
            const T *yb = p.ysave + sg.xo;
            for (int v = lt; v < Gc * YV; v += nlt) {
                const int g = v / YV;
                const int r = v - g * YV;
                cp_async<16>(ys + (size_t)g * PY + r * V, yb + r00 + (int64_t)g * Lc - NP + r * V);
            }
        }
        }
    }

    // Element path (any stride and alignment): one warp per chunk, one
    // cp.async per element.  The caller commits the group.
    __device__ static void load_elem(const ChunkParams<T> &p, const Sig &sg, int64_t tb, int Gc, int Lc, int w,
                                     T *As, T *xs, T *ys, bool with_y, bool rows_too, int lw0, int nlw) {
        constexpr int NWARP = THREADS / 32;
        const int N = p.N;
        const int lane = threadIdx.x & 31;
        const T *Ab = p.A + sg.ao;
        const T *inb = p.in + sg.xo;
        const T *zib = p.zi ? p.zi + sg.zo : nullptr;
        for (int g = (int)(threadIdx.x >> 5) - lw0; g < Gc; g += nlw) {
            int64_t row0;
            int lo, hi;
            rows(sg, tb, Lc, g, w, row0, lo, hi);
            if (rows_too) {
                // element e of the window is tap e % NP of row e / NP (a
                // compile-time divisor); taps N..NP-1 keep the zeros filled per batch
                T *dA = As + (size_t)g * GS;
                for (int e = lane; e < WC * NP; e += 32) {
                    const int r = e / NP;
                    const int i = e - r * NP;
                    if (i >= N) continue;
                    if (r >= lo && r < hi)
                        cp_async<sizeof(T)>(dA + e, Ab + (row0 + r) * p.as_t + i);
                    else
                        dA[e] = T(0);
                }
            }
            // inputs (x forward, grad_y backward), slot r <-> index row0 + r
            for (int r = lane; r < WC; r += 32) {
                T *dst = xs + (size_t)g * WC + r;
                if (r >= lo && r < hi)
                    cp_async<sizeof(T)>(dst, inb + row0 + r);
                else
                    *dst = T(0);
            }
            if (REV && with_y) {
                for (int r = lane; r < PY; r += 32) {
                    const int64_t j = row0 - NP + r;
                    T *dst = ys + (size_t)g * PY + r;
                    if (j >= sg.T)
                        *dst = T(0);
                    else if (j >= 0)
                        cp_async<sizeof(T)>(dst, p.ysave + sg.xo + j);
                    else if (-1 - j < N && zib)
                        *dst = zib[-1 - j];
                    else
                        *dst = T(0);
                }
            }
        }
    }

    // Vector rows and inputs when both allow it; vector rows with element
    // inputs when only the signal start or length is unaligned.  Called by
    // warps lw0 .. lw0+nlw-1 (every warp of the CTA by default), which share
    // the chunks among them; PART false fixes them at compile time (every
    // warp), which keeps the index arithmetic out of the registers of the
    // large-order instances.
    template <bool PART = false>
    __device__ static void load(const ChunkParams<T> &p, const Sig &sg, int64_t tb, int Gc, int Lc, int w, T *As,
                                T *xs, T *ys, bool with_y, int lw0_ = 0, int nlw_ = THREADS / 32) {
        const int lw0 = PART ? lw0_ : 0;
        const int nlw = PART ? nlw_ : THREADS / 32;
        if (p.loader == kLoadVec && sg.vx) {
            load_vec(p, sg, tb, Gc, Lc, w, As, xs, ys, with_y, lw0, nlw);
        } else if (p.loader == kLoadVec) {
            load_vec(p, sg, tb, Gc, Lc, w, As, nullptr, nullptr, false, lw0, nlw);
            load_elem(p, sg, tb, Gc, Lc, w, As, xs, ys, with_y, false, lw0, nlw);
        } else {
            load_elem(p, sg, tb, Gc, Lc, w, As, xs, ys, with_y, true, lw0, nlw);
        }
    }
};

// Phase A: NS steps of one window segment of a chunk-map lane running KF
// filters (ring positions U0..U0+NS-1), slots jbase.. of the window.  Bit q of
// xmask marks filter q as the zero-state filter (the one fed the input).  One
// broadcast load of a coefficient row feeds all KF filters of the lane.  The
// backward runs the adjoint recurrence in transposed form over reversed time
// (its maps come out as adjoint maps directly; the same maps built from
// forward basis filters accumulated against grad_y lose up to two orders of
// magnitude of accuracy in grad_x for strongly non-normal filters).
template <typename T, int NP, int KF, bool REV, bool NEG, int WC, int U0, int NS>
__device__ __forceinline__ void map_steps(const T *Ag, const T *xg, unsigned xmask, int jbase, T (&h)[KF][NP]) {
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const int u = (U0 + j) % NP;
        const int jj = jbase + j;
        const int slot = REV ? WC - 1 - jj : jj;
        T a[NP];
        lds_row<T, NP>(a, Ag + (size_t)slot * NP);
        if constexpr (NEG) {
#pragma unroll
            for (int i = 0; i < NP; ++i) a[i] = -a[i];
        }
        if constexpr (NP <= 16) {
            // every lane reads the input (a broadcast within the chunk); only
            // the zero-state filter takes it, through a 0/1 factor (measured
            // on B200 at order 16: forward 7 %, backward 4 % faster than a
            // select; order 24 keeps the select)
            const T xv = xg[slot];
#pragma unroll
            for (int q = 0; q < KF; ++q) {
                const T xsel = ((xmask >> q) & 1u) ? T(1) : T(0);
                if constexpr (REV)
                    step_scatter_sel<T, NP>(a, h[q], u, xsel, xv);
                else
                    h[q][u] = step_dot_sel<T, NP>(a, h[q], u, xsel, xv);
            }
        } else {
            const T xv = xmask ? xg[slot] : T(0);
#pragma unroll
            for (int q = 0; q < KF; ++q) {
                const T in = ((xmask >> q) & 1u) ? xv : T(0);
                if constexpr (REV)
                    step_scatter<T, NP>(a, h[q], u, in);
                else
                    h[q][u] = step_dot<T, NP>(a, h[q], u, in);
            }
        }
    }
}

// Filters per phase-A lane: two at orders 8..24, where one 16-byte broadcast
// row load per step otherwise feeds a single recurrence and the shared-memory
// wavefronts (one per coefficient and warp) bound the phase.  Orders 20 and 24
// run two CTAs per SM with the full register file (measured on B200 at order
// 24 against three CTAs of 80 registers with one filter per lane, whose
// spills dominated: forward 7 %, backward 5 % faster on 64 x 16000, ragged
// 1024-signal batch 10 % faster).
__host__ __device__ constexpr int filters_per_lane(int NP) { return NP >= 8 && NP <= 24 ? 2 : 1; }

// Stores the state of filter f of a chunk into an affine map laid out as NP
// rows of stride rs then z: basis filter f < N is column f of P, the
// zero-state filter f == N is z; f > N (an idle filter slot) stores nothing.
template <typename T, int NP, bool REV>
__device__ __forceinline__ void put_map_column(T *M, int rs, const T (&h)[NP], int f, int N) {
    if (f > N) return;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        if (i < N) {
            const T v = h[state_slot<REV, NP>(i)];
            if (f < N)
                M[i * rs + f] = v;
            else
                M[NP * rs + i] = v;
        }
    }
}

// Phase D: NS steps of the exact filter for one half-chunk, outputs to og.
template <typename T, int NP, bool REV, bool NEG, int WC, int U0, int NS>
__device__ __forceinline__ void fix_steps(const T *Ag, const T *xg, T *og, int jbase, T (&h)[NP]) {
    T o[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        const int u = (U0 + j) % NP;
        const int jj = jbase + j;
        const int slot = REV ? WC - 1 - jj : jj;
        T a[NP];
        lds_row<T, NP>(a, Ag + (size_t)slot * NP);
        if constexpr (NEG) {
#pragma unroll
            for (int i = 0; i < NP; ++i) a[i] = -a[i];
        }
        if constexpr (REV) {
            o[j] = step_scatter<T, NP>(a, h, u, xg[slot]);
        } else {
            h[u] = step_dot<T, NP>(a, h, u, xg[slot]);
            o[j] = h[u];
        }
    }
#pragma unroll
    for (int j = 0; j < NS; ++j) og[jbase + j] = o[j];
}

// ----------------------------------------------------------------------------
// The kernel.
// ----------------------------------------------------------------------------
template <typename T, int NP, bool REV, bool NEG>
__global__ void __launch_bounds__(Cfg<NP>::THREADS, NP <= 24 ? 2 : 3) chunked_kernel(ChunkParams<T> p) {
    constexpr int W = Cfg<NP>::W;
    constexpr int WD = Cfg<NP>::WD;
    constexpr int DS = Cfg<NP>::DS;
    constexpr int THREADS = Cfg<NP>::THREADS;
    constexpr int V = 16 / sizeof(T);
    constexpr int GSA = group_stride(W, NP, sizeof(T));
    constexpr int GSD = group_stride(WD, NP, sizeof(T));
    constexpr int RS = map_row_stride(NP, sizeof(T));
    constexpr int MS = map_stride(NP, sizeof(T));
    constexpr int PYD = WD + NP;
    constexpr int PSE = agg_p_elems(NP, sizeof(T));
    constexpr int ZSE = agg_z_elems(NP);
    constexpr int HME = half_map_elems(NP, sizeof(T));
    constexpr int KL = lookback_hops(NP, sizeof(T));
    using LA = Loader<T, NP, REV, W>;
    using LD = Loader<T, NP, REV, WD>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int N = p.N;
    const int G = p.G;
    const int L = p.L;
    const int LH = L / 2;  // phase D runs on half-chunks
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const SmemPlan S(sizeof(T), NP, G, REV);
    T *Abuf = reinterpret_cast<T *>(smem + S.abuf);
    T *ibuf = reinterpret_cast<T *>(smem + S.ibuf);
    T *obuf = reinterpret_cast<T *>(smem + S.obuf);
    T *ybuf = reinterpret_cast<T *>(smem + S.ybuf);
    T *maps = reinterpret_cast<T *>(smem + S.maps);  // [Gp][NP rows of RS | z]
    T *lbP = reinterpret_cast<T *>(smem + S.lbP);    // [2][KL][PSE]
    double *lbz = reinterpret_cast<double *>(smem + S.lbz);  // [2][KL][ZSE]
    // [G][HME]: map of the first half of each chunk in scan order (forward:
    // the lower half, backward: the upper half), P[i][k] then z
    T *hmap = reinterpret_cast<T *>(smem + S.half);
    double *st = reinterpret_cast<double *>(smem + S.st);    // [Gp][NP]
    double *s_in = reinterpret_cast<double *>(smem + S.sin); // [NP]
    int64_t *misc = reinterpret_cast<int64_t *>(smem + S.misc);
    int Gp = 1;
    while (Gp < G) Gp <<= 1;

    constexpr int KF = filters_per_lane(NP);
    const int TPC = (N + KF) / KF;  // phase-A lanes per chunk: N+1 filters, KF per lane
    const int grp = tid / TPC;
    const int kk = tid - grp * TPC;  // lane kk runs filters kk*KF .. kk*KF+KF-1
    const int warp = tid >> 5;
    const int aw = (G * TPC + 31) / 32;  // warps holding phase-A lanes
    const int nwin = L / W;  // phase-A windows per chunk
    const int64_t nbatches = p.roff ? p.bb[p.nsig] : p.nbatches;
    Sig *sgs = reinterpret_cast<Sig *>(misc + 1);

    // entries of the half maps beyond order N stay zero for the whole launch
    for (int e = tid; e < G * HME; e += THREADS) hmap[e] = T(0);

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const int64_t t = (int64_t)atomicAdd(p.counter, 1u);
            misc[0] = t;
            if (t < nbatches) {
                Sig q;
                if (p.roff) {
                    // ragged: batches are numbered signal by signal; find the
                    // signal whose range of batches holds the ticket
                    int64_t lo = 0, hi = p.nsig;  // bb[lo] <= t < bb[hi]
                    while (hi - lo > 1) {
                        const int64_t mid = (lo + hi) / 2;
                        if (p.bb[mid] <= t) lo = mid; else hi = mid;
                    }
                    q.T = p.roff[lo + 1] - p.roff[lo];
                    q.xo = p.roff[lo];
                    q.ao = p.roff[lo] * p.as_t;
                    q.zo = lo * N;
                    q.kb = t - p.bb[lo];
                    q.nb = p.bb[lo + 1] - p.bb[lo];
                    q.fb = p.bb[lo];
                    q.fs = 1;
                    q.pb = p.bb[lo];
                } else {
                    // uniform: batch kb of every signal before batch kb+1 of any
                    const int64_t b = t % p.B;
                    q.T = p.T;
                    q.xo = b * p.T;
                    q.ao = b * p.as_b;
                    q.zo = b * N;
                    q.kb = t / p.B;
                    q.nb = p.nbps;
                    q.fb = b;
                    q.fs = p.B;
                    q.pb = b * p.nbps;
                }
                // vector input windows need an aligned signal start and a
                // length of whole vectors (a window's last vector must not
                // reach past the signal)
                q.vx = (WD * (int)sizeof(T)) % 16 == 0 && (q.T * (int64_t)sizeof(T)) % 16 == 0 &&
                       is_aligned16<T>(p.in + q.xo) && (!p.ysave || is_aligned16<T>(p.ysave + q.xo));
                *sgs = q;
            }
        }
        __syncthreads();
        const int64_t ticket = misc[0];
        if (ticket >= nbatches) {
            if (tid == 0 && p.err_word) {
                // this CTA's own give-ups are in the status word by now
                const unsigned st_now = ld_acquire(p.status);
                if (st_now) {
                    volatile unsigned *ew = p.err_word;
                    *ew = *ew | st_now;
                }
            }
            break;
        }
        const Sig sg = *sgs;
        // scan order: the forward walks a signal's batches from its start, the
        // backward from its end; both cut the signal on the same grid
        const int64_t kb = sg.kb;                      // batch index in scan order
        const int64_t jb = REV ? sg.nb - 1 - kb : kb;  // batch index from the signal's start
        const int64_t tb = jb * (int64_t)G * L;        // first sample of the batch
        const int64_t rem = sg.T - tb;
        const int Gb = (int)min64(G, (rem + L - 1) / L);

        // ------------------------------------------------------------ phase A
        // chunk maps: N basis filters + one zero-state filter per chunk, in
        // scan order (backward: the adjoint recurrence over reversed time)
        if (p.loader == kLoadElem && N < NP)  // padded coefficient columns must read as zero
            for (int e = tid; e < 2 * G * GSA; e += THREADS)
                if ((e % GSA) % NP >= N) Abuf[e] = T(0);
        const bool active = grp < Gb && !p.fixonly;
        unsigned xmask = 0;
        T h[KF][NP];
#pragma unroll
        for (int q = 0; q < KF; ++q) {
            const int f = kk * KF + q;
            if (f == N) xmask |= 1u << q;
#pragma unroll
            for (int j = 0; j < NP; ++j) h[q][j] = (active && f < N && j == state_slot<REV, NP>(f)) ? T(1) : T(0);
        }
        if (!p.fixonly) {
            if constexpr (NP <= 16) {
                // Warps that hold no phase-A lane (aw .. 7) issue the next
                // window's loads while the others compute this one (one
                // barrier per window; measured 6 % faster at order 16 on
                // B200).
                // (the plan leaves at least one such warp at these orders)
                const bool lwarp = warp >= aw;
                const int nlw = THREADS / 32 - aw;
                // a whole batch inside its signal with 16-byte vectors takes
                // the flat copy path (no per-window range checks)
                const bool flat = NP <= 16 && LA::FLAT_OK && p.loader == kLoadVec && sg.vx && Gb == G && tb + (int64_t)G * L <= sg.T;
                auto issue = [&](int w, T *As, T *xs) {
                    if (flat)
                        LA::load_flat(p, sg, tb, G, L, w, As, xs, nullptr, false, tid - aw * 32, nlw * 32);
                    else
                        LA::template load<true>(p, sg, tb, Gb, L, w, As, xs, nullptr, false, aw, nlw);
                };
                if (lwarp) issue(0, Abuf, ibuf);
                cp_async_commit();
                for (int w = 0; w < nwin; ++w) {
                    const int s = w & 1;
                    cp_async_wait<0>();  // window w (issued by this thread, if a loader)
                    __syncthreads();     // window w is visible, window w-1's stage is free
                    if (lwarp && w + 1 < nwin)
                        issue(w + 1, Abuf + (size_t)(s ^ 1) * G * GSA, ibuf + (size_t)(s ^ 1) * G * W);
                    cp_async_commit();
                    if (active) {
                        if (w == nwin / 2) {
#pragma unroll
                            for (int q = 0; q < KF; ++q)
                                put_map_column<T, NP, REV>(hmap + (size_t)grp * HME, NP, h[q], kk * KF + q, N);
                        }
                        const T *Ag = Abuf + (size_t)s * G * GSA + (size_t)grp * GSA;
                        const T *xg = ibuf + (size_t)s * G * W + (size_t)grp * W;
#pragma unroll 1
                        for (int blk = 0; blk < W / NP; ++blk)
                            map_steps<T, NP, KF, REV, NEG, W, 0, NP>(Ag, xg, xmask, blk * NP, h);
                    }
                }
            } else {
                LA::load(p, sg, tb, Gb, L, 0, Abuf, ibuf, nullptr, false);
                cp_async_commit();
                for (int w = 0; w < nwin; ++w) {
                    const int s = w & 1;
                    if (w + 1 < nwin)
                        LA::load(p, sg, tb, Gb, L, w + 1, Abuf + (size_t)(s ^ 1) * G * GSA,
                                 ibuf + (size_t)(s ^ 1) * G * W, nullptr, false);
                    cp_async_commit();
                    cp_async_wait<1>();
                    __syncthreads();
                    if (active) {
                        if (w == nwin / 2) {
                            // the state after the first half of the chunk (in scan
                            // order): the lane's columns of the half map (or its z)
#pragma unroll
                            for (int q = 0; q < KF; ++q)
                                put_map_column<T, NP, REV>(hmap + (size_t)grp * HME, NP, h[q], kk * KF + q, N);
                        }
                        const T *Ag = Abuf + (size_t)s * G * GSA + (size_t)grp * GSA;
                        const T *xg = ibuf + (size_t)s * G * W + (size_t)grp * W;
#pragma unroll 1
                        for (int blk = 0; blk < W / NP; ++blk)
                            map_steps<T, NP, KF, REV, NEG, W, 0, NP>(Ag, xg, xmask, blk * NP, h);
                    }
                    __syncthreads();
                }
            }
            cp_async_wait<0>();
            __syncthreads();
        }

        // ------------------------------------------------------------ phase B
        // tree leaves (aliasing the window buffers): zero, then the chunk maps
        // (column k of a chunk's P from lane k, z from the zero-state lane),
        // identity beyond Gb.  Leaf 0 is the chunk scanned first: forward,
        // chunk g is leaf g; backward (from the top), chunk g is leaf Gb-1-g.
        if (!p.fixonly) {
        for (int e = tid; e < Gp * MS; e += THREADS) maps[e] = T(0);
        __syncthreads();
        if (active) {
#pragma unroll
            for (int q = 0; q < KF; ++q)
                put_map_column<T, NP, REV>(maps + (size_t)(REV ? Gb - 1 - grp : grp) * MS, RS, h[q], kk * KF + q, N);
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
                if (!REV && p.zi && tid < N) v = (double)p.zi[sg.zo + tid];
                s_in[tid] = v;
            }
        } else {
            // padded record: rows/columns beyond N of the root are zero
            for (int e = tid; e < PSE; e += THREADS) {
                const int r = e / NP, c = e - (e / NP) * NP;
                p.aggP[(size_t)me * PSE + e] = r < NP ? root[r * RS + c] : T(0);
            }
            for (int e = tid; e < ZSE; e += THREADS)
                p.aggz[(size_t)me * ZSE + e] = e < NP ? (double)root[NP * RS + e] : 0.0;
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(p.flags + me, kFlagAgg);
            if (tid < 32) {
                // warp 0 alone: parallel look-back.  Lane l watches predecessor
                // kb-1-l-32r; a round ends when every watched batch has
                // published; the nearest inclusive state ends the walk.
                int64_t found = -1;
                bool timeout = false;
                for (int64_t hi = kb - 1; hi >= 0 && found < 0 && !timeout; hi -= 32) {
                    const int64_t m = hi - lane;
                    unsigned f = kFlagInc;  // batches before 0 do not exist: treat as resolved
                    if (m >= 0) {
                        const unsigned *fp = p.flags + sg.fb + m * sg.fs;
                        f = ld_acquire(fp);
                        unsigned n = 0;
                        while (f == 0u) {
                            if (++n > p.spin_limit || ld_acquire(p.status) != 0u) {
                                atomicOr(p.status, kStatusFlagWait);
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
                    if (lane == 0) atomicOr(p.status, kStatusNoInclusive);
                    timeout = true;
                }
                // the flags seen above were acquired lane by lane; order every
                // lane's reads of the predecessors' data after them
                __threadfence();
                if (lane < NP) {
                    double v = 0.0;
                    if (!timeout && lane < N) v = __ldcg(p.incl + (size_t)(sg.fb + found * sg.fs) * N + lane);
                    s_in[lane] = v;
                }
                __syncwarp();
                // compose the aggregates found+1 .. kb-1 in order.  They are
                // staged KL at a time into a double-buffered shared
                // stage with 16-byte cp.async (L2 only, so a line of a record
                // published later is never served from this SM's L1); the next
                // round is in flight while this one is applied.
                constexpr int PV = PSE * (int)sizeof(T) / 16;  // vectors per P record
                constexpr int ZV = ZSE * 8 / 16;               // vectors per z record
                // lanes per row of the matvec: two for orders 8..16 (a shorter
                // FMA chain per hop), one otherwise
                constexpr int LPR = (NP >= 8 && NP <= 16) ? 2 : 1;
                constexpr int CPL = NP / LPR;  // columns per lane
                const int64_t first = timeout ? kb : found + 1;
                const int nround = (int)((kb - first + KL - 1) / KL);
                auto stage = [&](int r) {
                    const int64_t m0 = first + (int64_t)r * KL;
                    const int nh = (int)min64(KL, kb - m0);
                    T *dP = lbP + (size_t)(r & 1) * KL * PSE;
                    double *dz = lbz + (size_t)(r & 1) * KL * ZSE;
                    for (int v = lane; v < nh * (PV + ZV); v += 32) {
                        const int hh = v / (PV + ZV);
                        const int q = v - hh * (PV + ZV);
                        const int64_t idx = sg.fb + (m0 + hh) * sg.fs;
                        if (q < PV)
                            cp_async<16>(dP + (size_t)hh * PSE + q * (16 / sizeof(T)), p.aggP + (size_t)idx * PSE + q * (16 / sizeof(T)));
                        else
                            cp_async<16>(dz + (size_t)hh * ZSE + (q - PV) * 2, p.aggz + (size_t)idx * ZSE + (q - PV) * 2);
                    }
                };
                if (nround > 0) stage(0);
                cp_async_commit();
                const int half = LPR == 2 ? lane >> 4 : 0;
                const int row = LPR == 2 ? lane & 15 : lane;
                const bool act = row < NP;
                for (int r = 0; r < nround; ++r) {
                    if (r + 1 < nround) stage(r + 1);
                    cp_async_commit();
                    cp_async_wait<1>();
                    __syncwarp();
                    const int nh = (int)min64(KL, kb - first - (int64_t)r * KL);
                    const T *P0 = lbP + (size_t)(r & 1) * KL * PSE;
                    const double *z0 = lbz + (size_t)(r & 1) * KL * ZSE;
                    for (int hh = 0; hh < nh; ++hh) {
                        double v = 0.0;
                        if (act) {
                            // padded rows and state entries are zero: no order guards
                            const T *Pr = P0 + (size_t)hh * PSE + row * NP + half * CPL;
                            const double *sv = s_in + half * CPL;
                            double acc[4] = {half == 0 ? z0[hh * ZSE + row] : 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                            for (int q = 0; q < CPL; ++q) acc[q & 3] = fma((double)Pr[q], sv[q], acc[q & 3]);
                            v = (acc[0] + acc[1]) + (acc[2] + acc[3]);
                        }
                        if constexpr (LPR == 2) v += __shfl_xor_sync(0xffffffffu, v, 16);
                        __syncwarp();
                        if (act && half == 0) s_in[row] = v;
                        __syncwarp();
                    }
                }
                cp_async_wait<0>();
            }
        }
        __syncthreads();
        // inclusive state of this batch: root applied to s_in
        if (kb + 1 < sg.nb) {
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
        }  // !fixonly

        // ------------------------------------------------------------ phase D
        // fix-up: one lane per half-chunk (lane 2g: the lower half of chunk g,
        // lane 2g+1: the upper half) re-runs it from its exact entry state, in
        // scan order.  Forward: the lower half starts from the chunk's entry
        // state, the upper half from the first half's map applied to it.
        // Backward: the upper half starts from the adjoint state at the
        // chunk's top, the lower half from the upper half's adjoint map
        // applied to it.  The maps are applied in FP64.  A checkpointed
        // forward records every half-chunk's entry state; a fix-only launch
        // starts each half-chunk from the recorded one.
        const int Gd = 2 * Gb;  // half-chunks of the batch
        if (p.loader == kLoadElem && N < NP)
            for (int e = tid; e < DS * 2 * G * GSD; e += THREADS)
                if ((e % GSD) % NP >= N) Abuf[e] = T(0);
        const bool fix = tid < Gd;
        {
            const int g = tid >> 1;
            const int slot = !fix ? 0 : (REV ? Gb - 1 - g : g);
            const double *sv = st + (size_t)slot * NP;
            const bool via_half = REV ? (tid & 1) == 0 : (tid & 1) == 1;
            T *ck = (!REV && p.ckpt && fix) ? p.ckpt + ((size_t)(sgs->pb + jb) * 2 * G + tid) * N : nullptr;
            if (!REV && p.fixonly) {
#pragma unroll
                for (int i = 0; i < NP; ++i) h[0][state_slot<REV, NP>(i)] = (ck && i < N) ? ck[i] : T(0);
            } else if (fix && via_half) {
                const T *Hg = hmap + (size_t)g * HME;
#pragma unroll
                for (int i = 0; i < NP; ++i) {
                    double v = (double)Hg[NP * NP + i];
#pragma unroll
                    for (int k = 0; k < NP; ++k) v = fma((double)Hg[i * NP + k], sv[k], v);
                    h[0][state_slot<REV, NP>(i)] = i < N ? (T)v : T(0);
                }
            } else {
#pragma unroll
                for (int i = 0; i < NP; ++i) h[0][state_slot<REV, NP>(i)] = (fix && i < N) ? (T)sv[i] : T(0);
            }
            if (ck && !p.fixonly) {
                // boundary-state checkpoint: the half-chunk's exact entry state
#pragma unroll
                for (int i = 0; i < NP; ++i)
                    if (i < N) ck[i] = h[0][state_slot<REV, NP>(i)];
            }
        }
        const bool ti = REV && p.gA && p.as_t == 0;
        // grad_A rows are dense (B,T,N): 16-byte vectors when N fills NP
        const bool gA_vec = N == NP && NP % V == 0 && is_aligned16<T>(p.gA);
        __syncthreads();
        // Every warp loads the next window, then the phase-D lanes compute
        // (leaving the loads to the warps without phase-D lanes, as phase A
        // does, measured 10 % slower in the backward: those loads are the
        // larger part of the window's time there).  nwin windows of WD steps
        // cover a half-chunk.
        static_assert(DS == 2 && 2 * WD == W, "phase D is double buffered, half-length windows");
        // flat copies for a whole batch inside its signal (backward: lagged
        // outputs from t >= 0 as well)
        const bool dflat = NP <= 16 && LD::FLAT_OK && p.loader == kLoadVec && sg.vx && Gb == G && tb + (int64_t)G * L <= sg.T && (!REV || tb >= NP);
        auto dissue = [&](int w, T *As, T *xs, T *ys) {
            if (dflat)
                LD::load_flat(p, sg, tb, Gd, LH, w, As, xs, ys, REV, tid, THREADS);
            else
                LD::load(p, sg, tb, Gd, LH, w, As, xs, ys, REV);
        };
        dissue(0, Abuf, ibuf, ybuf);
        cp_async_commit();
        for (int w = 0; w < nwin; ++w) {
            const int s = w & 1;
            if (w + 1 < nwin)
                dissue(w + 1, Abuf + (size_t)(s ^ 1) * Gd * GSD, ibuf + (size_t)(s ^ 1) * Gd * WD,
                       ybuf + (size_t)(s ^ 1) * Gd * PYD);
            cp_async_commit();
            cp_async_wait<1>();
            __syncthreads();
            const T *As = Abuf + (size_t)s * Gd * GSD;
            const T *xs = ibuf + (size_t)s * Gd * WD;
            const T *ys = ybuf + (size_t)s * Gd * PYD;
            if (fix) {
                const T *Ag = As + (size_t)tid * GSD;
                const T *xg = xs + (size_t)tid * WD;
                T *og = obuf + (size_t)tid * WD;
                if constexpr (WD % NP == 0) {
#pragma unroll 1
                    for (int blk = 0; blk < WD / NP; ++blk) fix_steps<T, NP, REV, NEG, WD, 0, NP>(Ag, xg, og, blk * NP, h[0]);
                } else {
                    // NP == 2*WD: the ring advances by half a turn per window
                    static_assert(NP == 2 * WD, "window/order mismatch");
                    if (w & 1)
                        fix_steps<T, NP, REV, NEG, WD, WD, WD>(Ag, xg, og, 0, h[0]);
                    else
                        fix_steps<T, NP, REV, NEG, WD, 0, WD>(Ag, xg, og, 0, h[0]);
                }
            }
            __syncthreads();
            // flush the window's outputs (obuf is indexed by step): step j of
            // half-chunk g is sample tb + g*LH + w*WD + j forward and
            // tb + (g+1)*LH - w*WD - 1 - j backward
            for (int e = tid; e < Gd * WD; e += THREADS) {
                const int g = e / WD;
                const int j = e - g * WD;
                const int64_t t = REV ? tb + (int64_t)(g + 1) * LH - (int64_t)w * WD - 1 - j
                                      : tb + (int64_t)g * LH + (int64_t)w * WD + j;
                if (t < sg.T) p.out[sg.xo + t] = obuf[e];
            }
            if (REV && p.gA && !ti) {
                // one warp per half-chunk: row t = top-WD+rr has grad_x[t] =
                // obuf[g][WD-1-rr] and y[t-1-i] = ys[g][rr+NP-1-i]
                const T sgn = NEG ? T(1) : T(-1);
                for (int g = tid >> 5; g < Gd; g += THREADS / 32) {
                    const int64_t top = tb + (int64_t)(g + 1) * LH - (int64_t)w * WD;
                    const T *og = obuf + g * WD + (WD - 1);
                    const T *yg = ys + g * PYD + NP - 1;
                    if (gA_vec) {
                        // rows [top-WD, top) are one contiguous run of grad_A:
                        // vector v of the run holds taps i0.. of row rr
                        constexpr int QR = NP / V > 0 ? NP / V : 1;  // vectors per row (gA_vec: NP % V == 0)
                        constexpr int QPC = WD * QR;                 // vectors per half-chunk window
                        using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
                        const int64_t r0 = sg.xo + top - WD;  // row of slot 0; rows past the signal are skipped
#pragma unroll
                        for (int k = 0; k < (QPC + 31) / 32; ++k) {
                            const int v = lane + 32 * k;
                            const int rr = v / QR;
                            if ((QPC % 32 != 0 && v >= QPC) || top - WD + rr >= sg.T) continue;
                            const int i0 = (v - rr * QR) * V;
                            const T gx = sgn * og[-rr];
                            const T *yq = yg + rr - i0;
                            VT o;
                            T *ov = reinterpret_cast<T *>(&o);
#pragma unroll
                            for (int j = 0; j < V; ++j) ov[j] = gx * yq[-j];
                            *reinterpret_cast<VT *>(p.gA + (r0 + rr) * NP + i0) = o;
                        }
                    } else {
                        for (int e = lane; e < WD * N; e += 32) {
                            const int rr = e / N;
                            const int i = e - rr * N;
                            const int64_t t = top - WD + rr;
                            if (t >= sg.T) continue;
                            p.gA[(sg.xo + t) * N + i] = sgn * og[-rr] * yg[rr - i];
                        }
                    }
                }
            }
            __syncthreads();
        }
        cp_async_wait<0>();
        // the lower half of the signal's first chunk ends at t = 0 holding the
        // adjoint of the initial conditions (pending gradients of y[-1-i])
        if (REV && p.gzi && jb == 0 && tid == 0) {
#pragma unroll
            for (int i = 0; i < NP; ++i)
                if (i < N) p.gzi[sg.zo + i] = h[0][state_slot<REV, NP>(i)];
        }
    }
}

// ----------------------------------------------------------------------------
// Host side.
// ----------------------------------------------------------------------------
constexpr int kChunkLen = 256;   // target chunk length for mid-length signals (rounded to an even number of windows)

// Default target chunk length by signal length (measured on B200: 128 for
// 16,000-sample signals, 512 for 2^20-sample signals).
inline int64_t default_chunk(int64_t T) { return T < 65536 ? kChunkLen / 2 : (T < (1 << 19) ? kChunkLen : 2 * kChunkLen); }

// Process-wide target chunk length (the autotuner's knob; 0 = default).
std::atomic<int64_t> g_chunk_target{0};

// Process-wide error word of the chunked kernels (see ChunkParams::err_word).
std::atomic<unsigned *> g_err_word{nullptr};
constexpr int kMaxChunksPerBatch = 64;

inline int threads_for(int) { return 256; }  // scan group: one group of phase-A lanes per chunk
inline int window_for(int NP) { return window_steps(NP); }

struct Plan {
    int NP, G, L;
    int64_t nbps, nbatches;
};

// Chunks per batch: one group of N+1 lanes per chunk, capped so that the
// shared memory of a CTA fits the occupancy the kernel is built for
// (ctas_per_sm: two CTAs per SM up to order 24 and for fp64, three above).
// `force` > 0 fixes the chunk length (a checkpointed forward and its
// backward must cut the signal identically).
inline Plan make_plan(size_t esz, int64_t B, int64_t T, int64_t N, int64_t dflt = 0, int64_t force = 0) {
    Plan pl;
    pl.NP = padded_order(N);
    const int W = window_for(pl.NP);
    const int64_t want = force > 0 ? force : g_chunk_target.load(std::memory_order_relaxed);
    // default by signal length: short signals want more batches in flight,
    // long ones fewer look-back hops per sample
    const int64_t target = want > 0 ? want : (dflt > 0 ? dflt : default_chunk(T));
    pl.L = (int)(2 * W * ((target + 2 * W - 1) / (2 * W)));  // an even number of windows: halves split on one
    // chunks per batch: one group of phase-A lanes per chunk; with two filters
    // per lane at most 16 (a power-of-two tree; larger batches measured slower)
    const int KF = filters_per_lane(pl.NP);
    int G = (int)(threads_for(pl.NP) / (N + 1));
    const int Gk = (int)(threads_for(pl.NP) / ((N + KF) / KF));
    if (Gk > G) G = Gk < 16 ? Gk : (G > 16 ? G : 16);
    if (G > kMaxChunksPerBatch) G = kMaxChunksPerBatch;
    // orders up to 16 keep at least one warp free of phase-A lanes: it loads
    // the next window while the others compute
    if (pl.NP <= 16)
        while (G > 1 && G * ((N + KF) / KF) > threads_for(pl.NP) - 32) --G;
    const int ctas = ctas_per_sm(pl.NP, (int)esz);
    const size_t budget = (size_t)228 * 1024 / ctas - 1024;  // per-SM shared memory less the per-CTA reserve
    while (G > 1 && SmemPlan(esz, pl.NP, G, true).total > budget) --G;
    pl.G = G;
    const int64_t span = (int64_t)pl.G * pl.L;
    pl.nbps = (T + span - 1) / span;
    if (pl.nbps < 1) pl.nbps = 1;
    pl.nbatches = B * pl.nbps;
    return pl;
}

inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Whether coefficient rows can move as 16-byte vectors: dense rows of the
// padded order, 16-byte rows, 16-byte aligned base and signal strides.  (Input
// windows are checked per batch: ragged signals start anywhere.)
template <typename T>
bool vec_ok(const ChunkParams<T> &p, int NP) {
    const size_t esz = sizeof(T);
    if (p.N != NP || p.as_t != NP || (NP * esz) % 16 != 0) return false;
    return aligned16(p.A) && (p.as_b * esz) % 16 == 0;
}

template <typename T, int NP, bool REV, bool NEG>
cudaError_t launch_np(ChunkParams<T> p, cudaStream_t st) {
    auto kern = chunked_kernel<T, NP, REV, NEG>;
    const SmemPlan S(sizeof(T), NP, p.G, REV);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S.total);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Cfg<NP>::THREADS, S.total);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > p.nbatches) grid = p.nbatches;  // ragged: an upper bound on the batches
    p.loader = vec_ok(p, NP) ? kLoadVec : kLoadElem;
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
    p.err_word = g_err_word.load(std::memory_order_acquire);
    return p;
}

}  // namespace

bool chunked_supported(int64_t N) { return N >= 1 && N <= 32; }

void set_error_word(unsigned *word) { g_err_word.store(word, std::memory_order_release); }

void set_chunk_target(int64_t samples) {
    g_chunk_target.store(samples <= 0 ? 0 : (samples < 32 ? 32 : (samples > 4096 ? 4096 : samples)),
                         std::memory_order_relaxed);
}

int64_t chunk_target() { return g_chunk_target.load(std::memory_order_relaxed); }

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
    e = neg ? dispatch<T, true, true>(p, pl.NP, st) : dispatch<T, true, false>(p, pl.NP, st);
    if (e != cudaSuccess || !a.gA || a.a_stride_t != 0) return e;
    return ti_grad_a<T>(a.gx, a.y, a.zi, a.gA, a.B, a.T, a.N, neg, st);  // reads the grad_x just written
}

// ----------------------------------------------------------------------------
// Boundary-state checkpointing: the forward keeps the exact entry state of
// every half-chunk (N values per half-chunk, batch-major in the plan's layout)
// beside y, so that y need not be kept for the backward.  The backward first
// recomputes y from those states and x with a fix-only launch of the forward
// kernel (the exact pass alone: every half-chunk independent, no maps, no
// look-back), into its workspace, then runs the fused backward on it.  Both
// calls take the same chunk length, which fixes the plan (the chunk-length
// setting may change in between).
// ----------------------------------------------------------------------------
namespace {

struct CkptLayout {
    Plan pl;
    WsLayout l;
    size_t ybuf, total;
};

inline CkptLayout ckpt_layout(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk) {
    CkptLayout c;
    c.pl = make_plan(esz, B, T, N, 0, chunk);
    c.l = ws_layout(esz, c.pl.nbatches, N);
    c.ybuf = c.l.total;
    c.total = align256(c.ybuf + (size_t)B * T * esz);
    return c;
}

}  // namespace

int64_t chunked_checkpoint_chunk(size_t esz, int64_t T, int64_t N) { return make_plan(esz, 1, T, N).L; }

int64_t chunked_checkpoint_elems(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk) {
    if (!chunked_supported(N) || chunk <= 0) return 0;
    const Plan pl = make_plan(esz, B, T, N, 0, chunk);
    return pl.nbatches * 2 * pl.G * N;
}

size_t chunked_forward_ckpt_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk) {
    if (!chunked_supported(N) || chunk <= 0) return 0;
    return ws_layout(esz, make_plan(esz, B, T, N, 0, chunk).nbatches, N).total;
}

size_t chunked_backward_ckpt_workspace(size_t esz, int64_t B, int64_t T, int64_t N, int64_t chunk) {
    if (!chunked_supported(N) || chunk <= 0) return 0;
    return ckpt_layout(esz, B, T, N, chunk).total;
}

template <typename T>
cudaError_t chunked_forward_ckpt(const FwdArgs<T> &a, T *states, int64_t chunk, void *ws, size_t ws_bytes,
                                 cudaStream_t st) {
    const Plan pl = make_plan(sizeof(T), a.B, a.T, a.N, 0, chunk);
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
    p.ckpt = states;
    return dispatch<T, false, false>(p, pl.NP, st);
}

template <typename T>
cudaError_t chunked_backward_ckpt(const BwdArgs<T> &a, const T *x, const T *states, int64_t chunk, void *ws,
                                  size_t ws_bytes, cudaStream_t st) {
    const CkptLayout c = ckpt_layout(sizeof(T), a.B, a.T, a.N, chunk);
    if (ws_bytes < c.total) return cudaErrorInvalidValue;
    T *y = reinterpret_cast<T *>(static_cast<unsigned char *>(ws) + c.ybuf);
    // 1. y from the recorded half-chunk states (only the ticket counter and
    //    the status word of the workspace are used)
    cudaError_t e = cudaMemsetAsync(ws, 0, c.l.aggP, st);
    if (e != cudaSuccess) return e;
    ChunkParams<T> p = base_params<T>(c.pl, a.B, a.T, a.N, ws);
    p.in = x;
    p.A = a.A;
    p.as_b = a.a_stride_b;
    p.as_t = a.a_stride_t;
    p.zi = a.zi;
    p.out = y;
    p.ckpt = const_cast<T *>(states);
    p.fixonly = 1;
    e = dispatch<T, false, false>(p, c.pl.NP, st);
    if (e != cudaSuccess) return e;
    // 2. the fused backward on it, with the same plan
    e = cudaMemsetAsync(ws, 0, c.l.aggP, st);
    if (e != cudaSuccess) return e;
    ChunkParams<T> q = base_params<T>(c.pl, a.B, a.T, a.N, ws);
    q.in = a.gy;
    q.A = a.A;
    q.as_b = a.a_stride_b;
    q.as_t = a.a_stride_t;
    q.zi = a.zi;
    q.ysave = y;
    q.out = a.gx;
    q.gA = a.gA;
    q.gzi = a.gzi;
    return dispatch<T, true, false>(q, c.pl.NP, st);
}

template cudaError_t chunked_forward_ckpt<float>(const FwdArgs<float> &, float *, int64_t, void *, size_t,
                                                 cudaStream_t);
template cudaError_t chunked_forward_ckpt<double>(const FwdArgs<double> &, double *, int64_t, void *, size_t,
                                                  cudaStream_t);
template cudaError_t chunked_backward_ckpt<float>(const BwdArgs<float> &, const float *, const float *, int64_t,
                                                  void *, size_t, cudaStream_t);
template cudaError_t chunked_backward_ckpt<double>(const BwdArgs<double> &, const double *, const double *,
                                                   int64_t, void *, size_t, cudaStream_t);

// ----------------------------------------------------------------------------
// Ragged batches: nsig signals concatenated along time, signal s occupying
// samples [off[s], off[s+1]) of x / y and rows of A (S, N); zi (nsig, N).
// Batches are numbered signal by signal, so the workspace needs at most
// nsig + S / span + 1 batch records; the first batch of each signal (bb) is
// computed on the device from the offsets.
// ----------------------------------------------------------------------------
namespace {

constexpr unsigned kStatusBadOffsets = 8u;  // a signal with a negative length (treated as empty)

__global__ void __launch_bounds__(1024) batch_base_kernel(const int64_t *off, int64_t nsig, int64_t span,
                                                          int64_t *bb, unsigned *status) {
    __shared__ int64_t sh[1024];
    __shared__ int64_t carry;
    const int tid = threadIdx.x;
    if (tid == 0) {
        carry = 0;
        bb[0] = 0;
    }
    __syncthreads();
    for (int64_t base = 0; base < nsig; base += 1024) {
        const int64_t s = base + tid;
        int64_t v = 0;
        if (s < nsig) {
            int64_t len = off[s + 1] - off[s];
            if (len < 0) {
                atomicOr(status, kStatusBadOffsets);
                len = 0;
            }
            v = (len + span - 1) / span;
        }
        sh[tid] = v;
        __syncthreads();
        for (int d = 1; d < 1024; d <<= 1) {  // inclusive scan of the batch counts
            const int64_t t = tid >= d ? sh[tid - d] : 0;
            __syncthreads();
            sh[tid] += t;
            __syncthreads();
        }
        if (s < nsig) bb[s + 1] = carry + sh[tid];
        __syncthreads();
        if (tid == 1023) carry += sh[1023];
        __syncthreads();
    }
}

struct RaggedLayout {
    Plan pl;
    int64_t nbmax;
    WsLayout l;
    size_t bb, total;
};

inline RaggedLayout ragged_layout(size_t esz, int64_t nsig, int64_t S, int64_t N) {
    RaggedLayout r;
    // ragged batches are numbered signal by signal, so a signal's batches run
    // side by side and look back over each other: long chunks (fewer batches,
    // 1024 samples measured best on B200) unless the caller set a length
    r.pl = make_plan(esz, 1, int64_t(1) << 20, N, 4 * kChunkLen);
    const int64_t span = (int64_t)r.pl.G * r.pl.L;
    r.nbmax = nsig + S / span + 1;
    r.l = ws_layout(esz, r.nbmax, N);
    r.bb = r.l.total;
    r.total = align256(r.bb + (size_t)(nsig + 1) * sizeof(int64_t));
    return r;
}

template <typename T>
ChunkParams<T> ragged_params(const RaggedLayout &r, int64_t nsig, int64_t N, const int64_t *off, void *ws) {
    ChunkParams<T> p = base_params<T>(r.pl, nsig, 0, N, ws);
    unsigned char *w = static_cast<unsigned char *>(ws);
    // the batch records are laid out for the worst-case batch count, not the
    // one-batch plan base_params was given
    p.flags = reinterpret_cast<unsigned *>(w + r.l.flags);
    p.aggP = reinterpret_cast<T *>(w + r.l.aggP);
    p.aggz = reinterpret_cast<double *>(w + r.l.aggz);
    p.incl = reinterpret_cast<double *>(w + r.l.incl);
    p.nbatches = r.nbmax;
    p.roff = off;
    p.bb = reinterpret_cast<int64_t *>(w + r.bb);
    p.nsig = nsig;
    p.as_b = 0;
    p.as_t = N;
    return p;
}

template <typename T>
cudaError_t ragged_prologue(const RaggedLayout &r, const ChunkParams<T> &p, void *ws, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(ws, 0, r.l.aggP, st);  // header + flags
    if (e != cudaSuccess) return e;
    batch_base_kernel<<<1, 1024, 0, st>>>(p.roff, p.nsig, (int64_t)r.pl.G * r.pl.L, p.bb, p.status);
    return cudaGetLastError();
}

}  // namespace

size_t chunked_ragged_workspace(size_t esz, int64_t nsig, int64_t S, int64_t N) {
    if (!chunked_supported(N)) return 0;
    return ragged_layout(esz, nsig, S, N).total;
}

template <typename T>
cudaError_t chunked_forward_ragged(const T *x, const T *A, const int64_t *off, const T *zi, T *y, int64_t nsig,
                                   int64_t S, int64_t N, void *ws, size_t ws_bytes, cudaStream_t st) {
    const RaggedLayout r = ragged_layout(sizeof(T), nsig, S, N);
    if (ws_bytes < r.total) return cudaErrorInvalidValue;
    ChunkParams<T> p = ragged_params<T>(r, nsig, N, off, ws);
    p.in = x;
    p.A = A;
    p.zi = zi;
    p.out = y;
    cudaError_t e = ragged_prologue<T>(r, p, ws, st);
    if (e != cudaSuccess) return e;
    return dispatch<T, false, false>(p, r.pl.NP, st);
}

template <typename T>
cudaError_t chunked_backward_ragged(const T *gy, const T *A, const int64_t *off, const T *zi, const T *y, T *gx,
                                    T *gA, T *gzi, int64_t nsig, int64_t S, int64_t N, void *ws, size_t ws_bytes,
                                    cudaStream_t st) {
    const RaggedLayout r = ragged_layout(sizeof(T), nsig, S, N);
    if (ws_bytes < r.total) return cudaErrorInvalidValue;
    ChunkParams<T> p = ragged_params<T>(r, nsig, N, off, ws);
    p.in = gy;
    p.A = A;
    p.zi = zi;
    p.ysave = y;
    p.out = gx;
    p.gA = gA;
    p.gzi = gzi;
    cudaError_t e = ragged_prologue<T>(r, p, ws, st);
    if (e != cudaSuccess) return e;
    if (gzi) {  // empty signals get no batch: their grad_zi is zero
        e = cudaMemsetAsync(gzi, 0, (size_t)nsig * N * sizeof(T), st);
        if (e != cudaSuccess) return e;
    }
    return dispatch<T, true, false>(p, r.pl.NP, st);
}

template cudaError_t chunked_forward_ragged<float>(const float *, const float *, const int64_t *, const float *,
                                                   float *, int64_t, int64_t, int64_t, void *, size_t, cudaStream_t);
template cudaError_t chunked_forward_ragged<double>(const double *, const double *, const int64_t *, const double *,
                                                    double *, int64_t, int64_t, int64_t, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward_ragged<float>(const float *, const float *, const int64_t *, const float *,
                                                    const float *, float *, float *, float *, int64_t, int64_t,
                                                    int64_t, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward_ragged<double>(const double *, const double *, const int64_t *,
                                                     const double *, const double *, double *, double *, double *,
                                                     int64_t, int64_t, int64_t, void *, size_t, cudaStream_t);

// ----------------------------------------------------------------------------
// Failure detection without a fault: a chunked forward whose ticket queue
// starts past batch 0, so batch 1's look-back waits for a flag nothing ever
// sets.  With a short spin limit the wait gives up, records
// kStatusFlagWait in the status word and the kernel finishes normally.
// ----------------------------------------------------------------------------
size_t chunked_selftest_workspace() {
    const int64_t N = 2;
    const Plan pl = make_plan(4, 1, 1, N);
    const int64_t T = 2 * (int64_t)pl.G * pl.L;  // two batches
    return ws_layout(4, 2, N).total + align256((size_t)(2 * T + T * N) * sizeof(float));
}

cudaError_t chunked_selftest_timeout(void *ws, size_t ws_bytes, unsigned spin_limit, cudaStream_t st) {
    const int64_t N = 2;
    const Plan pl = make_plan(4, 1, 1, N);
    const int64_t T = 2 * (int64_t)pl.G * pl.L;
    const Plan p2 = make_plan(4, 1, T, N);
    if (ws_bytes < chunked_selftest_workspace() || p2.nbatches != 2) return cudaErrorInvalidValue;
    const WsLayout l = ws_layout(4, p2.nbatches, N);
    float *x = reinterpret_cast<float *>(static_cast<unsigned char *>(ws) + l.total);
    float *y = x + T;
    float *A = y + T;
    cudaError_t e = cudaMemsetAsync(ws, 0, chunked_selftest_workspace(), st);  // zero inputs, header, flags
    if (e != cudaSuccess) return e;
    const unsigned first = 1;  // skip batch 0: its flag is never published
    e = cudaMemcpyAsync(ws, &first, sizeof(first), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    ChunkParams<float> p = base_params<float>(p2, 1, T, N, ws);
    p.in = x;
    p.A = A;
    p.as_b = T * N;
    p.as_t = N;
    p.out = y;
    p.spin_limit = spin_limit;
    e = dispatch<float, false, false>(p, p2.NP, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);  // `first` lives on this host stack frame
}

template cudaError_t chunked_forward<float>(const FwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_forward<double>(const FwdArgs<double> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<float>(const BwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<double>(const BwdArgs<double> &, bool, void *, size_t, cudaStream_t);

}  // namespace lpcb
