// Forward filter for callers that cannot allocate device memory.
//
// The chunked forward kernel needs scratch memory in global memory (a ticket
// counter, a status word, one flag, aggregate and inclusive state per batch of
// chunks).  lpc_b200_forward takes that scratch as a caller-supplied
// workspace.  Some callers cannot provide one: code that runs where no
// allocator may be called (inside a host callback, from a real-time audio
// thread that must not block on the driver's allocator, from a plugin host
// that owns all device memory), or code that has no allocator at all (a thin
// FFI binding with no memory manager).  This entry point serves them with a
// fixed scratch array that lives in the library itself.
//
// The array is a file-scope __device__ variable, so every GPU that loads this
// library holds kStaticScratchBytes of device memory until the process exits.
// Its host-side name is only a stand-in for the symbol: the device address is
// looked up with cudaGetSymbolAddress on every call, for the device (and
// context) current at that moment.  The lookup allocates nothing; the first
// one on a device also loads the module there, which is why that first call
// must come before any stream capture.  Nothing is cached, so a device reset
// or another context made current between calls cannot leave a stale address.

#include "lpc_chunked.cuh"

using namespace lpcb;

namespace {

// 8 MiB: enough for about 6,500 batches of chunks, i.e. roughly 13 to 50
// million samples per call at order 16 (longer signals use longer chunks; the
// scratch grows with the number of batches and with N^2).
constexpr size_t kStaticScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of the scratch array in the current context.
int scratch_for_current_device(void **out) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || ptr == nullptr) return LPC_ERR_CUDA;
    *out = ptr;
    return LPC_OK;
}

template <typename T>
int run(const void *x, const void *A, const void *zi, void *y, int64_t B, int64_t T_, int64_t N, int64_t sb,
        int64_t st, void *scratch, cudaStream_t stream) {
    FwdArgs<T> p{static_cast<const T *>(x), static_cast<const T *>(A), static_cast<const T *>(zi),
                 static_cast<T *>(y), B, T_, N, sb, st};
    // chunked_forward clears the counter, status word and flags of the scratch
    // on `stream` before the kernel runs; the rest is written before it is read.
    // It refuses a plan larger than the scratch with cudaErrorInvalidValue (the
    // chunk-length setting changed since the size check): report that as the
    // size error it is.
    const cudaError_t e = chunked_forward<T>(p, false, scratch, kStaticScratchBytes, stream);
    if (e == cudaErrorInvalidValue) return LPC_ERR_WORKSPACE;
    return e == cudaSuccess ? LPC_OK : LPC_ERR_CUDA;
}

}  // namespace

extern "C" int lpc_b200_forward_noalloc(int dtype, const void *x, const void *A, const void *zi, void *y,
                                        int64_t B, int64_t T, int64_t N, int64_t a_stride_b,
                                        int64_t a_stride_t, void *stream) {
    if (dtype != LPC_F32 && dtype != LPC_F64) return LPC_ERR_INVALID_ARGUMENT;
    if (B < 0 || T < 0 || N < 1 || N > kMaxOrder || B >= (int64_t(1) << 31)) return LPC_ERR_INVALID_ARGUMENT;
    if (B > 0 && T > 0 && (!x || !A || !y)) return LPC_ERR_INVALID_ARGUMENT;
    if (a_stride_t < 0 || a_stride_b < 0 || (a_stride_t != 0 && a_stride_t < N)) return LPC_ERR_INVALID_ARGUMENT;
    if (!chunked_supported(N)) return LPC_ERR_UNSUPPORTED;  // orders above 32 have no chunked kernel
    if (B == 0 || T == 0) return LPC_OK;
    const size_t esz = dtype == LPC_F32 ? 4 : 8;
    if (chunked_forward_workspace(esz, B, T, N, a_stride_t) > kStaticScratchBytes) return LPC_ERR_WORKSPACE;
    void *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != LPC_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == LPC_F32) return run<float>(x, A, zi, y, B, T, N, a_stride_b, a_stride_t, scratch, s);
    return run<double>(x, A, zi, y, B, T, N, a_stride_b, a_stride_t, scratch, s);
}

extern "C" int lpc_b200_noalloc_status(unsigned *status, void *stream) {
    if (!status) return LPC_ERR_INVALID_ARGUMENT;
    void *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != LPC_OK) return rc;
    // the status word follows the ticket counter at the start of the scratch
    return lpc_b200_workspace_status(scratch, status, stream);
}
