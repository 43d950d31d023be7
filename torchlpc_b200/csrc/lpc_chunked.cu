#include "lpc_chunked.cuh"

namespace lpcb {

bool chunked_supported(int64_t) { return false; }
bool chunked_preferred(int64_t, int64_t, int64_t, int64_t) { return false; }
size_t chunked_forward_workspace(size_t, int64_t, int64_t, int64_t, int64_t) { return 0; }
size_t chunked_backward_workspace(size_t, int64_t, int64_t, int64_t, int64_t) { return 0; }

template <typename T>
cudaError_t chunked_forward(const FwdArgs<T> &, bool, void *, size_t, cudaStream_t) {
    return cudaErrorNotSupported;
}
template <typename T>
cudaError_t chunked_backward(const BwdArgs<T> &, bool, void *, size_t, cudaStream_t) {
    return cudaErrorNotSupported;
}
template cudaError_t chunked_forward<float>(const FwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_forward<double>(const FwdArgs<double> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<float>(const BwdArgs<float> &, bool, void *, size_t, cudaStream_t);
template cudaError_t chunked_backward<double>(const BwdArgs<double> &, bool, void *, size_t, cudaStream_t);

}  // namespace lpcb
