// torch operator layer of torchlpc_b200 (namespace torchlpc_b200).
//
// Thin: validates tensors with the reference's messages (torchlpc/csrc/cuda/
// lpc.cu:117-127, scan_cpu.cpp:146-156), allocates outputs and workspaces with
// the caching allocator, takes the current CUDA stream (so the ops can be
// captured in CUDA graphs) and calls the C ABI of liblpc_b200.  CUDA tensors
// only: there is no CPU implementation and no fallback.
#include <Python.h>
#include <ATen/ATen.h>
#include <mutex>
#include <sstream>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include "lpc_b200.h"

extern "C" {
// Importing torchlpc_b200._C loads this library, which runs the operator
// registrations below.
PyObject *PyInit__C(void) {
    static struct PyModuleDef module_def = {PyModuleDef_HEAD_INIT, "_C", nullptr, -1, nullptr};
    return PyModule_Create(&module_def);
}
}

namespace {

// Error word: one pinned host word (directly addressable by every device
// under unified addressing), installed as the library's process-wide error
// word on the first operator call.  A chunked kernel whose bounded wait gave
// up ORs its status into it; every operator reads it on entry (a plain host
// read, no synchronisation) and raises for the earlier call whose outputs are
// invalid.  check_status() synchronises first.
volatile unsigned *g_err_host = nullptr;
std::once_flag g_err_once;

void ensure_error_word() {
    std::call_once(g_err_once, [] {
        // leaked on purpose: the kernels may write it until the process exits
        auto *t = new at::Tensor(at::zeros({1}, at::TensorOptions().dtype(at::kInt).pinned_memory(true)));
        g_err_host = reinterpret_cast<volatile unsigned *>(t->data_ptr());
        lpc_b200_set_error_word(const_cast<unsigned *>(g_err_host));
    });
}

unsigned take_error_word() {
    ensure_error_word();
    const unsigned w = *g_err_host;
    if (w) *g_err_host = 0;
    return w;
}

void raise_pending() {
    const unsigned w = take_error_word();
    if (w) {
        std::ostringstream m;
        m << "torchlpc_b200: a bounded device-side wait of a chunked kernel gave up in an earlier call "
             "(status word 0x"
          << std::hex << w << "; 1: a predecessor's flag never appeared, 2: inconsistent flags, 8: a ragged "
          << "signal with a negative length); the outputs of that call are invalid";
        TORCH_CHECK(false, m.str());
    }
}

int dtype_code(const at::Tensor &t) {
    if (t.scalar_type() == at::kFloat) return LPC_F32;
    if (t.scalar_type() == at::kDouble) return LPC_F64;
    TORCH_CHECK(!t.is_complex(), "torchlpc_b200: complex dtypes are not supported");
    TORCH_CHECK(false, "torchlpc_b200: unsupported dtype ", t.scalar_type(),
                " (float32 and float64 are supported)");
    return -1;
}

void check_status(int status, const char *what) {
    TORCH_CHECK(status == LPC_OK, "torchlpc_b200::", what, " failed: ",
                lpc_b200_status_string(status));
}

void check_cuda(const at::Tensor &t, const char *name) {
    TORCH_CHECK(t.is_cuda(), "torchlpc_b200 runs on CUDA devices only; ", name, " is on ",
                t.device());
}

at::Tensor workspace(size_t bytes, const at::Tensor &like) {
    if (bytes == 0) return at::Tensor();
    return at::empty({(int64_t)bytes}, like.options().dtype(at::kByte));
}

void *ptr_or_null(const at::Tensor &t) { return t.defined() ? t.data_ptr() : nullptr; }

// Coefficients as (pointer tensor, stride_b, stride_t).  A (B,T,N) keeps a
// stride-0 time dimension (time-invariant filter, e.g. an expanded (B,N));
// a 2-D A (B,N) is time-invariant.  The last dimension must be unit-stride.
struct Coeffs {
    at::Tensor t;
    int64_t sb, st;
};

Coeffs coeffs(const at::Tensor &A, int64_t B, int64_t T, int64_t N, bool allow_time_invariant) {
    if (A.dim() == 2) {
        TORCH_CHECK(A.size(0) == B && A.size(1) == N, "Coefficients must have shape (B, order)");
        at::Tensor a = A.contiguous();
        return {a, N, 0};
    }
    TORCH_CHECK(A.dim() == 3, "Coefficients must be 3D (B, T, order)");
    TORCH_CHECK(A.size(0) == B && A.size(1) == T, "Coefficients must have shape (B, T, order)");
    const bool ti = allow_time_invariant && A.stride(1) == 0 && A.stride(2) == 1 && A.stride(0) >= 0;
    if (ti) return {A, A.stride(0), 0};
    at::Tensor a = A;
    if (!(a.stride(2) == 1 && a.stride(1) >= N && a.stride(0) >= 0 && (B <= 1 || a.stride(0) >= T * a.stride(1))))
        a = a.contiguous();
    return {a, a.stride(0), a.stride(1)};
}

at::Tensor lpc(const at::Tensor &x, const at::Tensor &A, const c10::optional<at::Tensor> &zi_opt,
               int64_t algo) {
    raise_pending();
    TORCH_CHECK(x.is_floating_point() || x.is_complex(), "Input must be floating point or complex");
    TORCH_CHECK(A.scalar_type() == x.scalar_type(),
                "Coefficients must have the same scalar type as input");
    TORCH_CHECK(x.dim() == 2, "Input must be 2D");
    check_cuda(x, "x");
    check_cuda(A, "A");
    const int64_t B = x.size(0), T = x.size(1), N = A.size(-1);
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = *zi_opt;
        TORCH_CHECK(zi.scalar_type() == x.scalar_type(),
                    "Initial conditions must have the same scalar type as input");
        TORCH_CHECK(zi.dim() == 2, "Initial conditions must be 2D");
        TORCH_CHECK(x.size(0) == zi.size(0), "Batch size of input and initial conditions must match");
        TORCH_CHECK(zi.size(1) == N, "Initial conditions must have shape (B, order)");
        check_cuda(zi, "zi");
        zi = zi.contiguous();
    }
    const int dt = dtype_code(x);
    const c10::cuda::CUDAGuard guard(x.device());
    Coeffs c = coeffs(A, B, T, N, true);
    at::Tensor xc = x.contiguous();
    at::Tensor y = at::empty({B, T}, x.options());
    const size_t wsb = lpc_b200_forward_workspace_size(dt, (int)algo, B, T, N, c.st);
    at::Tensor ws = workspace(wsb, x);
    auto stream = c10::cuda::getCurrentCUDAStream();
    check_status(lpc_b200_forward(dt, (int)algo, xc.data_ptr(), c.t.data_ptr(), ptr_or_null(zi),
                                  y.data_ptr(), B, T, N, c.sb, c.st, ptr_or_null(ws), wsb,
                                  stream.stream()),
                 "lpc");
    return y;
}

// Returns (grad_x, grad_A, grad_zi); unwanted gradients come back as empty
// tensors.  grad_A has A's shape: (B,T,N) for a 3-D A (a stride-0 A is
// materialised first so the per-sample gradient is exact), (B,N) for a 2-D A.
std::tuple<at::Tensor, at::Tensor, at::Tensor> lpc_backward(
    const at::Tensor &grad_y, const at::Tensor &A, const c10::optional<at::Tensor> &zi_opt,
    const at::Tensor &y, bool need_A, bool need_zi, int64_t algo) {
    raise_pending();
    TORCH_CHECK(grad_y.dim() == 2 && y.dim() == 2 && grad_y.sizes() == y.sizes(),
                "grad_y and y must be (B, T)");
    TORCH_CHECK(A.scalar_type() == y.scalar_type() && grad_y.scalar_type() == y.scalar_type(),
                "dtype mismatch");
    check_cuda(grad_y, "grad_y");
    check_cuda(A, "A");
    check_cuda(y, "y");
    const int64_t B = y.size(0), T = y.size(1), N = A.size(-1);
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = zi_opt->contiguous();
        TORCH_CHECK(zi.dim() == 2 && zi.size(0) == B && zi.size(1) == N, "zi must be (B, order)");
    }
    const int dt = dtype_code(y);
    const c10::cuda::CUDAGuard guard(y.device());
    Coeffs c = coeffs(A, B, T, N, /*allow_time_invariant=*/A.dim() == 2 || !need_A);
    at::Tensor gyc = grad_y.contiguous(), yc = y.contiguous();
    at::Tensor gx = at::empty({B, T}, y.options());
    at::Tensor gA, gzi;
    if (need_A) gA = c.st == 0 ? at::empty({B, N}, y.options()) : at::empty({B, T, N}, y.options());
    if (need_zi) gzi = at::empty({B, N}, y.options());
    const size_t wsb = lpc_b200_backward_workspace_size(dt, (int)algo, B, T, N, c.st);
    at::Tensor ws = workspace(wsb, y);
    auto stream = c10::cuda::getCurrentCUDAStream();
    check_status(lpc_b200_backward(dt, (int)algo, gyc.data_ptr(), c.t.data_ptr(), ptr_or_null(zi),
                                   yc.data_ptr(), gx.data_ptr(), ptr_or_null(gA), ptr_or_null(gzi),
                                   B, T, N, c.sb, c.st, ptr_or_null(ws), wsb, stream.stream()),
                 "lpc_backward");
    if (!need_A) gA = at::empty({0}, y.options());
    if (!need_zi) gzi = at::empty({0}, y.options());
    return {gx, gA, gzi};
}

at::Tensor scan(const at::Tensor &input, const at::Tensor &weights, const c10::optional<at::Tensor> &init_opt,
                int64_t algo) {
    raise_pending();
    TORCH_CHECK(input.is_floating_point() || input.is_complex(),
                "Input must be floating point or complex");
    TORCH_CHECK(weights.scalar_type() == input.scalar_type(),
                "Weights must have the same scalar type as input");
    TORCH_CHECK(input.dim() == 2, "Input must be 2D");
    TORCH_CHECK(weights.sizes() == input.sizes(), "Weights must have the same size as input");
    check_cuda(input, "input");
    check_cuda(weights, "weights");
    const int64_t B = input.size(0), T = input.size(1);
    at::Tensor init;
    if (init_opt.has_value() && init_opt->defined()) {
        init = *init_opt;
        TORCH_CHECK(init.scalar_type() == input.scalar_type(),
                    "Initials must have the same scalar type as input");
        TORCH_CHECK(init.dim() == 1, "Initials must be 1D");
        TORCH_CHECK(init.size(0) == B,
                    "The first dimension of initials must be the same as the first dimension of input");
        init = init.contiguous();
    }
    const int dt = dtype_code(input);
    const c10::cuda::CUDAGuard guard(input.device());
    at::Tensor ic = input.contiguous(), wc = weights.contiguous();
    at::Tensor out = at::empty({B, T}, input.options());
    const size_t wsb = lpc_b200_scan_workspace_size(dt, (int)algo, B, T);
    at::Tensor ws = workspace(wsb, input);
    auto stream = c10::cuda::getCurrentCUDAStream();
    check_status(lpc_b200_scan(dt, (int)algo, ic.data_ptr(), wc.data_ptr(), ptr_or_null(init),
                               out.data_ptr(), B, T, ptr_or_null(ws), wsb, stream.stream()),
                 "scan");
    return out;
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> scan_backward(
    const at::Tensor &grad_out, const at::Tensor &decay, const c10::optional<at::Tensor> &init_opt,
    const at::Tensor &out, bool need_decay, bool need_init, int64_t algo) {
    raise_pending();
    TORCH_CHECK(grad_out.dim() == 2 && grad_out.sizes() == out.sizes() && decay.sizes() == out.sizes(),
                "grad_out, decay and out must be (B, T)");
    check_cuda(grad_out, "grad_out");
    const int64_t B = out.size(0), T = out.size(1);
    at::Tensor init;
    if (init_opt.has_value() && init_opt->defined()) init = init_opt->contiguous();
    const int dt = dtype_code(out);
    const c10::cuda::CUDAGuard guard(out.device());
    at::Tensor goc = grad_out.contiguous(), dc = decay.contiguous(), oc = out.contiguous();
    at::Tensor gi = at::empty({B, T}, out.options());
    at::Tensor gd = need_decay ? at::empty({B, T}, out.options()) : at::empty({0}, out.options());
    at::Tensor g0 = need_init ? at::empty({B}, out.options()) : at::empty({0}, out.options());
    const size_t wsb = lpc_b200_scan_backward_workspace_size(dt, (int)algo, B, T);
    at::Tensor ws = workspace(wsb, out);
    auto stream = c10::cuda::getCurrentCUDAStream();
    check_status(lpc_b200_scan_backward(dt, (int)algo, goc.data_ptr(), dc.data_ptr(), ptr_or_null(init),
                                        oc.data_ptr(), gi.data_ptr(), need_decay ? gd.data_ptr() : nullptr,
                                        need_init ? g0.data_ptr() : nullptr, B, T, ptr_or_null(ws), wsb,
                                        stream.stream()),
                 "scan_backward");
    return {gi, gd, g0};
}

// Ragged batches: x (S,), A (S, N), offsets (nsig+1,) int64 on the same
// device, zi (nsig, N) or none.
void check_ragged(const at::Tensor &x, const at::Tensor &A, const at::Tensor &offsets) {
    TORCH_CHECK(x.dim() == 1, "ragged input must be 1D (S,)");
    TORCH_CHECK(A.dim() == 2 && A.size(0) == x.size(0), "ragged coefficients must be (S, order)");
    TORCH_CHECK(A.scalar_type() == x.scalar_type(), "Coefficients must have the same scalar type as input");
    TORCH_CHECK(offsets.dim() == 1 && offsets.size(0) >= 1 && offsets.scalar_type() == at::kLong,
                "offsets must be a 1D int64 tensor of nsig+1 sample offsets");
    check_cuda(x, "x");
    check_cuda(A, "A");
    check_cuda(offsets, "offsets");
    TORCH_CHECK(offsets.device() == x.device(), "offsets must be on the device of x");
}

at::Tensor lpc_ragged(const at::Tensor &x, const at::Tensor &A, const at::Tensor &offsets,
                      const c10::optional<at::Tensor> &zi_opt) {
    raise_pending();
    check_ragged(x, A, offsets);
    const int64_t S = x.size(0), N = A.size(1), nsig = offsets.size(0) - 1;
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = zi_opt->contiguous();
        TORCH_CHECK(zi.scalar_type() == x.scalar_type() && zi.dim() == 2 && zi.size(0) == nsig &&
                        zi.size(1) == N,
                    "Initial conditions must be (nsig, order) of the input's dtype");
    }
    const int dt = dtype_code(x);
    const c10::cuda::CUDAGuard guard(x.device());
    at::Tensor xc = x.contiguous(), ac = A.contiguous(), oc = offsets.contiguous();
    at::Tensor y = at::empty({S}, x.options());
    const size_t wsb = lpc_b200_ragged_workspace_size(dt, nsig, S, N);
    at::Tensor ws = workspace(wsb, x);
    check_status(lpc_b200_forward_ragged(dt, xc.data_ptr(), ac.data_ptr(), oc.data_ptr<int64_t>(),
                                         ptr_or_null(zi), y.data_ptr(), nsig, S, N, ptr_or_null(ws), wsb,
                                         c10::cuda::getCurrentCUDAStream().stream()),
                 "lpc_ragged");
    return y;
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> lpc_backward_ragged(
    const at::Tensor &grad_y, const at::Tensor &A, const at::Tensor &offsets,
    const c10::optional<at::Tensor> &zi_opt, const at::Tensor &y, bool need_A, bool need_zi) {
    raise_pending();
    check_ragged(y, A, offsets);
    TORCH_CHECK(grad_y.sizes() == y.sizes() && grad_y.scalar_type() == y.scalar_type(),
                "grad_y and y must both be (S,) of one dtype");
    check_cuda(grad_y, "grad_y");
    const int64_t S = y.size(0), N = A.size(1), nsig = offsets.size(0) - 1;
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = zi_opt->contiguous();
        TORCH_CHECK(zi.dim() == 2 && zi.size(0) == nsig && zi.size(1) == N, "zi must be (nsig, order)");
    }
    const int dt = dtype_code(y);
    const c10::cuda::CUDAGuard guard(y.device());
    at::Tensor gyc = grad_y.contiguous(), ac = A.contiguous(), oc = offsets.contiguous(), yc = y.contiguous();
    at::Tensor gx = at::empty({S}, y.options());
    at::Tensor gA = need_A ? at::empty({S, N}, y.options()) : at::Tensor();
    at::Tensor gzi = need_zi ? at::empty({nsig, N}, y.options()) : at::Tensor();
    const size_t wsb = lpc_b200_ragged_workspace_size(dt, nsig, S, N);
    at::Tensor ws = workspace(wsb, y);
    check_status(lpc_b200_backward_ragged(dt, gyc.data_ptr(), ac.data_ptr(), oc.data_ptr<int64_t>(),
                                          ptr_or_null(zi), yc.data_ptr(), gx.data_ptr(), ptr_or_null(gA),
                                          ptr_or_null(gzi), nsig, S, N, ptr_or_null(ws), wsb,
                                          c10::cuda::getCurrentCUDAStream().stream()),
                 "lpc_backward_ragged");
    if (!need_A) gA = at::empty({0}, y.options());
    if (!need_zi) gzi = at::empty({0}, y.options());
    return {gx, gA, gzi};
}

// Boundary-state checkpointing: the forward returns y and the chunk entry
// states; the backward takes x and those states instead of y.
std::tuple<at::Tensor, at::Tensor> lpc_checkpointed(const at::Tensor &x, const at::Tensor &A,
                                                    const c10::optional<at::Tensor> &zi_opt, int64_t chunk) {
    raise_pending();
    TORCH_CHECK(x.is_floating_point(), "Input must be floating point");
    TORCH_CHECK(A.scalar_type() == x.scalar_type(), "Coefficients must have the same scalar type as input");
    TORCH_CHECK(x.dim() == 2 && A.dim() == 3, "checkpointed filter: x (B,T), A (B,T,order)");
    check_cuda(x, "x");
    check_cuda(A, "A");
    const int64_t B = x.size(0), T = x.size(1), N = A.size(-1);
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = zi_opt->contiguous();
        TORCH_CHECK(zi.scalar_type() == x.scalar_type() && zi.dim() == 2 && zi.size(0) == B && zi.size(1) == N,
                    "Initial conditions must be (B, order) of the input's dtype");
    }
    const int dt = dtype_code(x);
    const c10::cuda::CUDAGuard guard(x.device());
    Coeffs c = coeffs(A, B, T, N, false);
    at::Tensor xc = x.contiguous();
    at::Tensor y = at::empty({B, T}, x.options());
    const int64_t ne = lpc_b200_checkpoint_elems(dt, B, T, N, chunk);
    TORCH_CHECK(ne > 0 || B * T == 0, "torchlpc_b200::lpc_checkpointed: unsupported order or chunk length");
    at::Tensor states = at::empty({std::max<int64_t>(ne, 0)}, x.options());
    const size_t wsb = lpc_b200_forward_checkpointed_workspace_size(dt, B, T, N, chunk);
    at::Tensor ws = workspace(wsb, x);
    check_status(lpc_b200_forward_checkpointed(dt, xc.data_ptr(), c.t.data_ptr(), ptr_or_null(zi), y.data_ptr(),
                                               states.data_ptr(), B, T, N, c.sb, c.st, chunk, ptr_or_null(ws),
                                               wsb, c10::cuda::getCurrentCUDAStream().stream()),
                 "lpc_checkpointed");
    return {y, states};
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> lpc_backward_checkpointed(
    const at::Tensor &grad_y, const at::Tensor &A, const c10::optional<at::Tensor> &zi_opt, const at::Tensor &x,
    const at::Tensor &states, int64_t chunk, bool need_A, bool need_zi) {
    raise_pending();
    TORCH_CHECK(grad_y.dim() == 2 && x.dim() == 2 && grad_y.sizes() == x.sizes(), "grad_y and x must be (B, T)");
    TORCH_CHECK(A.scalar_type() == x.scalar_type() && grad_y.scalar_type() == x.scalar_type() &&
                    states.scalar_type() == x.scalar_type(),
                "dtype mismatch");
    check_cuda(grad_y, "grad_y");
    check_cuda(A, "A");
    check_cuda(x, "x");
    check_cuda(states, "states");
    const int64_t B = x.size(0), T = x.size(1), N = A.size(-1);
    at::Tensor zi;
    if (zi_opt.has_value() && zi_opt->defined()) {
        zi = zi_opt->contiguous();
        TORCH_CHECK(zi.dim() == 2 && zi.size(0) == B && zi.size(1) == N, "zi must be (B, order)");
    }
    const int dt = dtype_code(x);
    TORCH_CHECK(states.numel() == std::max<int64_t>(lpc_b200_checkpoint_elems(dt, B, T, N, chunk), 0),
                "checkpoint states do not match (B, T, order, chunk length)");
    const c10::cuda::CUDAGuard guard(x.device());
    Coeffs c = coeffs(A, B, T, N, false);
    at::Tensor gyc = grad_y.contiguous(), xc = x.contiguous(), sc = states.contiguous();
    at::Tensor gx = at::empty({B, T}, x.options());
    at::Tensor gA = need_A ? at::empty({B, T, N}, x.options()) : at::Tensor();
    at::Tensor gzi = need_zi ? at::empty({B, N}, x.options()) : at::Tensor();
    const size_t wsb = lpc_b200_backward_checkpointed_workspace_size(dt, B, T, N, chunk);
    at::Tensor ws = workspace(wsb, x);
    check_status(lpc_b200_backward_checkpointed(dt, gyc.data_ptr(), c.t.data_ptr(), ptr_or_null(zi),
                                                xc.data_ptr(), sc.data_ptr(), gx.data_ptr(), ptr_or_null(gA),
                                                ptr_or_null(gzi), B, T, N, c.sb, c.st, chunk, ptr_or_null(ws), wsb,
                                                c10::cuda::getCurrentCUDAStream().stream()),
                 "lpc_backward_checkpointed");
    if (!need_A) gA = at::empty({0}, x.options());
    if (!need_zi) gzi = at::empty({0}, x.options());
    return {gx, gA, gzi};
}

// The error word: optionally synchronise the current stream, return the word
// and clear it.
int64_t check_status_op(bool synchronize) {
    if (synchronize) c10::cuda::getCurrentCUDAStream().synchronize();
    return (int64_t)take_error_word();
}

// Runs the library's bounded-wait self-test (a chunked forward whose
// look-back waits for a flag nothing sets, given up after spin_limit polls)
// with a workspace from the caching allocator on `like`'s device; returns the
// C status (LPC_ERR_TIMEOUT when the wait gave up as designed).  The give-up
// also reaches the error word, as any other would.
int64_t selftest_timeout_op(const at::Tensor &like, int64_t spin_limit) {
    check_cuda(like, "like");
    ensure_error_word();
    const c10::cuda::CUDAGuard guard(like.device());
    const size_t wsb = lpc_b200_selftest_workspace_size();
    at::Tensor ws = at::empty({(int64_t)wsb}, like.options().dtype(at::kByte));
    unsigned st = 0;
    return lpc_b200_selftest_timeout(ws.data_ptr(), wsb, (unsigned)spin_limit, &st,
                                     c10::cuda::getCurrentCUDAStream().stream());
}

at::Tensor cpu_refused_ragged(const at::Tensor &, const at::Tensor &, const at::Tensor &,
                              const c10::optional<at::Tensor> &) {
    TORCH_CHECK(false, "torchlpc_b200 runs on CUDA devices only (no CPU implementation)");
    return at::Tensor();
}

at::Tensor cpu_refused(const at::Tensor &, const at::Tensor &, const c10::optional<at::Tensor> &, int64_t) {
    TORCH_CHECK(false, "torchlpc_b200 runs on CUDA devices only (no CPU implementation)");
    return at::Tensor();
}

}  // namespace

TORCH_LIBRARY(torchlpc_b200, m) {
    m.def("lpc(Tensor x, Tensor A, Tensor? zi, int algo=0) -> Tensor");
    m.def("lpc_backward(Tensor grad_y, Tensor A, Tensor? zi, Tensor y, bool need_A, bool need_zi, "
          "int algo=0) -> (Tensor, Tensor, Tensor)");
    m.def("lpc_ragged(Tensor x, Tensor A, Tensor offsets, Tensor? zi) -> Tensor");
    m.def("lpc_backward_ragged(Tensor grad_y, Tensor A, Tensor offsets, Tensor? zi, Tensor y, bool need_A, "
          "bool need_zi) -> (Tensor, Tensor, Tensor)");
    m.def("lpc_checkpointed(Tensor x, Tensor A, Tensor? zi, int chunk) -> (Tensor, Tensor)");
    m.def("lpc_backward_checkpointed(Tensor grad_y, Tensor A, Tensor? zi, Tensor x, Tensor states, int chunk, "
          "bool need_A, bool need_zi) -> (Tensor, Tensor, Tensor)");
    m.def("check_status(bool synchronize) -> int", &check_status_op);
    m.def("selftest_timeout(Tensor like, int spin_limit) -> int");
    m.def("scan(Tensor input, Tensor weights, Tensor? initials, int algo=0) -> Tensor");
    m.def("scan_backward(Tensor grad_out, Tensor decay, Tensor? init, Tensor out, bool need_decay, "
          "bool need_init, int algo=0) -> (Tensor, Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(torchlpc_b200, CUDA, m) {
    m.impl("lpc", &lpc);
    m.impl("lpc_backward", &lpc_backward);
    m.impl("scan", &scan);
    m.impl("scan_backward", &scan_backward);
    m.impl("lpc_ragged", &lpc_ragged);
    m.impl("lpc_backward_ragged", &lpc_backward_ragged);
    m.impl("lpc_checkpointed", &lpc_checkpointed);
    m.impl("lpc_backward_checkpointed", &lpc_backward_checkpointed);
    m.impl("selftest_timeout", &selftest_timeout_op);
}

TORCH_LIBRARY_IMPL(torchlpc_b200, CPU, m) {
    m.impl("lpc", &cpu_refused);
    m.impl("scan", &cpu_refused);
    m.impl("lpc_ragged", &cpu_refused_ragged);
}
