// fj_xla.cc -- XLA FFI handlers over the C ABI of libfj_uvlm.so, for JAX callers.
//
// The reference's aero path calls compute_v_ind (aero/aic.py:208-310, imported by name at
// aero/uvlm.py:15) and jnp.linalg.solve (aero/uvlm.py:985); these handlers let
// flapjax_b200/fj_jax.py bind the same operations as jax.ffi custom calls, with
// jax.custom_vjp rules that call the adjoint twins (fj_vind_vjp, fj_lu_solve_t).
//
// Built only where jaxlib's FFI headers exist (python -m flapjax_b200.build --xla, which
// takes the include directory from jax.ffi.include_dir()); these machines have no jaxlib.
// Every handler runs on the stream XLA passes and returns fj_last_error_string() on error.
#include <cuda_runtime.h>

#include "fj_uvlm.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status(int st) {
    return st == FJ_OK ? ffi::Error::Success() : ffi::Error(ffi::ErrorCode::kInternal, fj_last_error_string());
}

// One lattice zeta (rows+1, cols+1, 3) with circulations gamma (rows, cols).
struct Lattice {
    const double* z;
    const double* g;
    int rows, cols;
};

Lattice lattice(const ffi::Buffer<ffi::F64>& zeta, const ffi::Buffer<ffi::F64>& gamma) {
    const auto d = gamma.dimensions();
    return {zeta.typed_data(), gamma.typed_data(), (int)d[0], (int)d[1]};
}

// compute_v_ind of one lattice at the targets (n, 3); mirror (6,) = point, normal, used
// when has_mirror != 0 (the image is subtracted, aero/aic.py:294-308).
ffi::Error VInd(cudaStream_t stream, ffi::Buffer<ffi::F64> targets, ffi::Buffer<ffi::F64> zeta,
                ffi::Buffer<ffi::F64> gamma, ffi::Buffer<ffi::U8> ws, ffi::Span<const double> mirror,
                int64_t has_mirror, int64_t kernel, double r_cut, int64_t precision, ffi::ResultBuffer<ffi::F64> v) {
    const Lattice L = lattice(zeta, gamma);
    const double* mp = has_mirror ? mirror.begin() : nullptr;
    const double* mn = has_mirror ? mirror.begin() + 3 : nullptr;
    return status(fj_vind(targets.typed_data(), (int64_t)targets.element_count() / 3, &L.z, &L.g, &L.rows, &L.cols,
                          1, mp, mn, (int)kernel, r_cut, (int)precision, v->typed_data(), ws.typed_data(),
                          ws.element_count(), (fj_stream_t)stream));
}

// Cotangents of compute_v_ind of one lattice: target, vertex and circulation adjoints of
// the velocity cotangent lam (n, 3), zeroed here and accumulated by fj_vind_vjp.
ffi::Error VIndVjp(cudaStream_t stream, ffi::Buffer<ffi::F64> targets, ffi::Buffer<ffi::F64> zeta,
                   ffi::Buffer<ffi::F64> gamma, ffi::Buffer<ffi::F64> lam, ffi::Buffer<ffi::U8> ws, int64_t kernel,
                   double r_cut, ffi::ResultBuffer<ffi::F64> t_bar, ffi::ResultBuffer<ffi::F64> z_bar,
                   ffi::ResultBuffer<ffi::F64> g_bar) {
    const Lattice L = lattice(zeta, gamma);
    cudaMemsetAsync(t_bar->typed_data(), 0, t_bar->size_bytes(), stream);
    cudaMemsetAsync(z_bar->typed_data(), 0, z_bar->size_bytes(), stream);
    cudaMemsetAsync(g_bar->typed_data(), 0, g_bar->size_bytes(), stream);
    double* zb = z_bar->typed_data();
    double* gb = g_bar->typed_data();
    return status(fj_vind_vjp(targets.typed_data(), (int64_t)targets.element_count() / 3, &L.z, &L.g, &L.rows,
                              &L.cols, 1, nullptr, nullptr, (int)kernel, r_cut, lam.typed_data(), t_bar->typed_data(),
                              &zb, &gb, ws.typed_data(), ws.element_count(), (fj_stream_t)stream));
}

// getrf of the row-major (n, n) a into lu (a copy) and 0-based pivot rows.
ffi::Error LuFactor(cudaStream_t stream, ffi::Buffer<ffi::F64> a, ffi::Buffer<ffi::U8> ws,
                    ffi::ResultBuffer<ffi::F64> lu, ffi::ResultBuffer<ffi::S32> piv) {
    const int n = (int)a.dimensions()[0];
    cudaMemcpyAsync(lu->typed_data(), a.typed_data(), a.size_bytes(), cudaMemcpyDeviceToDevice, stream);
    return status(fj_lu_factor(lu->typed_data(), n, piv->typed_data(), ws.typed_data(), ws.element_count(),
                               (fj_stream_t)stream));
}

// x = A^-1 b (transpose = 0) or A^-T b (transpose = 1) from the factors.
ffi::Error LuSolve(cudaStream_t stream, ffi::Buffer<ffi::F64> lu, ffi::Buffer<ffi::S32> piv, ffi::Buffer<ffi::F64> b,
                   ffi::Buffer<ffi::U8> ws, int64_t transpose, ffi::ResultBuffer<ffi::F64> x) {
    const int n = (int)lu.dimensions()[0];
    cudaMemcpyAsync(x->typed_data(), b.typed_data(), b.size_bytes(), cudaMemcpyDeviceToDevice, stream);
    auto fn = transpose ? fj_lu_solve_t : fj_lu_solve;
    return status(fn(lu.typed_data(), n, piv.typed_data(), x->typed_data(), ws.typed_data(), ws.element_count(),
                     (fj_stream_t)stream));
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(FjVInd, VInd,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::U8>>()
                                  .Attr<ffi::Span<const double>>("mirror")
                                  .Attr<int64_t>("has_mirror")
                                  .Attr<int64_t>("kernel")
                                  .Attr<double>("r_cut")
                                  .Attr<int64_t>("precision")
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(FjVIndVjp, VIndVjp,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::U8>>()
                                  .Attr<int64_t>("kernel")
                                  .Attr<double>("r_cut")
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(FjLuFactor, LuFactor,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::U8>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::S32>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(FjLuSolve, LuSolve,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::S32>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::U8>>()
                                  .Attr<int64_t>("transpose")
                                  .Ret<ffi::Buffer<ffi::F64>>());
