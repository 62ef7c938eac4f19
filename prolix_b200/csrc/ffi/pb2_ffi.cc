// XLA FFI handlers over the C ABI: what a prolix maintainer registers with
// jax.ffi.register_ffi_target so that make_energy_fn(..., implicit_solvent=True)
// and the BAOAB apply_fn run on these kernels inside a jitted JAX program.
//
// The reference's pattern for a hand-written kernel is a jax.custom_vjp
// whose forward returns the energy and whose backward returns the analytic
// forces (prolix physics/optimization.py:21-126); pb2_ffi_energy_forces
// gives both in one call.  pb2_ffi_baoab is the functional apply_fn
// (physics/settle.py:1698-1744): state in, n steps, state out.
//
// Each handler takes the batch handle (pb2_batch *, created once per
// system topology with pb2_batch_create) as an int64 attribute and works on
// the buffers XLA hands it, on XLA's stream: it allocates nothing and does
// not synchronise.
//
// Built only when the XLA FFI headers are present (python -m
// prolix_b200._build --ffi /path/to/xla/include, or PB2_XLA_FFI_INCLUDE);
// this image has no JAX, so it is neither built nor tested here.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "prolix_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status_error(int rc, const char *what) {
  if (rc == PB2_OK) return ffi::Error::Success();
  return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + " failed with status " +
                                                   std::to_string(rc));
}

// positions (n, 3) f64 -> energies (n_systems, PB2_NTERMS) f64, forces (n, 3) f64
ffi::Error EnergyForces(cudaStream_t stream, int64_t batch, ffi::Buffer<ffi::F64> positions,
                        ffi::ResultBuffer<ffi::F64> energies, ffi::ResultBuffer<ffi::F64> forces) {
  auto *b = reinterpret_cast<pb2_batch *>(batch);
  int32_t n_sys = 0;
  int64_t n_atoms = 0;
  if (int rc = pb2_batch_info(b, &n_sys, &n_atoms)) return status_error(rc, "pb2_batch_info");
  if (positions.element_count() != static_cast<size_t>(3 * n_atoms) ||
      forces->element_count() != static_cast<size_t>(3 * n_atoms) ||
      energies->element_count() != static_cast<size_t>(n_sys) * PB2_NTERMS)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "buffer sizes do not match the batch");
  return status_error(pb2_energy_forces_device(b, positions.typed_data(), energies->typed_data(),
                                               forces->typed_data(), stream),
                      "pb2_energy_forces_device");
}

// (x, p, f) (n, 3) f64 each -> the state n_steps BAOAB steps later, in new buffers
ffi::Error Baoab(cudaStream_t stream, int64_t batch, int64_t n_steps, ffi::Buffer<ffi::F64> x,
                 ffi::Buffer<ffi::F64> p, ffi::Buffer<ffi::F64> f, ffi::ResultBuffer<ffi::F64> x_out,
                 ffi::ResultBuffer<ffi::F64> p_out, ffi::ResultBuffer<ffi::F64> f_out) {
  auto *b = reinterpret_cast<pb2_batch *>(batch);
  const size_t bytes = x.size_bytes();
  if (p.size_bytes() != bytes || f.size_bytes() != bytes || x_out->size_bytes() != bytes)
    return ffi::Error(ffi::ErrorCode::kInvalidArgument, "state buffers differ in size");
  // the entry point works in place: copy the inputs into the result buffers first
  if (cudaMemcpyAsync(x_out->typed_data(), x.typed_data(), bytes, cudaMemcpyDeviceToDevice, stream) ||
      cudaMemcpyAsync(p_out->typed_data(), p.typed_data(), bytes, cudaMemcpyDeviceToDevice, stream) ||
      cudaMemcpyAsync(f_out->typed_data(), f.typed_data(), bytes, cudaMemcpyDeviceToDevice, stream))
    return ffi::Error(ffi::ErrorCode::kInternal, "state copy failed");
  return status_error(pb2_langevin_run_device(b, x_out->typed_data(), p_out->typed_data(),
                                              f_out->typed_data(), static_cast<int32_t>(n_steps),
                                              stream),
                      "pb2_langevin_run_device");
}

}  // namespace

XLA_FFI_DEFINE_HANDLER_SYMBOL(pb2_ffi_energy_forces, EnergyForces,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("batch")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(pb2_ffi_baoab, Baoab,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Attr<int64_t>("batch")
                                  .Attr<int64_t>("n_steps")
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Arg<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>()
                                  .Ret<ffi::Buffer<ffi::F64>>());
