// y = L x on caller buffers without any device allocation at call time.
//
// The multi-pass bit-mask kernel keeps a running sum of D^2 complex values
// between its passes.  quac_lrho_apply_device allocates that buffer with
// cudaMalloc on its first call for a system; this variant uses a fixed
// file-scope device array instead, so a call neither allocates nor frees
// device memory (and so never triggers the device-wide synchronisation of
// cudaFree, nor competes with a caller's own memory pool).
//
// Limits and rules:
//   - at most kNoAllocMaxElems = 2^20 complex values per vector (16 MiB of
//     scratch: a 10-qubit density matrix); larger systems are rejected;
//   - quac_lrho_noalloc_setup must be called once per system, with the
//     system's device current, before the first apply: it compiles the
//     term program if needed, looks up the scratch
//     address of the current device and loads every kernel the apply can
//     launch (CUDA's lazy module loading would otherwise load, and allocate
//     device memory for, a kernel at its first launch);
//   - the apply follows quac_set_lrho_precision like quac_lrho_apply_device
//     (complex128 or complex64 contraction) and returns once the result is
//     complete;
//   - the scratch is shared by every system on a device: calls that overlap
//     in time (two host threads, or two streams) race on it and give wrong
//     results; serialise them.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>

#include "runtime.h"

namespace quac {
namespace {

constexpr size_t kNoAllocMaxElems = size_t(1) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocMaxElems];

std::atomic<double2 *> g_scratch_of_device[kMaxDevices];

}  // namespace
}  // namespace quac

using namespace quac;

extern "C" int quac_lrho_noalloc_setup(qsystem qs) {
  if (qs->mat_allocated != 1) { fail(0, "ERROR! call construct_matrix first\n"); return 1; }
  int dev = -1;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    fail(0, "ERROR! quac_lrho_noalloc_setup: no usable current device (%s)\n", cudaGetErrorString(rc));
    return 1;
  }
  void *addr = nullptr;
  rc = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
  if (rc != cudaSuccess || addr == nullptr) {
    fail(0, "ERROR! quac_lrho_noalloc_setup: cudaGetSymbolAddress failed on device %d (%s)\n", dev,
         cudaGetErrorString(rc));
    return 1;
  }
  g_scratch_of_device[dev].store((double2 *)addr);
  stream_of(qs);
  ensure_program(qs);
  if (has_error() || !qs->impl->prog) return 1;
  preload_lrho_kernels(*qs->impl->prog);
  return has_error() ? 1 : 0;
}

extern "C" int quac_lrho_apply_device_noalloc(qsystem qs, const void *x_dev, void *y_dev) {
  if (qs->mat_allocated != 1) { fail(0, "ERROR! call construct_matrix first\n"); return 1; }
  if (!qs->impl->td.empty()) {
    fail(0, "ERROR! quac_lrho_apply_device_noalloc: time-dependent terms need quac_lrho_apply_device\n");
    return 1;
  }
  const int mode = qs->dm_equations ? 0 : 1;
  if (!qs->impl->prog || qs->impl->prog_mode != mode) {
    fail(0, "ERROR! call quac_lrho_noalloc_setup on this system before quac_lrho_apply_device_noalloc\n");
    return 1;
  }
  DeviceProgram &P = *qs->impl->prog;
  const size_t n = (size_t)P.dev.D * P.dev.ncols;
  if (n > kNoAllocMaxElems) {
    fail(0, "ERROR! quac_lrho_apply_device_noalloc: %zu complex values exceed the fixed scratch of %zu\n", n,
         kNoAllocMaxElems);
    return 1;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices || !g_scratch_of_device[dev].load()) {
    fail(0, "ERROR! quac_lrho_apply_device_noalloc: quac_lrho_noalloc_setup was not called on this device\n");
    return 1;
  }
  Epi e;
  zero_epi(e);
  e.kout = (double2 *)y_dev;
  cudaStream_t s = stream_of(qs);
  if (P.has_qubit && !P.passes.empty()) {
    // the first pass writes the running sum without reading it, so only the
    // time-limit error word has to start at zero
    if (P.errflag) QCUDA(cudaMemsetAsync(P.errflag, 0, sizeof(int), s));
    launch_qubit_passes(P.passes, (const double2 *)x_dev, g_scratch_of_device[dev].load(), e, s,
                        options().lrho_f32 != 0);
  } else {
    // the single-pass kernels use no scratch
    launch_lrho_any(P, (const double2 *)x_dev, e, s);
  }
  QCUDA(cudaStreamSynchronize(s));
  check_program_error(P, s);
  return has_error() ? 1 : 0;
}
