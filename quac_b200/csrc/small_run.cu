// Small density-matrix systems with a device-side observable monitor.
//
// QuaC programs read populations from a TS monitor after every step
// (examples/simple_jc_test.c:76-90); done on the host, each step costs a
// handful of launches and a host round trip while the state is a few KB.
// Here one CTA keeps the whole state and the Runge-Kutta stage vectors in
// shared memory and runs many fixed RK4 steps in one launch, writing the
// expectation values Tr(O rho) of the registered observables after every
// step into a device buffer; the host hands them to the caller's callback
// in batches.  The L.x inside is the generic term-table form of the other
// kernels (dr, dc, left / right Hamiltonian maps, jumps) read from L1.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "runtime.h"

namespace quac {

namespace {

constexpr int ST = 512;

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// (L x)[i] for element i = c * D + r, x in shared memory
__device__ __forceinline__ double2 lx_elem(const DevProg &P, const double2 *x, int r, int c) {
  const int D = P.D;
  const double2 xs = x[c * D + r];
  double2 d = __ldg(P.dr + r);
  const double2 dcc = __ldg(P.dc + c);
  d.x += dcc.x;
  d.y += dcc.y;
  double2 acc = cm(d, xs);
  for (int t = 0; t < P.nJd; t++) {
    const double2 f = cm(__ldg(P.Jdrow + (size_t)t * D + r), __ldg(P.Jdcol + (size_t)t * D + c));
    const double2 v = cm(f, xs);
    acc.x += v.x;
    acc.y += v.y;
  }
  for (int t = 0; t < P.nL; t++) {
    const int p = __ldg(P.Lmap + (size_t)t * D + r);
    if (p < 0) continue;
    const double2 v = cm(__ldg(P.Lval + (size_t)t * D + r), x[c * D + p]);
    acc.x += v.x;
    acc.y += v.y;
  }
  for (int t = 0; t < P.nR; t++) {
    const int q = __ldg(P.Rmap + (size_t)t * D + c);
    if (q < 0) continue;
    const double2 v = cm(__ldg(P.Rval + (size_t)t * D + c), x[q * D + r]);
    acc.x += v.x;
    acc.y += v.y;
  }
  for (int t = 0; t < P.nJ; t++) {
    const int p = __ldg(P.Jmap + (size_t)t * D + r);
    if (p < 0) continue;
    const int q = __ldg(P.Jmap + (size_t)t * D + c);
    if (q < 0) continue;
    const double2 f = cm(__ldg(P.Jrow + (size_t)t * D + r), __ldg(P.Jcol + (size_t)t * D + c));
    const double2 v = cm(f, x[q * D + p]);
    acc.x += v.x;
    acc.y += v.y;
  }
  return acc;
}

// out[i] = base[i] + h * (L x)[i]
__device__ __forceinline__ void stage(const DevProg &P, const double2 *x, const double2 *base, double2 *out,
                                      double h) {
  const int D = P.D, n = D * D;
  for (int i = threadIdx.x; i < n; i += ST) {
    const int c = i / D, r = i - c * D;
    const double2 k = lx_elem(P, x, r, c);
    const double2 b = base[i];
    out[i] = make_double2(fma(h, k.x, b.x), fma(h, k.y, b.y));
  }
  __syncthreads();
}

// nsteps fixed RK4 steps of length h (Horner form of the degree-4 Taylor
// polynomial, identical to the four-stage form for constant L), then the
// observables after every step: values[step * nobs + o] = sum_c
// oval[o][c] rho[omap[o][c], c]
__global__ void __launch_bounds__(ST, 1) k_small_rk4(const DevProg P, double2 *state, int nsteps, double h, int nobs,
                                                     const int *omap, const double2 *oval, double2 *values) {
  extern __shared__ __align__(16) double2 sm[];
  __shared__ double2 red[ST / 32];
  const int D = P.D, n = D * D;
  double2 *y = sm, *va = sm + n, *vb = sm + 2 * n;
  for (int i = threadIdx.x; i < n; i += ST) y[i] = state[i];
  __syncthreads();
  for (int st = 0; st < nsteps; st++) {
    stage(P, y, y, va, 0.25 * h);
    stage(P, va, y, vb, h / 3.0);
    stage(P, vb, y, va, 0.5 * h);
    stage(P, va, y, y, h);  // element i of y is read and rewritten by the same thread
    for (int o = 0; o < nobs; o++) {
      double2 s = make_double2(0.0, 0.0);
      for (int c = threadIdx.x; c < D; c += ST) {
        const int j = __ldg(omap + (size_t)o * D + c);
        if (j >= 0) {
          const double2 v = cm(__ldg(oval + (size_t)o * D + c), y[c * D + j]);
          s.x += v.x;
          s.y += v.y;
        }
      }
      for (int k = 16; k > 0; k >>= 1) {
        s.x += __shfl_down_sync(0xffffffffu, s.x, k);
        s.y += __shfl_down_sync(0xffffffffu, s.y, k);
      }
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
      __syncthreads();
      if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int w = 0; w < ST / 32; w++) {
          t.x += red[w].x;
          t.y += red[w].y;
        }
        values[(size_t)st * nobs + o] = t;
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < n; i += ST) state[i] = y[i];
}

}  // namespace

constexpr int64_t SMALL_MAX_ELEMS = 4096;  // three stage vectors in 192 KB of shared memory

// Whether the one-CTA kernel can hold the system's state and stage vectors.
bool small_rk4_eligible(const DeviceProgram &P) {
  return P.dev.ncols == P.dev.D && (int64_t)P.dev.D * P.dev.D <= SMALL_MAX_ELEMS;
}

// nsteps fixed RK4 steps of length h on the device-resident state, the
// observables recorded after each one into values (nsteps x nobs)
void launch_small_rk4(const DeviceProgram &P, double2 *state, int nsteps, double h, int nobs, const int *omap,
                      const double2 *oval, double2 *values, cudaStream_t s) {
  const size_t smem = 3 * (size_t)P.dev.D * P.dev.D * sizeof(double2);
  ensure_smem((const void *)k_small_rk4, smem);
  k_small_rk4<<<1, ST, smem, s>>>(P.dev, state, nsteps, h, nobs, omap, oval, values);
  count_launch();
  QCUDA(cudaGetLastError());
}

}  // namespace quac
