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

// Systems of at most ST elements: each thread's element keeps its terms as
// (index into x, coefficient) pairs in registers, built once per launch in
// the order lx_elem visits them (diagonal, diagonal jumps, left, right,
// jumps), so a stage is KREG independent shared-memory reads and the same
// floating-point operations as lx_elem, in the same order.
constexpr int KREG = 12;

struct TermList {
  int idx[KREG];
  double2 coef[KREG];
  int n;
};

__device__ __forceinline__ void tl_put(TermList &L, int idx, double2 coef, bool &over) {
  if (L.n >= KREG) {
    over = true;
    return;
  }
#pragma unroll
  for (int j = 0; j < KREG; j++)
    if (j == L.n) {
      L.idx[j] = idx;
      L.coef[j] = coef;
    }
  L.n++;
}

__device__ void build_terms(const DevProg &P, int r, int c, TermList &L, bool &over) {
  const int D = P.D, i = c * D + r;
  L.n = 0;
  double2 d = __ldg(P.dr + r);
  const double2 dcc = __ldg(P.dc + c);
  d.x += dcc.x;
  d.y += dcc.y;
  tl_put(L, i, d, over);
  for (int t = 0; t < P.nJd; t++)
    tl_put(L, i, cm(__ldg(P.Jdrow + (size_t)t * D + r), __ldg(P.Jdcol + (size_t)t * D + c)), over);
  for (int t = 0; t < P.nL; t++) {
    const int p = __ldg(P.Lmap + (size_t)t * D + r);
    if (p >= 0) tl_put(L, c * D + p, __ldg(P.Lval + (size_t)t * D + r), over);
  }
  for (int t = 0; t < P.nR; t++) {
    const int q = __ldg(P.Rmap + (size_t)t * D + c);
    if (q >= 0) tl_put(L, q * D + r, __ldg(P.Rval + (size_t)t * D + c), over);
  }
  for (int t = 0; t < P.nJ; t++) {
    const int p = __ldg(P.Jmap + (size_t)t * D + r);
    const int q = __ldg(P.Jmap + (size_t)t * D + c);
    if (p >= 0 && q >= 0)
      tl_put(L, q * D + p, cm(__ldg(P.Jrow + (size_t)t * D + r), __ldg(P.Jcol + (size_t)t * D + c)), over);
  }
}

// out[i] = base[i] + h * (L x)[i] from the thread's term list (i < n only)
__device__ __forceinline__ void stage_reg(const TermList &L, int i, bool mine, const double2 *x,
                                          const double2 *base, double2 *out, double h) {
  if (mine) {
    double2 acc = cm(L.coef[0], x[L.idx[0]]);
#pragma unroll
    for (int k = 1; k < KREG; k++)
      if (k < L.n) {
        const double2 v = cm(L.coef[k], x[L.idx[k]]);
        acc.x += v.x;
        acc.y += v.y;
      }
    const double2 b = base[i];
    out[i] = make_double2(fma(h, acc.x, b.x), fma(h, acc.y, b.y));
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
  // one element per thread and at most KREG terms each: term lists in
  // registers (a uniform decision for the whole CTA)
  TermList TL;
  TL.n = 0;
  bool over = n > ST;
  const int me = threadIdx.x;
  const bool mine = me < n;
  if (!over && mine) build_terms(P, me - (me / D) * D, me / D, TL, over);
  const bool reg = !__syncthreads_or(over);
  for (int st = 0; st < nsteps; st++) {
    if (reg) {
      stage_reg(TL, me, mine, y, y, va, 0.25 * h);
      stage_reg(TL, me, mine, va, y, vb, h / 3.0);
      stage_reg(TL, me, mine, vb, y, va, 0.5 * h);
      stage_reg(TL, me, mine, va, y, y, h);  // element i of y is read and rewritten by the same thread
    } else {
      stage(P, y, y, va, 0.25 * h);
      stage(P, va, y, vb, h / 3.0);
      stage(P, vb, y, va, 0.5 * h);
      stage(P, va, y, y, h);
    }
    if (D <= 32) {
      // every observable lives in warp 0 (one lane per column): shuffle
      // sums, no block barrier; the same values as the block reduction
      // below (the other warps' partial sums are zero)
      if (threadIdx.x < 32)
        for (int o = 0; o < nobs; o++) {
          double2 s = make_double2(0.0, 0.0);
          const int c = threadIdx.x;
          if (c < D) {
            const int j = __ldg(omap + (size_t)o * D + c);
            if (j >= 0) s = cm(__ldg(oval + (size_t)o * D + c), y[c * D + j]);
          }
          for (int k = 16; k > 0; k >>= 1) {
            s.x += __shfl_down_sync(0xffffffffu, s.x, k);
            s.y += __shfl_down_sync(0xffffffffu, s.y, k);
          }
          if (threadIdx.x == 0) values[(size_t)st * nobs + o] = s;
        }
      continue;
    }
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
