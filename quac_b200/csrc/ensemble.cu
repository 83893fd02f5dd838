// Batched ensembles: thousands of independent Lindblad systems of uneven
// Hilbert dimension, each integrated to tmax with its own adaptive
// Dormand-Prince 5(4) step, in one persistent launch replayed from a CUDA
// graph.
//
// Work decomposition.  An instance is integrated by a group of gw warps
// (gw a power of two, 1 <= gw <= warps per CTA).  Groups of one item are
// consecutive warps of one CTA; an item holds up to W/gw instances of the
// same group size.  Items are ordered longest first (elements per thread)
// and pulled by the CTAs of a persistent grid from an atomic counter.
// Group size and CTA shape come from the autotuner (quac_ensemble_tune).
//
// Per instance the group stages the stage input x_s of the whole D x D
// density matrix and the instance's term tables in shared memory (the
// gathers of L.x read only shared memory); the state y and the stage
// derivatives live in a per-group slot of global scratch that stays in L2.
// Each thread owns the elements tid, tid + 32 gw, ... and is the only one
// reading or writing them in the slot, so only the shared-memory stage
// input needs group barriers.
//
// Precision modes.
//   0 (FP64): every L.x in complex128.
//   1 (FP32 right-hand side, FP64 state): K1 = L y and K7 = L y5 (the FSAL
//     stage) in complex128; stages 2..6 evaluate only the increment
//     dK_s = L (x_s - y) in complex64 (x_s - y = h sum_j a_sj K_j is small),
//     so K_s = K1 + dK_s keeps the FP64 K1; stage combinations, the state,
//     the error norm and the step controller stay FP64.
//
// There is no reference counterpart: QuaC integrates one system per
// time_step_sys call (qsystem.c:895-1098).  Each instance follows the
// equations and the step controller of time_step_sys with -ts_rk_type 5dp
// (basic controller, exponent -1/5, factor clamp [0.1, 10], step limits).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "runtime.h"

namespace quac {

bool compile_host(qsystem qs, int mode, HostProg &hp);

namespace {

// Dormand-Prince 5(4) tableau (Dormand & Prince 1980).
__constant__ double eA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.2, 0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
__constant__ double eE[7] = {35.0 / 384.0 - 5179.0 / 57600.0,
                             0.0,
                             500.0 / 1113.0 - 7571.0 / 16695.0,
                             125.0 / 192.0 - 393.0 / 640.0,
                             -2187.0 / 6784.0 + 92097.0 / 339200.0,
                             11.0 / 84.0 - 187.0 / 2100.0,
                             -1.0 / 40.0};

struct EnsInst {
  int id;          // caller's index
  int D, nL, nR, nJ, nJd;
  int gw;          // warps of the integrating group
  int tbytes;      // bytes of the packed tables (multiple of 16)
  int v32off;      // byte offset of the complex64 values in the table block
  int moff;        // byte offset of the maps in the table block
  long long toff;  // byte offset of the table block
  long long yoff;  // offset (complex values) of the state
  long long poff;  // offset of the populations (caller's order)
};

struct EnsItem {
  int first, count, gw, pad;
};

struct EnsStatus {
  double t, h;
  long long steps, rejected;
  int flags;   // 1: step limit reached, 2: non-finite error norm
  int redone;  // complex64 mode: steps whose estimate was taken again in complex128
  int f64_steps;  // complex64 mode: steps taken in complex128 after the error budget ran out
};

struct EnsParams {
  const EnsInst *inst;  // work order
  const unsigned char *tables;
  double2 *state;
  unsigned char *scratch;
  long long slot_bytes;  // per warp
  int slot_elems;        // per warp
  int arena_bytes;       // shared memory per warp
  EnsStatus *status;     // caller's order
  const EnsItem *items;
  int nitems;
  int *counter;
  double t0, tmax, h0, atol, rtol, hmin, hmax;
  long long max_steps;
  double redo_margin;    // complex64 mode: |err - 1| below this re-evaluates the step in complex128
  double f32_budget;     // complex64 mode: estimated accumulated complex64 error that switches an instance to complex128
};

__device__ __forceinline__ void cmac(double &ax, double &ay, double2 a, double2 b) {
  ax = fma(a.x, b.x, ax);
  ax = fma(-a.y, b.y, ax);
  ay = fma(a.x, b.y, ay);
  ay = fma(a.y, b.x, ay);
}
__device__ __forceinline__ void cmac(float &ax, float &ay, float2 a, float2 b) {
  ax = fmaf(a.x, b.x, ax);
  ax = fmaf(-a.y, b.y, ax);
  ay = fmaf(a.x, b.y, ay);
  ay = fmaf(a.y, b.x, ay);
}
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

// (L x)[r, c] for U elements at once (terms outer, elements inner: U
// independent FMA chains).  Tables in shared memory, element (r, c) at c*D + r:
//   (dr[r] + dc[c] + sum Jdr[r] Jdc[c]) x[r,c] + sum Lv[r] x[Lm[r], c]
//   + sum Rv[c] x[r, Rm[c]] + sum Jr[r] Jc[c] x[Jm[r], Jm[c]]
// Empty operator rows carry map 0 and value 0 (set on the host), so there
// is no branch on the maps.
template <int U, typename V, typename R>
__device__ __forceinline__ void eval_multi(const V *__restrict__ x, const V *__restrict__ vals,
                                           const int *__restrict__ maps, const int D, const int nL, const int nR,
                                           const int nJ, const int nJd, const int (&r)[U], const int (&c)[U],
                                           V (&out)[U]) {
  const V *Lv = vals, *Rv = Lv + nL * D, *Jr = Rv + nR * D, *Jc = Jr + nJ * D, *Jdr = Jc + nJ * D;
  const V *Jdc = Jdr + nJd * D, *dr = Jdc + nJd * D, *dc = dr + D;
  const int *Lm = maps, *Rm = Lm + nL * D, *Jm = Rm + nR * D;
  R ax[U], ay[U];
#pragma unroll
  for (int u = 0; u < U; u++) {
    const V a = dr[r[u]], b = dc[c[u]];
    R dx = a.x + b.x, dy = a.y + b.y;
    for (int t = 0; t < nJd; t++) cmac(dx, dy, Jdr[t * D + r[u]], Jdc[t * D + c[u]]);
    ax[u] = 0;
    ay[u] = 0;
    cmac(ax[u], ay[u], mk(dx, dy), x[c[u] * D + r[u]]);
  }
  for (int t = 0; t < nL; t++) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int p = Lm[t * D + r[u]];
      cmac(ax[u], ay[u], Lv[t * D + r[u]], x[c[u] * D + p]);
    }
  }
  for (int t = 0; t < nR; t++) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int q = Rm[t * D + c[u]];
      cmac(ax[u], ay[u], Rv[t * D + c[u]], x[q * D + r[u]]);
    }
  }
  for (int t = 0; t < nJ; t++) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int p = Jm[t * D + r[u]], q = Jm[t * D + c[u]];
      const V a = Jr[t * D + r[u]], b = Jc[t * D + c[u]];
      cmac(ax[u], ay[u], mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x), x[q * D + p]);
    }
  }
#pragma unroll
  for (int u = 0; u < U; u++) out[u] = mk(ax[u], ay[u]);
}

__device__ __forceinline__ void group_sync(int gi, int gw) {
  if (gw == 1) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(gi + 1), "r"(gw * 32) : "memory");
}

__device__ double group_sum(double v, int gi, int gw, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (gw == 1) return v;
  const int w = (int)(threadIdx.x >> 5) - gi * gw;
  if ((threadIdx.x & 31) == 0) red[gi * gw + w] = v;
  group_sync(gi, gw);
  double s = 0.0;
  for (int k = 0; k < gw; k++) s += red[gi * gw + k];
  group_sync(gi, gw);
  return s;
}

__device__ double group_max(double v, int gi, int gw, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (gw == 1) return v;
  const int w = (int)(threadIdx.x >> 5) - gi * gw;
  if ((threadIdx.x & 31) == 0) red[gi * gw + w] = v;
  group_sync(gi, gw);
  double s = 0.0;
  for (int k = 0; k < gw; k++) s = fmax(s, red[gi * gw + k]);
  group_sync(gi, gw);
  return s;
}

__device__ __forceinline__ double2 axpy(double2 y, double a, double2 x) {
  return make_double2(fma(a, x.x, y.x), fma(a, x.y, y.y));
}
__device__ __forceinline__ double2 axpy(double2 y, double a, float2 x) {
  return make_double2(fma(a, (double)x.x, y.x), fma(a, (double)x.y, y.y));
}

// Element iterator over e = start, start + step, ... < n with (r, c) = (e % D, e / D).
struct ElemIt {
  int e, r, c, dr, dc, D, n, step;
  __device__ ElemIt() {}
  __device__ ElemIt(int start, int step_, int D_) : e(start), D(D_), n(D_ * D_), step(step_) {
    c = start / D;
    r = start - c * D;
    dc = step / D;
    dr = step - dc * D;
  }
  __device__ __forceinline__ bool ok() const { return e < n; }
  __device__ __forceinline__ void next() {
    e += step;
    r += dr;
    c += dc;
    if (r >= D) { r -= D; c++; }
  }
};

// Calls f(e, r, c, ok) for this thread's elements lt, lt + gt, ... in rounds
// of U; lanes past the end get the round's first element with ok = false.
template <int U, typename F>
__device__ __forceinline__ void for_rounds(int lt, int gt, int D, F &&f) {
  ElemIt it[U];
#pragma unroll
  for (int u = 0; u < U; u++) it[u] = ElemIt(lt + u * gt, U * gt, D);
  while (it[0].ok()) {
    int e[U], r[U], c[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      ok[u] = it[u].ok();
      e[u] = ok[u] ? it[u].e : it[0].e;
      r[u] = ok[u] ? it[u].r : it[0].r;
      c[u] = ok[u] ? it[u].c : it[0].c;
    }
    f(e, r, c, ok);
#pragma unroll
    for (int u = 0; u < U; u++) it[u].next();
  }
}

template <int MODE, int U>
__device__ void integrate_instance(const EnsParams &P, const EnsInst &I, int gi, int gw, unsigned char *sm,
                                   double *red) {
  const int D = I.D, n = D * D;
  const int gt = 32 * gw;
  const int lt = (int)threadIdx.x - gi * gt;
  const int nL = I.nL, nR = I.nR, nJ = I.nJ, nJd = I.nJd;
  // tables -> shared memory (after the stage-input buffer)
  const int xbytes = ((n * 16 + 15) / 16) * 16;
  unsigned char *tb = sm + xbytes;
  {
    const uint4 *src = (const uint4 *)(P.tables + I.toff);
    uint4 *dst = (uint4 *)tb;
    for (int k = lt; k < I.tbytes / 16; k += gt) dst[k] = src[k];
  }
  const double2 *v64 = (const double2 *)tb;
  const float2 *v32 = (const float2 *)(tb + I.v32off);
  const int *maps = (const int *)(tb + I.moff);
  double2 *x64 = (double2 *)sm;
  float2 *x32 = (float2 *)sm;
  // slot scratch of the group: Yb | K1 | K7 | K2..K6 (MODE 0: complex128, MODE 1: complex64 increments)
  const int C = gw * P.slot_elems;
  unsigned char *slot = P.scratch + ((size_t)blockIdx.x * (blockDim.x >> 5) + (size_t)gi * gw) * P.slot_bytes;
  double2 *const ys = P.state + I.yoff, *const yb = (double2 *)slot;
  double2 *K1 = (double2 *)slot + C, *K7 = (double2 *)slot + 2 * (size_t)C;
  double2 *const Kb64 = (double2 *)slot + 3 * (size_t)C;  // K_{j+2} at Kb64 + j C
  float2 *const Kb32 = (float2 *)Kb64;                      // dK_{j+2} at Kb32 + j C
  int iy = 0;
  double t = P.t0, h = P.h0;
  long long steps = 0, rej = 0, redo = 0, f64_steps = 0;
  int flags = 0;
  // complex64 mode: estimated complex64 error accumulated by the accepted
  // steps; past P.f32_budget the instance continues in complex128
  double e32 = 0.0, dk_step = 0.0;
  bool all64 = MODE == 0;
  const double tend_tol = 1e-12 * fmax(1.0, fabs(P.tmax));
  double bsum = 0.0;
  for (int j = 0; j < 6; j++) bsum += eA[6][j];
  group_sync(gi, gw);

  auto eval64_into = [&](double2 *dst) {
    for_rounds<U>(lt, gt, D, [&](const int(&e)[U], const int(&r)[U], const int(&c)[U], const bool(&ok)[U]) {
      double2 o[U];
      eval_multi<U, double2, double>(x64, v64, maps, D, nL, nR, nJ, nJd, r, c, o);
#pragma unroll
      for (int u = 0; u < U; u++)
        if (ok[u]) dst[e[u]] = o[u];
    });
  };

  // K1 = L y (complex128)
  for (ElemIt it(lt, gt, D); it.ok(); it.next()) x64[it.e] = ys[it.e];
  group_sync(gi, gw);
  eval64_into(K1);
  group_sync(gi, gw);

  // one attempt of the step from (t, y) with length ht: stages 2..7 into
  // the slot, y5, and the weighted error norm; f64 = all stages complex128
  // (MODE 0, and MODE 1's re-evaluation near the accept threshold)
  auto attempt = [&](bool f64, double ht, const double2 *y, double2 *y5) -> double {
    for (int s = 1; s < 6; s++) {
      if (f64) {
        for_rounds<U>(lt, gt, D, [&](const int(&e)[U], const int(&)[U], const int(&)[U], const bool(&ok)[U]) {
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (!ok[u]) continue;
            double2 v = axpy(y[e[u]], ht * eA[s][0], K1[e[u]]);
            for (int j = 1; j < s; j++) v = axpy(v, ht * eA[s][j], Kb64[(size_t)(j - 1) * C + e[u]]);
            x64[e[u]] = v;
          }
        });
      } else {
        double cs = 0.0;
        for (int j = 0; j < s; j++) cs += eA[s][j];
        for_rounds<U>(lt, gt, D, [&](const int(&e)[U], const int(&)[U], const int(&)[U], const bool(&ok)[U]) {
#pragma unroll
          for (int u = 0; u < U; u++) {
            if (!ok[u]) continue;
            double2 v = axpy(make_double2(0.0, 0.0), ht * cs, K1[e[u]]);
            for (int j = 1; j < s; j++) v = axpy(v, ht * eA[s][j], Kb32[(size_t)(j - 1) * C + e[u]]);
            x32[e[u]] = make_float2((float)v.x, (float)v.y);
          }
        });
      }
      group_sync(gi, gw);
      if (f64) {
        eval64_into(Kb64 + (size_t)(s - 1) * C);
      } else {
        float2 *dst = Kb32 + (size_t)(s - 1) * C;
        for_rounds<U>(lt, gt, D, [&](const int(&e)[U], const int(&r)[U], const int(&c)[U], const bool(&ok)[U]) {
          float2 o[U];
          eval_multi<U, float2, float>(x32, v32, maps, D, nL, nR, nJ, nJd, r, c, o);
#pragma unroll
          for (int u = 0; u < U; u++)
            if (ok[u]) dst[e[u]] = o[u];
        });
      }
      group_sync(gi, gw);
    }
    // stage 7: y5 = y + h sum b_j K_j (complex128), K7 = L y5
    for_rounds<U>(lt, gt, D, [&](const int(&e)[U], const int(&)[U], const int(&)[U], const bool(&ok)[U]) {
#pragma unroll
      for (int u = 0; u < U; u++) {
        if (!ok[u]) continue;
        double2 v;
        if (f64) {
          v = axpy(y[e[u]], ht * eA[6][0], K1[e[u]]);
          for (int j = 1; j < 6; j++) v = axpy(v, ht * eA[6][j], Kb64[(size_t)(j - 1) * C + e[u]]);
        } else {
          v = axpy(y[e[u]], ht * bsum, K1[e[u]]);
          for (int j = 1; j < 6; j++) v = axpy(v, ht * eA[6][j], Kb32[(size_t)(j - 1) * C + e[u]]);
        }
        x64[e[u]] = v;
        y5[e[u]] = v;
      }
    });
    group_sync(gi, gw);
    eval64_into(K7);
    // error norm: h sum_j e_j K_j, weighted RMS (own elements only: no barrier needed)
    double loc = 0.0, dkloc = 0.0;
    for (ElemIt it(lt, gt, D); it.ok(); it.next()) {
      double2 er;
      if (f64) {
        er = axpy(make_double2(0.0, 0.0), ht * eE[0], K1[it.e]);
        for (int j = 1; j < 6; j++) er = axpy(er, ht * eE[j], Kb64[(size_t)(j - 1) * C + it.e]);
        er = axpy(er, ht * eE[6], K7[it.e]);
      } else {
        // sum_j e_j = 0, so sum_j e_j K_j = sum_{j=2..6} e_j dK_j + e_7 (K7 - K1)
        const double2 k1 = K1[it.e], k7 = K7[it.e];
        er = make_double2(ht * eE[6] * (k7.x - k1.x), ht * eE[6] * (k7.y - k1.y));
        double dk = 0.0;
        for (int j = 1; j < 6; j++) {
          const float2 d = Kb32[(size_t)(j - 1) * C + it.e];
          er = axpy(er, ht * eE[j], d);
          dk += fabs(eA[6][j]) * (fabs((double)d.x) + fabs((double)d.y));
        }
        dkloc = fmax(dkloc, dk);
      }
      const double2 a = y[it.e], b = y5[it.e];
      const double m = fmax(sqrt(a.x * a.x + a.y * a.y), sqrt(b.x * b.x + b.y * b.y));
      const double q = sqrt(er.x * er.x + er.y * er.y) / (P.atol + P.rtol * m);
      loc += q * q;
    }
    const double en = sqrt(group_sum(loc, gi, gw, red) / (double)n);
    // rounding of the complex64 increments in y5 = y + h sum_j b_j K_j:
    // about eps32 |b_j dK_j| per element and stage, with a factor 8 for
    // the complex64 sums inside each dK_j
    if (!f64) dk_step = 8.0 * 5.96e-8 * ht * group_max(dkloc, gi, gw, red);
    return en;
  };

  while (t < P.tmax - tend_tol) {
    if (steps >= P.max_steps) { flags |= 1; break; }
    bool last = false;
    double ht = h;
    if (t + ht >= P.tmax - tend_tol) { ht = P.tmax - t; last = true; }
    const double2 *y = iy ? yb : ys;
    double2 *y5 = iy ? ys : yb;
    dk_step = 0.0;
    double err = attempt(all64, ht, y, y5);
    // MODE 1: an estimate near the accept threshold is taken again with
    // complex128 stages, so accept / reject follows the complex128 decision
    if (MODE == 1 && !all64 && isfinite(err) && fabs(err - 1.0) < P.redo_margin) {
      group_sync(gi, gw);
      err = attempt(true, ht, y, y5);
      dk_step = 0.0;
      redo++;
    }
    if (!isfinite(err)) { flags |= 2; break; }
    double fac = err > 0 ? 0.9 * pow(err, -0.2) : 10.0;
    fac = fmin(10.0, fmax(0.1, fac));
    const double hnew = fmin(P.hmax, fmax(P.hmin, ht * fac));
    if (err <= 1.0 || ht <= P.hmin * (1 + 1e-12)) {
      iy ^= 1;
      double2 *tmp = K1;  // first same as last
      K1 = K7;
      K7 = tmp;
      t = last ? P.tmax : t + ht;
      steps++;
      if (MODE == 1) {
        if (all64) f64_steps++;
        e32 += dk_step;
        if (!(e32 <= P.f32_budget)) all64 = true;
      }
    } else {
      rej++;
    }
    h = hnew;
    group_sync(gi, gw);
  }
  if (iy == 1) {
    for (ElemIt it(lt, gt, D); it.ok(); it.next()) ys[it.e] = yb[it.e];
  }
  if (lt == 0) {
    EnsStatus st;
    st.t = t;
    st.h = h;
    st.steps = steps;
    st.rejected = rej;
    st.flags = flags;
    st.redone = (int)redo;
    st.f64_steps = (int)f64_steps;
    P.status[I.id] = st;
  }
}

template <int MODE, int NT>
__global__ void __launch_bounds__(NT) k_ensemble(const EnsParams P) {
  extern __shared__ __align__(16) unsigned char arena[];
  __shared__ int item_s;
  __shared__ double red[32];
  const int warp = (int)(threadIdx.x >> 5);
  for (;;) {
    if (threadIdx.x == 0) item_s = atomicAdd(P.counter, 1);
    __syncthreads();
    const int it = item_s;
    if (it >= P.nitems) break;
    const EnsItem item = P.items[it];
    const int gi = warp / item.gw;
    if (gi < item.count) {
      const EnsInst I = P.inst[item.first + gi];
      integrate_instance<MODE, (NT > 512 ? 1 : 2)>(P, I, gi, item.gw, arena + (size_t)gi * item.gw * P.arena_bytes, red);
    }
    __syncthreads();
  }
}

int device_attr(cudaDeviceAttr a) {
  int dev = 0, v = 0;
  QCUDA(cudaGetDevice(&dev));
  QCUDA(cudaDeviceGetAttribute(&v, a, dev));
  return v;
}

int num_sms_ens() { return device_attr(cudaDevAttrMultiProcessorCount); }

// Re(diag rho) of every instance (one warp per instance), caller's order.
__global__ void k_ens_diag(const EnsInst *inst, const double2 *state, double *out, int n) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= n) return;
  const EnsInst I = inst[w];
  for (int k = lane; k < I.D; k += 32) out[I.poff + k] = state[I.yoff + (long long)k * I.D + k].x;
}

}  // namespace
}  // namespace quac

using namespace quac;

// ---------------------------------------------------------------- host side
struct quac_ensemble_s {
  int64_t n = 0;
  std::vector<EnsInst> inst;  // caller's order, gw unset
  std::vector<unsigned char> tables;
  std::vector<long long> need_bytes;  // shared memory per instance
  long long total = 0;                // complex values of all states
  int mode = 0;
  double atol = 5e-7, rtol = 5e-7, hmin = 0.01, hmax = 1.0;
  long long max_steps = 1000000;
  double redo_margin = 0.1;
  double f32_budget = 1e-7;
  int warps = 16, cps = 1, ept = 8;  // launch shape
  // device
  unsigned char *d_tables = nullptr, *d_scratch = nullptr;
  double2 *d_state = nullptr;
  EnsInst *d_inst = nullptr;
  EnsStatus *d_status = nullptr;
  EnsItem *d_items = nullptr;
  int *d_counter = nullptr;
  size_t scratch_bytes = 0, items_cap = 0;
  cudaStream_t stream = nullptr;
  // graph of the current plan
  cudaGraphExec_t graph = nullptr;
  bool plan_valid = false;
  EnsParams params{};
  double key[4] = {0, 0, 0, 0};
  int grid = 0;
  size_t smem = 0;
  std::vector<EnsStatus> status;
  bool status_valid = false;
};

namespace {

int pow2_ceil(long long v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Shared memory a CTA of the given shape may use (bytes, per warp).
int arena_per_warp(int warps, int cps) {
  const int per_sm = device_attr(cudaDevAttrMaxSharedMemoryPerMultiprocessor);
  const int per_block = device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin);
  const int stat = 512;                       // item index + reduction slots, rounded up
  long long cta = per_sm / cps - 1024 - stat;  // 1 KB per CTA is reserved by the hardware
  cta = std::min<long long>(cta, per_block - stat);
  return (int)((cta / warps) / 16 * 16);
}

// Group size of every instance for a launch shape; false if one does not fit.
bool plan_groups(quac_ensemble E, int warps, int cps, int ept, std::vector<int> &gw, int arena) {
  gw.assign(E->n, 0);
  for (int64_t i = 0; i < E->n; i++) {
    const long long n2 = (long long)E->inst[i].D * E->inst[i].D;
    const long long fit = (E->need_bytes[i] + arena - 1) / arena;
    const long long want = (n2 + 32LL * ept - 1) / (32LL * ept);
    int g = pow2_ceil(std::max<long long>(1, std::max(fit, want)));
    if (g > warps) g = warps;
    while (g > 1 && warps / g > 15) g <<= 1;  // named barriers 1..15
    if ((long long)g * arena < E->need_bytes[i]) return false;
    gw[i] = g;
  }
  return true;
}

bool ens_fail(const char *msg) {
  fail(0, "ERROR! %s\n", msg);
  return false;
}

// Builds items, scratch and the launch parameters for the current shape.
bool build_plan(quac_ensemble E) {
  const int arena = arena_per_warp(E->warps, E->cps);
  std::vector<int> gw;
  if (!plan_groups(E, E->warps, E->cps, E->ept, gw, arena))
    return ens_fail("an ensemble instance does not fit the shared memory of this launch shape");
  // work order: group size descending, then size descending
  std::vector<int> order(E->n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const long long ea = (long long)E->inst[a].D * E->inst[a].D, eb = (long long)E->inst[b].D * E->inst[b].D;
    if (gw[a] != gw[b]) return gw[a] > gw[b];
    return ea > eb;
  });
  std::vector<EnsInst> work(E->n);
  std::vector<EnsItem> items;
  std::vector<long long> cost;
  long long slot_elems = 2;
  for (int64_t k = 0; k < E->n;) {
    const int g = gw[order[k]];
    const int per = E->warps / g;
    EnsItem it{(int)k, 0, g, 0};
    long long c = 0;
    while (k < E->n && it.count < per && gw[order[k]] == g) {
      EnsInst I = E->inst[order[k]];
      I.gw = g;
      work[k] = I;
      const long long n2 = (long long)I.D * I.D;
      slot_elems = std::max(slot_elems, (n2 + g - 1) / g);
      c = std::max(c, (n2 + 32LL * g - 1) / (32LL * g));
      it.count++;
      k++;
    }
    items.push_back(it);
    cost.push_back(c);
  }
  // longest first
  std::vector<int> io(items.size());
  std::iota(io.begin(), io.end(), 0);
  std::stable_sort(io.begin(), io.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<EnsItem> sorted(items.size());
  for (size_t k = 0; k < io.size(); k++) sorted[k] = items[io[k]];
  slot_elems = (slot_elems + 1) / 2 * 2;
  // complex128 stage storage in both modes: the complex64 mode re-evaluates
  // steps near the accept threshold with complex128 stages
  const long long bpe = 8 * 16;
  const int grid = num_sms_ens() * E->cps;
  const size_t need = (size_t)grid * E->warps * slot_elems * bpe;
  if (need > E->scratch_bytes) {
    if (E->d_scratch) QCUDA(cudaFree(E->d_scratch));
    E->d_scratch = nullptr;
    QCUDA(cudaMalloc(&E->d_scratch, need));
    E->scratch_bytes = need;
  }
  if (!E->d_inst) QCUDA(cudaMalloc(&E->d_inst, E->n * sizeof(EnsInst)));
  if (sorted.size() > E->items_cap) {
    if (E->d_items) QCUDA(cudaFree(E->d_items));
    QCUDA(cudaMalloc(&E->d_items, sorted.size() * sizeof(EnsItem)));
    E->items_cap = sorted.size();
  }
  QCUDA(cudaMemcpyAsync(E->d_inst, work.data(), E->n * sizeof(EnsInst), cudaMemcpyHostToDevice, E->stream));
  QCUDA(cudaMemcpyAsync(E->d_items, sorted.data(), sorted.size() * sizeof(EnsItem), cudaMemcpyHostToDevice,
                        E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  EnsParams &p = E->params;
  p.inst = E->d_inst;
  p.tables = E->d_tables;
  p.state = E->d_state;
  p.scratch = E->d_scratch;
  p.slot_bytes = slot_elems * bpe;
  p.slot_elems = (int)slot_elems;
  p.arena_bytes = arena;
  p.status = E->d_status;
  p.items = E->d_items;
  p.nitems = (int)sorted.size();
  p.counter = E->d_counter;
  p.atol = E->atol;
  p.rtol = E->rtol;
  p.hmin = E->hmin;
  p.hmax = E->hmax;
  p.max_steps = E->max_steps;
  p.redo_margin = E->redo_margin;
  p.f32_budget = E->f32_budget;
  E->grid = grid;
  E->smem = (size_t)arena * E->warps;
  E->plan_valid = true;
  if (E->graph) QCUDA(cudaGraphExecDestroy(E->graph));
  E->graph = nullptr;
  return !has_error();
}

}  // namespace

namespace {

template <int MODE, int NT>
void launch_ens(const EnsParams &p, int grid, int warps, size_t smem, cudaStream_t s, bool attr_only) {
  if (attr_only) {
    QCUDA(cudaFuncSetAttribute(k_ensemble<MODE, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return;
  }
  k_ensemble<MODE, NT><<<grid, warps * 32, smem, s>>>(p);
}

void launch_mode(quac_ensemble E, const EnsParams &p, bool attr_only) {
  if (E->mode == 0 && E->warps <= 16) launch_ens<0, 512>(p, E->grid, E->warps, E->smem, E->stream, attr_only);
  else if (E->mode == 0) launch_ens<0, 1024>(p, E->grid, E->warps, E->smem, E->stream, attr_only);
  else if (E->warps <= 16) launch_ens<1, 512>(p, E->grid, E->warps, E->smem, E->stream, attr_only);
  else launch_ens<1, 1024>(p, E->grid, E->warps, E->smem, E->stream, attr_only);
}

// Captures counter reset + persistent launch for (t0, tmax, dt0).
bool prepare_graph(quac_ensemble E, double t0, double tmax, double dt0) {
  if (!E->plan_valid && !build_plan(E)) return false;
  if (E->graph && E->key[0] == t0 && E->key[1] == tmax && E->key[2] == dt0 && E->key[3] == E->mode) return true;
  if (E->graph) QCUDA(cudaGraphExecDestroy(E->graph));
  E->graph = nullptr;
  EnsParams p = E->params;
  p.t0 = t0;
  p.tmax = tmax;
  p.h0 = dt0;
  launch_mode(E, p, true);  // shared-memory attribute, before the capture begins
  cudaGraph_t g = nullptr;
  QCUDA(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal));
  QCUDA(cudaMemsetAsync(E->d_counter, 0, sizeof(int), E->stream));
  launch_mode(E, p, false);
  const cudaError_t le = cudaGetLastError();
  QCUDA(cudaStreamEndCapture(E->stream, &g));
  QCUDA(le);
  if (has_error()) return false;
  QCUDA(cudaGraphInstantiate(&E->graph, g, 0));
  QCUDA(cudaGraphDestroy(g));
  E->key[0] = t0;
  E->key[1] = tmax;
  E->key[2] = dt0;
  E->key[3] = E->mode;
  return !has_error();
}

void launch_graph(quac_ensemble E) {
  QCUDA(cudaGraphLaunch(E->graph, E->stream));
  count_launch();
  E->status_valid = false;
}

bool read_status(quac_ensemble E) {
  if (E->status_valid) return true;
  E->status.resize(E->n);
  QCUDA(cudaMemcpyAsync(E->status.data(), E->d_status, E->n * sizeof(EnsStatus), cudaMemcpyDeviceToHost,
                        E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  E->status_valid = !has_error();
  return E->status_valid;
}

}  // namespace

extern "C" {

int quac_ensemble_create(quac_ensemble *out, int64_t n, const qsystem *systems) {
  *out = nullptr;
  if (n <= 0 || n > (1 << 24)) { fail(0, "ERROR! ensemble size %ld out of range\n", (long)n); return 1; }
  quac_ensemble E = new quac_ensemble_s();
  E->n = n;
  E->inst.resize(n);
  E->need_bytes.resize(n);
  long long yoff = 0, poff = 0;
  for (int64_t i = 0; i < n; i++) {
    HostProg hp;
    if (!systems[i]->impl->td.empty()) {
      fail(0, "ERROR! ensemble instance %ld has time-dependent terms (not supported in ensembles)\n", (long)i);
      delete E;
      return 1;
    }
    if (!compile_host(systems[i], 0, hp)) { delete E; return 1; }
    const int D = hp.D;
    if (hp.ncols != D || (long long)D * D > (1 << 24)) {
      fail(0, "ERROR! ensemble instance %ld: dimension %d not supported\n", (long)i, D);
      delete E;
      return 1;
    }
    EnsInst I{};
    I.id = (int)i;
    I.D = D;
    I.nL = (int)hp.Lmap.size();
    I.nR = (int)hp.Rmap.size();
    I.nJ = (int)hp.Jmap.size();
    I.nJd = (int)hp.Jdrow.size();
    // empty operator rows: map 0 with value 0, so the kernel needs no branch
    for (size_t t = 0; t < hp.Lmap.size(); t++)
      for (int k = 0; k < D; k++)
        if (hp.Lmap[t][k] < 0) { hp.Lmap[t][k] = 0; hp.Lval[t][k] = 0.0; }
    for (size_t t = 0; t < hp.Rmap.size(); t++)
      for (int k = 0; k < D; k++)
        if (hp.Rmap[t][k] < 0) { hp.Rmap[t][k] = 0; hp.Rval[t][k] = 0.0; }
    for (size_t t = 0; t < hp.Jmap.size(); t++)
      for (int k = 0; k < D; k++)
        if (hp.Jmap[t][k] < 0) { hp.Jmap[t][k] = 0; hp.Jrow[t][k] = 0.0; hp.Jcol[t][k] = 0.0; }
    std::vector<cplx> vals;
    for (auto *tab : {&hp.Lval, &hp.Rval, &hp.Jrow, &hp.Jcol, &hp.Jdrow, &hp.Jdcol})
      for (auto &m : *tab) vals.insert(vals.end(), m.begin(), m.end());
    vals.insert(vals.end(), hp.dr.begin(), hp.dr.end());
    vals.insert(vals.end(), hp.dc.begin(), hp.dc.end());
    std::vector<int> maps;
    for (auto *tab : {&hp.Lmap, &hp.Rmap, &hp.Jmap})
      for (auto &m : *tab) {
        for (int x : m)
          if (x < 0 || x >= D) {
            fail(0, "ERROR! ensemble instance %ld: corrupt term map\n", (long)i);
            delete E;
            return 1;
          }
        maps.insert(maps.end(), m.begin(), m.end());
      }
    const size_t nv = vals.size();
    I.v32off = (int)(nv * 16);
    I.moff = (int)((I.v32off + nv * 8 + 15) / 16 * 16);
    I.tbytes = (int)((I.moff + maps.size() * 4 + 15) / 16 * 16);
    I.toff = (long long)E->tables.size();
    E->tables.resize(E->tables.size() + I.tbytes, 0);
    unsigned char *b = E->tables.data() + I.toff;
    for (size_t k = 0; k < nv; k++) {
      const double v64[2] = {vals[k].real(), vals[k].imag()};
      const float v32[2] = {(float)vals[k].real(), (float)vals[k].imag()};
      memcpy(b + 16 * k, v64, 16);
      memcpy(b + I.v32off + 8 * k, v32, 8);
    }
    memcpy(b + I.moff, maps.data(), maps.size() * 4);
    I.yoff = yoff;
    I.poff = poff;
    yoff += (long long)D * D;
    poff += D;
    E->inst[i] = I;
    E->need_bytes[i] = ((long long)D * D * 16 + 15) / 16 * 16 + I.tbytes;
  }
  E->total = yoff;
  QCUDA(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  QCUDA(cudaMalloc(&E->d_tables, E->tables.size()));
  QCUDA(cudaMemcpy(E->d_tables, E->tables.data(), E->tables.size(), cudaMemcpyHostToDevice));
  QCUDA(cudaMalloc(&E->d_state, E->total * sizeof(double2)));
  QCUDA(cudaMemset(E->d_state, 0, E->total * sizeof(double2)));
  QCUDA(cudaMalloc(&E->d_status, n * sizeof(EnsStatus)));
  QCUDA(cudaMalloc(&E->d_counter, sizeof(int)));
  if (has_error()) { quac_ensemble_destroy(E); return 1; }
  *out = E;
  return 0;
}

int quac_ensemble_destroy(quac_ensemble E) {
  if (!E) return 0;
  if (E->graph) cudaGraphExecDestroy(E->graph);
  for (void *p : {(void *)E->d_tables, (void *)E->d_scratch, (void *)E->d_state, (void *)E->d_inst,
                  (void *)E->d_status, (void *)E->d_items, (void *)E->d_counter})
    if (p) cudaFree(p);
  if (E->stream) cudaStreamDestroy(E->stream);
  delete E;
  return 0;
}

int quac_ensemble_set_options(quac_ensemble E, int precision, double atol, double rtol, double hmin, double hmax,
                              int64_t max_steps) {
  if (precision != 0 && precision != 1) { fail(0, "ERROR! ensemble precision must be 0 (FP64) or 1 (FP32 RHS)\n"); return 1; }
  if (!(atol > 0) || !(rtol >= 0) || !(hmin > 0) || !(hmax >= hmin) || max_steps <= 0) {
    fail(0, "ERROR! invalid ensemble step options\n");
    return 1;
  }
  E->mode = precision;
  E->atol = atol;
  E->rtol = rtol;
  E->hmin = hmin;
  E->hmax = hmax;
  E->max_steps = max_steps;
  E->plan_valid = false;
  return 0;
}

int quac_ensemble_set_redo_margin(quac_ensemble E, double margin) {
  if (!(margin >= 0.0) || margin > 1.0) { fail(0, "ERROR! ensemble redo margin must lie in [0, 1]\n"); return 1; }
  E->redo_margin = margin;
  E->plan_valid = false;
  return 0;
}

int quac_ensemble_set_fp32_budget(quac_ensemble E, double budget) {
  if (!(budget >= 0.0)) { fail(0, "ERROR! ensemble complex64 error budget must be >= 0\n"); return 1; }
  E->f32_budget = budget;
  return 0;
}

int64_t quac_ensemble_f64_steps(quac_ensemble E, int64_t i) {
  if (i < 0 || i >= E->n) { fail(0, "ERROR! ensemble index out of range\n"); return -1; }
  if (!read_status(E)) return -1;
  return E->status[i].f64_steps;
}

int64_t quac_ensemble_redone_steps(quac_ensemble E, int64_t i) {
  if (i < 0 || i >= E->n) { fail(0, "ERROR! ensemble index out of range\n"); return -1; }
  if (!read_status(E)) return -1;
  return E->status[i].redone;
}

int quac_ensemble_set_shape(quac_ensemble E, int warps, int ctas_per_sm, int elems_per_thread) {
  if (!(warps == 4 || warps == 8 || warps == 16 || warps == 32) || ctas_per_sm < 1 || ctas_per_sm > 4 ||
      elems_per_thread < 1 || elems_per_thread > 4096) {
    fail(0, "ERROR! invalid ensemble launch shape\n");
    return 1;
  }
  std::vector<int> gw;
  if (!plan_groups(E, warps, ctas_per_sm, elems_per_thread, gw, arena_per_warp(warps, ctas_per_sm))) {
    fail(0, "ERROR! an ensemble instance does not fit the shared memory of this launch shape\n");
    return 1;
  }
  E->warps = warps;
  E->cps = ctas_per_sm;
  E->ept = elems_per_thread;
  E->plan_valid = false;
  return 0;
}

int quac_ensemble_get_shape(quac_ensemble E, int *warps, int *ctas_per_sm, int *elems_per_thread) {
  *warps = E->warps;
  *ctas_per_sm = E->cps;
  *elems_per_thread = E->ept;
  return 0;
}

int64_t quac_ensemble_state_offset(quac_ensemble E, int64_t i) {
  if (i < 0 || i > E->n) return -1;
  return i == E->n ? E->total : E->inst[i].yoff;
}

void *quac_ensemble_state_device_ptr(quac_ensemble E) { return E->d_state; }

int quac_ensemble_set_states(quac_ensemble E, const PetscScalar *rho) {
  QCUDA(cudaMemcpyAsync(E->d_state, rho, E->total * sizeof(double2), cudaMemcpyHostToDevice, E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  return has_error() ? 1 : 0;
}

int quac_ensemble_get_states(quac_ensemble E, PetscScalar *rho) {
  QCUDA(cudaMemcpyAsync(rho, E->d_state, E->total * sizeof(double2), cudaMemcpyDeviceToHost, E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  return has_error() ? 1 : 0;
}

int quac_ensemble_run(quac_ensemble E, double t0, double tmax, double dt0) {
  if (!(tmax >= t0) || !(dt0 > 0)) { fail(0, "ERROR! invalid ensemble time span\n"); return 1; }
  if (!prepare_graph(E, t0, tmax, dt0)) return 1;
  launch_graph(E);
  if (!read_status(E)) return 1;
  int64_t bad = 0;
  for (int64_t i = 0; i < E->n; i++)
    if (E->status[i].flags) bad++;
  if (bad) {
    fail(0, "ERROR! %ld ensemble instances did not reach the final time\n", (long)bad);
    return 1;
  }
  return 0;
}

int quac_ensemble_get_stats(quac_ensemble E, int64_t i, double *t, int64_t *steps, int64_t *rejected, int *flags) {
  if (i < 0 || i >= E->n) { fail(0, "ERROR! ensemble index out of range\n"); return 1; }
  if (!read_status(E)) return 1;
  const EnsStatus &s = E->status[i];
  if (t) *t = s.t;
  if (steps) *steps = s.steps;
  if (rejected) *rejected = s.rejected;
  if (flags) *flags = s.flags;
  return 0;
}

int quac_ensemble_populations(quac_ensemble E, double *pops_host) {
  double *d = nullptr;
  long long np = 0;
  for (auto &I : E->inst) np += I.D;
  EnsInst *du = nullptr;
  QCUDA(cudaMallocAsync(&d, np * sizeof(double), E->stream));
  QCUDA(cudaMallocAsync(&du, E->n * sizeof(EnsInst), E->stream));
  QCUDA(cudaMemcpyAsync(du, E->inst.data(), E->n * sizeof(EnsInst), cudaMemcpyHostToDevice, E->stream));
  const int threads = 256;
  const int blocks = (int)((E->n * 32 + threads - 1) / threads);
  k_ens_diag<<<blocks, threads, 0, E->stream>>>(du, E->d_state, d, (int)E->n);
  count_launch();
  QCUDA(cudaGetLastError());
  QCUDA(cudaMemcpyAsync(pops_host, d, np * sizeof(double), cudaMemcpyDeviceToHost, E->stream));
  QCUDA(cudaFreeAsync(d, E->stream));
  QCUDA(cudaFreeAsync(du, E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  return has_error() ? 1 : 0;
}

// Times each candidate launch shape on a short run from the current states
// (t0 .. t0 + t_probe), keeps the fastest and restores the states.
int quac_ensemble_tune(quac_ensemble E, double t0, double t_probe, double dt0, double *best_ms) {
  if (!(t_probe > 0) || !(dt0 > 0)) { fail(0, "ERROR! invalid tuning span\n"); return 1; }
  double2 *snap = nullptr;
  QCUDA(cudaMalloc(&snap, E->total * sizeof(double2)));
  QCUDA(cudaMemcpyAsync(snap, E->d_state, E->total * sizeof(double2), cudaMemcpyDeviceToDevice, E->stream));
  cudaEvent_t a, b;
  QCUDA(cudaEventCreate(&a));
  QCUDA(cudaEventCreate(&b));
  const int W0 = E->warps, C0 = E->cps, P0 = E->ept;
  double best = 1e300;
  int bw = W0, bc = C0, bp = P0;
  for (int warps : {8, 16, 32})
    for (int cps : {1, 2})
      for (int ept : {2, 4, 8, 16, 32}) {
        std::vector<int> gw;
        if (!plan_groups(E, warps, cps, ept, gw, arena_per_warp(warps, cps))) continue;
        E->warps = warps;
        E->cps = cps;
        E->ept = ept;
        E->plan_valid = false;
        if (!prepare_graph(E, t0, t0 + t_probe, dt0)) break;
        QCUDA(cudaMemcpyAsync(E->d_state, snap, E->total * sizeof(double2), cudaMemcpyDeviceToDevice, E->stream));
        QCUDA(cudaEventRecord(a, E->stream));
        launch_graph(E);
        QCUDA(cudaEventRecord(b, E->stream));
        QCUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        QCUDA(cudaEventElapsedTime(&ms, a, b));
        if (has_error()) break;
        if (ms < best) {
          best = ms;
          bw = warps;
          bc = cps;
          bp = ept;
        }
      }
  E->warps = bw;
  E->cps = bc;
  E->ept = bp;
  E->plan_valid = false;
  QCUDA(cudaMemcpyAsync(E->d_state, snap, E->total * sizeof(double2), cudaMemcpyDeviceToDevice, E->stream));
  QCUDA(cudaStreamSynchronize(E->stream));
  QCUDA(cudaFree(snap));
  QCUDA(cudaEventDestroy(a));
  QCUDA(cudaEventDestroy(b));
  if (best_ms) *best_ms = best;
  return has_error() ? 1 : 0;
}

}  // extern "C"
