// Linear combinations of stage vectors for the multi-stage integrators:
//   out[i] = base[i] + sum_j coef[j] * in_j[i]            (up to 8 inputs)
// optionally accumulating the weighted error norm of the combination
//   sum_i (|out_i - base_i| / (atol + rtol * max(|base_i|, |ref_i|)))^2
// (mode 1: out is not written, only the norm of sum_j coef_j in_j is taken
// against base and ref).
#include <cmath>

#include "common.h"

namespace quac {

namespace {

constexpr int NT = 256;

struct LinArgs {
  const double2 *in[8];
  double coef[8];
  int nin;
  const double2 *base;
  double2 *out;
  const double2 *ref;  // second vector of the error weight (norm mode)
  double atol, rtol;
  double *nsum;        // norm accumulator (norm mode)
};

__global__ void k_lincomb(const LinArgs A, int64_t n) {
  __shared__ double red[NT / 32];
  double loc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    double2 s = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (j < A.nin) {
        const double2 v = A.in[j][i];
        s.x = fma(A.coef[j], v.x, s.x);
        s.y = fma(A.coef[j], v.y, s.y);
      }
    }
    if (A.nsum) {
      const double2 b = A.base[i], r = A.ref[i];
      const double m = fmax(sqrt(b.x * b.x + b.y * b.y), sqrt(r.x * r.x + r.y * r.y));
      const double q = sqrt(s.x * s.x + s.y * s.y) / (A.atol + A.rtol * m);
      loc += q * q;
    } else {
      const double2 b = A.base ? A.base[i] : make_double2(0.0, 0.0);
      A.out[i] = make_double2(b.x + s.x, b.y + s.y);
    }
  }
  if (A.nsum) {
    for (int o = 16; o > 0; o >>= 1) loc += __shfl_down_sync(0xffffffffu, loc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; w++) t += red[w];
      atomicAdd(A.nsum, t);
    }
  }
}

int grid_of(int64_t n) {
  int64_t b = (n + NT - 1) / NT;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

// sums[0] += ||A - B^H||^2 over the block, sums[1] += ||A||^2, where A is
// the 32 x 32 block (bi, bj) of X and B the block (bj, bi)
__global__ void k_herm_asym(const double2 *__restrict__ x, int64_t D, double *sums) {
  __shared__ double2 tb[32][33];
  __shared__ double red[2][8];
  const int64_t r0 = (int64_t)blockIdx.x * 32, c0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // block (bj, bi) -> tb, element (c0 + i, r0 + j) stored at tb[j][i]
  for (int i = ty; i < 32; i += 8) {
    const int64_t row = c0 + tx, col = r0 + i;
    tb[i][tx] = (row < D && col < D) ? x[col * D + row] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double a2 = 0.0, d2 = 0.0;
  for (int j = ty; j < 32; j += 8) {
    const int64_t row = r0 + tx, col = c0 + j;
    if (row < D && col < D) {
      const double2 a = x[col * D + row];   // X[row, col]
      const double2 b = tb[tx][j];          // X[col, row]
      const double dx = a.x - b.x, dy = a.y + b.y;
      d2 += dx * dx + dy * dy;
      a2 += a.x * a.x + a.y * a.y;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_down_sync(0xffffffffu, d2, o);
    a2 += __shfl_down_sync(0xffffffffu, a2, o);
  }
  if (tx == 0) { red[0][ty] = d2; red[1][ty] = a2; }
  __syncthreads();
  if (tx == 0 && ty == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int k = 0; k < 8; k++) { s0 += red[0][k]; s1 += red[1][k]; }
    atomicAdd(&sums[0], s0);
    atomicAdd(&sums[1], s1);
  }
}

// y[i] += a * x[i] (complex a): one time-dependent term's contribution
__global__ void k_caxpy(double2 *__restrict__ y, const double2 *__restrict__ x, double2 a, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const double2 v = x[i];
    double2 w = y[i];
    w.x = fma(a.x, v.x, fma(-a.y, v.y, w.x));
    w.y = fma(a.x, v.y, fma(a.y, v.x, w.y));
    y[i] = w;
  }
}

// The stage epilogue of the fused L.x kernels (Epi) applied to a given
// K = L x: kout, up to three updates base_u + coef_u K and the error norm
__global__ void k_epilogue(const double2 *__restrict__ K, const Epi E, int64_t n) {
  __shared__ double red[NT / 32];
  double loc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const double2 k = K[i];
    if (E.kout) E.kout[i] = k;
    double2 u[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int j = 0; j < E.nupd; j++) {
      const double2 b = E.base[j] ? E.base[j][i] : make_double2(0.0, 0.0);
      u[j] = make_double2(fma(E.coef[j], k.x, b.x), fma(E.coef[j], k.y, b.y));
      E.out[j][i] = u[j];
    }
    if (E.nsum) {
      const double2 ev = u[E.err_upd];
      const double2 y = E.ny[i];
      const double2 yn = E.yn_upd >= 0 ? u[E.yn_upd] : E.nyn[i];
      const double q = sqrt(ev.x * ev.x + ev.y * ev.y) /
                       (E.atol + E.rtol * fmax(sqrt(y.x * y.x + y.y * y.y), sqrt(yn.x * yn.x + yn.y * yn.y)));
      loc += q * q;
    }
  }
  if (E.nsum) {
    for (int o = 16; o > 0; o >>= 1) loc += __shfl_down_sync(0xffffffffu, loc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = loc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; w++) t += red[w];
      atomicAdd(E.nsum, t);
    }
  }
}

}  // namespace

void launch_caxpy(double2 *y, const double2 *x, cplx a, int64_t n, cudaStream_t s) {
  k_caxpy<<<grid_of(n), NT, 0, s>>>(y, x, make_double2(a.real(), a.imag()), n);
  count_launch();
  QCUDA(cudaGetLastError());
}

void launch_epilogue(const double2 *K, const Epi &e, int64_t n, cudaStream_t s) {
  k_epilogue<<<grid_of(n), NT, 0, s>>>(K, e, n);
  count_launch();
  QCUDA(cudaGetLastError());
}

void launch_lincomb(double2 *out, const double2 *base, int nin, const double2 *const *in,
                    const double *coef, int64_t n, cudaStream_t s) {
  LinArgs A;
  memset(&A, 0, sizeof(A));
  A.nin = nin;
  for (int j = 0; j < nin; j++) { A.in[j] = in[j]; A.coef[j] = coef[j]; }
  A.base = base;
  A.out = out;
  k_lincomb<<<grid_of(n), NT, 0, s>>>(A, n);
  count_launch();
  QCUDA(cudaGetLastError());
}

void launch_lincomb_norm(const double2 *base, const double2 *ref, int nin, const double2 *const *in,
                         const double *coef, int64_t n, double atol, double rtol, double *nsum,
                         cudaStream_t s) {
  LinArgs A;
  memset(&A, 0, sizeof(A));
  A.nin = nin;
  for (int j = 0; j < nin; j++) { A.in[j] = in[j]; A.coef[j] = coef[j]; }
  A.base = base;
  A.ref = ref;
  A.atol = atol;
  A.rtol = rtol;
  A.nsum = nsum;
  k_lincomb<<<grid_of(n), NT, 0, s>>>(A, n);
  count_launch();
  QCUDA(cudaGetLastError());
}

double hermitian_asymmetry(const double2 *x, int64_t D, cudaStream_t s) {
  double *d = nullptr;
  double h[2] = {0.0, 0.0};
  QCUDA(cudaMallocAsync(&d, 2 * sizeof(double), s));
  QCUDA(cudaMemsetAsync(d, 0, 2 * sizeof(double), s));
  const unsigned nb = (unsigned)((D + 31) / 32);
  k_herm_asym<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(x, D, d);
  count_launch();
  QCUDA(cudaMemcpyAsync(h, d, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaFreeAsync(d, s));
  QCUDA(cudaStreamSynchronize(s));
  return h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
}

}  // namespace quac
