// Steady state: solve (L + e0 vec(I)^T) x = e0 by restarted GMRES on the
// GPU (solver.c:33-221 does the same system with PETSc KSPGMRES(100),
// rtol 1e-11, x0 = b = e0; row 0 carries the trace functional,
// solver.c:60-75).
//
// Every vector operation runs on device buffers; the Krylov basis V is one
// (m+1) x n block so the Gram-Schmidt projections are two streaming
// kernels per pass (multi-dot, multi-axpy), repeated once (CGS2).  Only the
// (m+1) x m Hessenberg matrix lives on the host.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <cstring>
#include <type_traits>
#include <vector>

#include "runtime.h"

namespace quac {

namespace {

constexpr int NT = 256;
constexpr int CHUNK = 1024;  // largest chunk of w staged per block (multi-dot)
constexpr int FUSE_NB = 32;  // small-n path (n <= FUSE_NB * 256): multi-dot partials per projection
constexpr int CGS_EB = 32;   // small-n Gram-Schmidt: elements per block
constexpr int CGS_KG = 8;    //   and k-groups per element (CGS_EB * CGS_KG threads)
constexpr int GMRES_MAXM = 1024;  // largest restart length
// Arnoldi steps are queued up to GMRES_LAG ahead of the host's Givens
// updates; their Hessenberg columns come back through GMRES_RING slots.
constexpr int GMRES_LAG = 2;
constexpr int GMRES_RING = 4;
static_assert(GMRES_RING > GMRES_LAG, "a slot is reused only after the host has read it");

__device__ __forceinline__ double2 cmuls(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// Krylov basis elements: complex128, or complex64 in the FP32-inner solver
// (every product and sum is still formed in double precision).
__device__ __forceinline__ double2 ldv(const double2 *p) { return *p; }
__device__ __forceinline__ double2 ldv(const float2 *p) {
  const float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void stv(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void stv(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// y[0] += sum_i x[i*(D+1)]  (the stabilising trace row); slice z of a batch
// works on x + z*D*D and y + z*D*D
__global__ void k_trace_add(const double2 *__restrict__ x, double2 *__restrict__ y, int64_t D) {
  __shared__ double2 red[NT / 32];
  x += (size_t)blockIdx.z * D * D;
  y += (size_t)blockIdx.z * D * D;
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = threadIdx.x; i < D; i += NT) {
    const double2 v = x[i * (D + 1)];
    acc.x += v.x; acc.y += v.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = make_double2(0.0, 0.0);
    for (int w = 0; w < NT / 32; w++) { s.x += red[w].x; s.y += red[w].y; }
    y[0].x += s.x;
    y[0].y += s.y;
  }
}

// partial[k*nb + blk] = sum over this block's chunk (chunk <= CHUNK
// elements) of conj(V_k[i]) w[i].  The chunk of w is staged in shared
// memory; each warp then takes one basis vector k = blockIdx.y * 8 + warp,
// so all projections run side by side (grid nb x ceil(nk / 8)).
// A batch (gridDim.z > 1) projects w + z*n into partial + z*nk*nb.
template <typename VT>
__device__ __forceinline__ void multidot_body(const VT *__restrict__ V, const double2 *__restrict__ w, int64_t n,
                                              int nk, double2 *__restrict__ partial, int chunk) {
  __shared__ double2 ws[CHUNK];
  w += (size_t)blockIdx.z * n;
  partial += (size_t)blockIdx.z * nk * gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * chunk;
  const int len = (int)min((int64_t)chunk, n - i0);
  for (int i = threadIdx.x; i < len; i += NT) ws[i] = w[i0 + i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.y * (NT / 32) + (threadIdx.x >> 5);
  if (k >= nk) return;
  const VT *vk = V + (size_t)k * n + i0;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
  for (int i = lane; i < len; i += 32) {
    double2 a = ldv(vk + i);
    a.y = -a.y;
    const double2 p = cmuls(a, ws[i]);
    acc.x += p.x; acc.y += p.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if (lane == 0) partial[(size_t)k * gridDim.x + blockIdx.x] = acc;
}

template <typename VT>
__global__ void k_multidot(const VT *__restrict__ V, const double2 *__restrict__ w, int64_t n,
                           int nk, double2 *__restrict__ partial, int chunk) {
  multidot_body(V, w, n, nk, partial, chunk);
}

// Graph form: nk = *jp + 1 read on the device (the grid is sized for the
// longest restart; blocks past nk leave at once).
template <typename VT>
__global__ void k_multidot_j(const VT *__restrict__ V, const double2 *__restrict__ w, int64_t n,
                             const int *__restrict__ jp, double2 *__restrict__ partial, int chunk) {
  const int nk = *jp + 1;
  if ((int)blockIdx.y * (NT / 32) >= nk) return;
  multidot_body(V, w, n, nk, partial, chunk);
}

// h[k] (+)= sum_b partial[k*nb + b]; one block per k.  accumulate != 0 adds.
__global__ void k_reduce_rows(const double2 *__restrict__ partial, int nb, double2 *__restrict__ h,
                              int accumulate) {
  __shared__ double2 red[NT / 32];
  const int k = blockIdx.x;
  double2 acc = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < nb; b += NT) {
    acc.x += partial[(size_t)k * nb + b].x;
    acc.y += partial[(size_t)k * nb + b].y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = make_double2(0.0, 0.0);
    for (int q = 0; q < NT / 32; q++) { s.x += red[q].x; s.y += red[q].y; }
    if (accumulate) { h[k].x += s.x; h[k].y += s.y; }
    else h[k] = s;
  }
}

// w[i] -= sum_k c[k] V_k[i]   (c = the projections just computed)
template <typename VT>
__global__ void k_multiaxpy(const VT *__restrict__ V, const double2 *__restrict__ c, int64_t n,
                            int nk, double2 *__restrict__ w, double sign) {
  __shared__ double2 cs[GMRES_MAXM + 1];
  for (int k = threadIdx.x; k < nk; k += NT) cs[k] = c[k];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    double2 acc = w[i];
    for (int k = 0; k < nk; k++) {
      const double2 p = cmuls(cs[k], ldv(V + (size_t)k * n + i));
      acc.x = fma(sign, p.x, acc.x);
      acc.y = fma(sign, p.y, acc.y);
    }
    w[i] = acc;
  }
}

// w[i] -= sum_k c[k] V_k[i], and npart[block] = sum over the block's i of |w[i]|^2
// (the second Gram-Schmidt pass fused with the norm of the result).
template <typename VT>
__global__ void k_multiaxpy_norm(const VT *__restrict__ V, const double2 *__restrict__ c, int64_t n,
                                 int nk, double2 *__restrict__ w, double *__restrict__ npart) {
  __shared__ double2 cs[GMRES_MAXM + 1];
  __shared__ double red[NT / 32];
  for (int k = threadIdx.x; k < nk; k += NT) cs[k] = c[k];
  __syncthreads();
  double ss = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    double2 acc = w[i];
    for (int k = 0; k < nk; k++) {
      const double2 p = cmuls(cs[k], ldv(V + (size_t)k * n + i));
      acc.x -= p.x;
      acc.y -= p.y;
    }
    w[i] = acc;
    ss = fma(acc.x, acc.x, fma(acc.y, acc.y, ss));
  }
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < NT / 32; q++) t += red[q];
    npart[blockIdx.x] = t;
  }
}

// h[k] += h2[k] for k < nk; h[nk] = (sqrt(sum npart), 0).  One block.
__global__ void k_arnoldi_finish(double2 *__restrict__ h, const double2 *__restrict__ h2, int nk,
                                 const double *__restrict__ npart, int nparts) {
  __shared__ double red[NT / 32];
  for (int k = threadIdx.x; k < nk; k += NT) {
    h[k].x += h2[k].x;
    h[k].y += h2[k].y;
  }
  double ss = 0.0;
  for (int b = threadIdx.x; b < nparts; b += NT) ss += npart[b];
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < NT / 32; q++) t += red[q];
    h[nk] = make_double2(sqrt(t), 0.0);
  }
}

// Small-n Gram-Schmidt pass (nb <= FUSE_NB multi-dot partials per
// projection): every block sums the projections h_k = sum_b partial[k][b]
// itself (fixed order; block 0 stores them in hout), then
// w[i] -= sum_k h_k V_k[i] with CGS_KG k-groups per element, combined in a
// fixed order.  NORM: npart[block] = sum of |w[i]|^2 over its elements.
template <typename VT, bool NORM>
__device__ __forceinline__ void cgs_small_body(const VT *__restrict__ V, const double2 *__restrict__ partial, int nb,
                                               int nk, int64_t n, double2 *__restrict__ w,
                                               double2 *__restrict__ hout, double *__restrict__ npart) {
  __shared__ double2 cs[GMRES_MAXM + 1];
  __shared__ double2 red[CGS_KG][CGS_EB];
  __shared__ double nred[CGS_EB / 32 > 0 ? CGS_EB / 32 : 1];
  for (int k = threadIdx.x; k < nk; k += CGS_EB * CGS_KG) {
    double2 acc = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; b++) {
      const double2 v = partial[(size_t)k * nb + b];
      acc.x += v.x; acc.y += v.y;
    }
    cs[k] = acc;
    if (blockIdx.x == 0) hout[k] = acc;
  }
  __syncthreads();
  const int e = threadIdx.x % CGS_EB, g = threadIdx.x / CGS_EB;
  const int64_t i = (int64_t)blockIdx.x * CGS_EB + e;
  double2 acc = make_double2(0.0, 0.0);
  if (i < n) {
#pragma unroll 4
    for (int k = g; k < nk; k += CGS_KG) {
      const double2 p = cmuls(cs[k], ldv(V + (size_t)k * n + i));
      acc.x += p.x; acc.y += p.y;
    }
  }
  red[g][e] = acc;
  __syncthreads();
  if (g == 0) {
    double ss = 0.0;
    if (i < n) {
      double2 t = red[0][e];
      for (int q = 1; q < CGS_KG; q++) { t.x += red[q][e].x; t.y += red[q][e].y; }
      double2 wi = w[i];
      wi.x -= t.x;
      wi.y -= t.y;
      w[i] = wi;
      ss = wi.x * wi.x + wi.y * wi.y;
    }
    if (NORM) {
      for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
      if ((e & 31) == 0) nred[e >> 5] = ss;
    }
  }
  if (NORM) {
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < (CGS_EB + 31) / 32; q++) t += nred[q];
      npart[blockIdx.x] = t;
    }
  }
}

template <typename VT, bool NORM>
__global__ void __launch_bounds__(CGS_EB * CGS_KG)
k_cgs_small(const VT *__restrict__ V, const double2 *__restrict__ partial, int nb, int nk, int64_t n,
            double2 *__restrict__ w, double2 *__restrict__ hout, double *__restrict__ npart) {
  cgs_small_body<VT, NORM>(V, partial, nb, nk, n, w, hout, npart);
}

// Graph form: step j = *jp; the first pass writes its projections to ring
// slot j % GMRES_RING of hd (slots of `stride` entries), the second to h2.
template <typename VT, bool NORM>
__global__ void __launch_bounds__(CGS_EB * CGS_KG)
k_cgs_small_j(const VT *__restrict__ V, const double2 *__restrict__ partial, int nb, const int *__restrict__ jp,
              int64_t n, double2 *__restrict__ w, double2 *__restrict__ hd, int stride, double2 *__restrict__ h2,
              double *__restrict__ npart) {
  const int j = *jp;
  double2 *hout = NORM ? h2 : hd + (size_t)(j % GMRES_RING) * stride;
  cgs_small_body<VT, NORM>(V, partial, nb, j + 1, n, w, hout, npart);
}

// Small-n end of an Arnoldi step: every block sums the nparts partial norms
// (fixed order), block 0 completes the Hessenberg column (hj[k] += h2[k],
// hj[nk] = ||w||), and all blocks write vnext = w / ||w|| (0 if ||w|| = 0).
template <typename VT>
__device__ __forceinline__ void finish_scale_body(double2 *__restrict__ hj, const double2 *__restrict__ h2, int nk,
                                                  const double *__restrict__ npart, int nparts,
                                                  const double2 *__restrict__ w, VT *__restrict__ vnext, int64_t n) {
  __shared__ double nv;
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int b = threadIdx.x; b < nparts; b += 32) t += npart[b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) nv = sqrt(t);
  }
  __syncthreads();
  const double norm = nv;
  if (blockIdx.x == 0) {
    for (int k = threadIdx.x; k < nk; k += blockDim.x) {
      hj[k].x += h2[k].x;
      hj[k].y += h2[k].y;
    }
    if (threadIdx.x == 0) hj[nk] = make_double2(norm, 0.0);
  }
  const double sc = norm > 0.0 ? 1.0 / norm : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = w[i];
    stv(vnext + i, make_double2(v.x * sc, v.y * sc));
  }
}

template <typename VT>
__global__ void k_finish_scale(double2 *__restrict__ hj, const double2 *__restrict__ h2, int nk,
                               const double *__restrict__ npart, int nparts, const double2 *__restrict__ w,
                               VT *__restrict__ vnext, int64_t n) {
  finish_scale_body(hj, h2, nk, npart, nparts, w, vnext, n);
}

// Graph form: step j = *jp completes ring slot j % GMRES_RING of hd and writes
// V_{j+1}.
template <typename VT>
__global__ void k_finish_scale_j(double2 *__restrict__ hd, int stride, const double2 *__restrict__ h2,
                                 const int *__restrict__ jp, const double *__restrict__ npart, int nparts,
                                 const double2 *__restrict__ w, VT *__restrict__ V, int64_t n) {
  const int j = *jp;
  finish_scale_body(hd + (size_t)(j % GMRES_RING) * stride, h2, j + 1, npart, nparts, w, V + (size_t)(j + 1) * n, n);
}

// out = V_j (as complex128) for j = *jp
template <typename VT>
__global__ void k_load_vj(const VT *__restrict__ V, const int *__restrict__ jp, int64_t n, double2 *__restrict__ out) {
  const VT *vj = V + (size_t)(*jp) * n;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) out[i] = ldv(vj + i);
}

__global__ void k_step_inc(int *jp) {
  if (threadIdx.x == 0) *jp += 1;
}

// out = in * s (s real); also used to copy and convert (s = 1)
template <typename TI, typename TO>
__global__ void k_scale(const TI *__restrict__ in, TO *__restrict__ out, int64_t n, double s) {
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const double2 v = ldv(in + i);
    stv(out + i, make_double2(v.x * s, v.y * s));
  }
}

// out = w / hn->x (0 if hn->x is 0): the next basis vector, scaled by the
// norm the Arnoldi step left on the device
template <typename VT>
__global__ void k_scale_by_norm(const double2 *__restrict__ w, VT *__restrict__ out, int64_t n,
                                const double2 *__restrict__ hn) {
  const double nv = hn->x;
  const double sc = nv > 0.0 ? 1.0 / nv : 0.0;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const double2 v = w[i];
    stv(out + i, make_double2(v.x * sc, v.y * sc));
  }
}

// r = e0 - r
__global__ void k_e0_minus(double2 *__restrict__ r, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    double2 v = r[i];
    v.x = (i == 0 ? 1.0 : 0.0) - v.x;
    v.y = -v.y;
    r[i] = v;
  }
}

// ---- deflation by a proposed dominant subspace U (D x kd, orthonormal) ----
// W = { vec(u_i u_j^H) } (kd^2 orthonormal vectors); W^H x = U^H X U.
constexpr int DR = 128;  // rows per block
constexpr int DC = 32;   // columns per block
constexpr int KDMAX = 16;

// partial[b][i*kd + j] = sum over this block's rows r and columns c of conj(U[r,i]) X[r,c] U[c,j]
__global__ void k_defl_proj(const double2 *__restrict__ X, const double2 *__restrict__ U, int D, int kd,
                            double2 *__restrict__ partial) {
  __shared__ double2 Uc[DC][KDMAX];
  __shared__ double2 red[DR / 32][KDMAX * KDMAX];
  const int r = blockIdx.x * DR + threadIdx.x, c0 = blockIdx.y * DC;
  for (int q = threadIdx.x; q < DC * kd; q += DR) {
    const int cc = q / kd, j = q % kd;
    Uc[cc][j] = (c0 + cc < D) ? U[(size_t)j * D + c0 + cc] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2 T[KDMAX];
  for (int j = 0; j < KDMAX; j++) T[j] = make_double2(0.0, 0.0);
  if (r < D) {
    for (int cc = 0; cc < DC && c0 + cc < D; cc++) {
      const double2 x = X[(size_t)(c0 + cc) * D + r];
#pragma unroll
      for (int j = 0; j < KDMAX; j++) {
        if (j < kd) {
          const double2 u = Uc[cc][j];
          T[j].x = fma(x.x, u.x, fma(-x.y, u.y, T[j].x));
          T[j].y = fma(x.x, u.y, fma(x.y, u.x, T[j].y));
        }
      }
    }
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = 0; i < kd; i++) {
    double2 ui = (r < D) ? U[(size_t)i * D + r] : make_double2(0.0, 0.0);
    ui.y = -ui.y;
#pragma unroll
    for (int j = 0; j < KDMAX; j++) {
      if (j < kd) {
        double2 p = cmuls(ui, T[j]);
        for (int o = 16; o > 0; o >>= 1) {
          p.x += __shfl_down_sync(0xffffffffu, p.x, o);
          p.y += __shfl_down_sync(0xffffffffu, p.y, o);
        }
        if (lane == 0) red[w][i * kd + j] = p;
      }
    }
  }
  __syncthreads();
  const int b = blockIdx.y * gridDim.x + blockIdx.x;
  for (int q = threadIdx.x; q < kd * kd; q += DR) {
    double2 acc = make_double2(0.0, 0.0);
    for (int ww = 0; ww < DR / 32; ww++) { acc.x += red[ww][q].x; acc.y += red[ww][q].y; }
    partial[(size_t)b * kd * kd + q] = acc;
  }
}

// z = sum_b partial[b]; mode 0: zc = z; mode 1: zc = Cm z (Cm = E^-1,
// kd^2 x kd^2 row-major).  zc[i*kd + j] is the coefficient of u_i u_j^H.
__global__ void k_defl_coef(const double2 *__restrict__ partial, int nb, const double2 *__restrict__ Cm,
                            int kd, double2 *__restrict__ zc, int mode) {
  __shared__ double2 z[KDMAX * KDMAX];
  const int K2 = kd * kd;
  for (int q = threadIdx.x; q < K2; q += blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; b++) { acc.x += partial[(size_t)b * K2 + q].x; acc.y += partial[(size_t)b * K2 + q].y; }
    z[q] = acc;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < K2; q += blockDim.x) {
    if (mode == 0) {  // projections only
      zc[q] = z[q];
    } else {
      double2 acc = make_double2(0.0, 0.0);
      for (int p = 0; p < K2; p++) {
        const double2 t = cmuls(Cm[(size_t)q * K2 + p], z[p]);
        acc.x += t.x; acc.y += t.y;
      }
      zc[q] = acc;
    }
  }
}

// out[r,c] = in[r,c] + sum_{i,j} U[r,i] C[i,j] conj(U[c,j])   (in == nullptr: 0)
__global__ void k_defl_expand(const double2 *__restrict__ in, double2 *__restrict__ out,
                              const double2 *__restrict__ U, const double2 *__restrict__ cvec, int D, int kd) {
  __shared__ double2 C[KDMAX * KDMAX];
  __shared__ double2 Uc[DC][KDMAX];
  const int r = blockIdx.x * DR + threadIdx.x, c0 = blockIdx.y * DC;
  for (int q = threadIdx.x; q < kd * kd; q += DR) C[q] = cvec[q];
  for (int q = threadIdx.x; q < DC * kd; q += DR) {
    const int cc = q / kd, j = q % kd;
    double2 u = (c0 + cc < D) ? U[(size_t)j * D + c0 + cc] : make_double2(0.0, 0.0);
    u.y = -u.y;
    Uc[cc][j] = u;
  }
  __syncthreads();
  if (r >= D) return;
  double2 P[KDMAX];
#pragma unroll
  for (int j = 0; j < KDMAX; j++) {
    double2 acc = make_double2(0.0, 0.0);
    if (j < kd) {
      for (int i = 0; i < kd; i++) {
        const double2 t = cmuls(U[(size_t)i * D + r], C[i * kd + j]);
        acc.x += t.x; acc.y += t.y;
      }
    }
    P[j] = acc;
  }
  for (int cc = 0; cc < DC && c0 + cc < D; cc++) {
    const size_t e = (size_t)(c0 + cc) * D + r;
    double2 v = in ? in[e] : make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < KDMAX; j++) {
      if (j < kd) {
        const double2 t = cmuls(P[j], Uc[cc][j]);
        v.x += t.x; v.y += t.y;
      }
    }
    out[e] = v;
  }
}

// Small-n deflation with W and AW = A W stored explicitly (K2 vectors of n
// each): w <- w - AW (Ei z), z_p = sum_b partial[p][b] = (W^H w)_p from the
// multi-dot.  Every block sums z and forms c = Ei z itself (fixed order);
// each element's sum over q is split over CGS_KG groups combined in a
// fixed order.
__global__ void __launch_bounds__(CGS_EB * CGS_KG)
k_defl_apply_small(const double2 *__restrict__ AW, const double2 *__restrict__ Ei,
                   const double2 *__restrict__ partial, int nb, int K2, int64_t n, double2 *__restrict__ w) {
  __shared__ double2 z[KDMAX * KDMAX];
  __shared__ double2 c[KDMAX * KDMAX];
  __shared__ double2 red[CGS_KG][CGS_EB];
  for (int p = threadIdx.x; p < K2; p += CGS_EB * CGS_KG) {
    double2 acc = make_double2(0.0, 0.0);
    for (int b = 0; b < nb; b++) {
      const double2 v = partial[(size_t)p * nb + b];
      acc.x += v.x; acc.y += v.y;
    }
    z[p] = acc;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < K2; q += CGS_EB * CGS_KG) {
    double2 acc = make_double2(0.0, 0.0);
    for (int p = 0; p < K2; p++) {
      const double2 t = cmuls(Ei[(size_t)q * K2 + p], z[p]);
      acc.x += t.x; acc.y += t.y;
    }
    c[q] = acc;
  }
  __syncthreads();
  const int e = threadIdx.x % CGS_EB, g = threadIdx.x / CGS_EB;
  const int64_t i = (int64_t)blockIdx.x * CGS_EB + e;
  double2 acc = make_double2(0.0, 0.0);
  if (i < n) {
#pragma unroll 4
    for (int q = g; q < K2; q += CGS_KG) {
      const double2 t = cmuls(c[q], AW[(size_t)q * n + i]);
      acc.x += t.x; acc.y += t.y;
    }
  }
  red[g][e] = acc;
  __syncthreads();
  if (g == 0 && i < n) {
    double2 t = red[0][e];
    for (int q = 1; q < CGS_KG; q++) { t.x += red[q][e].x; t.y += red[q][e].y; }
    double2 wi = w[i];
    wi.x -= t.x;
    wi.y -= t.y;
    w[i] = wi;
  }
}

// W[q*n + c*D + r] = U[r,k] conj(U[c,l]) for q = k*kd + l (the stored
// deflation basis, every column in one launch)
__global__ void k_defl_formW(const double2 *__restrict__ U, int D, int kd, double2 *__restrict__ W) {
  const int64_t n = (int64_t)D * D, total = n * kd * kd;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(t / n);
    const int64_t e = t - (int64_t)q * n;
    const int c = (int)(e / D), r = (int)(e - (int64_t)c * D);
    double2 b = U[(size_t)(q % kd) * D + c];
    b.y = -b.y;
    W[t] = cmuls(U[(size_t)(q / kd) * D + r], b);
  }
}

// Y += (X Z) / 2 for X (D x D) and Z (D x k, k <= KDMAX), both column-major:
// thread = row r, block column = a segment of XSEG columns of X, segments
// summed with atomics (Y zeroed by the caller).
constexpr int XSEG = 64;
__global__ void k_x_mul(const double2 *__restrict__ X, const double2 *__restrict__ Z, int D, int k,
                        double2 *__restrict__ Y) {
  __shared__ double2 Zs[XSEG][KDMAX];
  const int r = blockIdx.x * DR + threadIdx.x, c0 = blockIdx.y * XSEG;
  for (int q = threadIdx.x; q < XSEG * k; q += DR) {
    const int cc = q / k, i = q % k;
    Zs[cc][i] = (c0 + cc < D) ? Z[(size_t)i * D + c0 + cc] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (r >= D) return;
  double2 acc[KDMAX];
#pragma unroll
  for (int i = 0; i < KDMAX; i++) acc[i] = make_double2(0.0, 0.0);
  const int cend = min(XSEG, D - c0);
  for (int cc = 0; cc < cend; cc++) {
    const double2 xv = X[(size_t)(c0 + cc) * D + r];
#pragma unroll
    for (int i = 0; i < KDMAX; i++) {
      if (i < k) {
        const double2 t = cmuls(xv, Zs[cc][i]);
        acc[i].x += t.x; acc[i].y += t.y;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < KDMAX; i++) {
    if (i < k) {
      atomicAdd(&Y[(size_t)i * D + r].x, 0.5 * acc[i].x);
      atomicAdd(&Y[(size_t)i * D + r].y, 0.5 * acc[i].y);
    }
  }
}

// Y += (X^H Z) / 2: one warp per row r of the result, reading column r of X.
__global__ void k_xh_mul(const double2 *__restrict__ X, const double2 *__restrict__ Z, int D, int k,
                         double2 *__restrict__ Y) {
  const int r = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (r >= D) return;  // uniform across the warp
  double2 acc[KDMAX];
#pragma unroll
  for (int i = 0; i < KDMAX; i++) acc[i] = make_double2(0.0, 0.0);
  for (int c = lane; c < D; c += 32) {
    double2 xv = X[(size_t)r * D + c];
    xv.y = -xv.y;
#pragma unroll
    for (int i = 0; i < KDMAX; i++) {
      if (i < k) {
        const double2 t = cmuls(xv, Z[(size_t)i * D + c]);
        acc[i].x += t.x; acc[i].y += t.y;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < KDMAX; i++) {
    if (i < k) {
      double2 v = acc[i];
      for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
      }
      if (lane == 0) {
        atomicAdd(&Y[(size_t)i * D + r].x, 0.5 * v.x);
        atomicAdd(&Y[(size_t)i * D + r].y, 0.5 * v.y);
      }
    }
  }
}

// y += a * x  (a real)
__global__ void k_axpy_inplace(double2 *__restrict__ y, const double2 *__restrict__ x, int64_t n, double a) {
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const double2 v = x[i], w = y[i];
    y[i] = make_double2(w.x + a * v.x, w.y + a * v.y);
  }
}

int grid_for(int64_t n) {
  int64_t b = (n + NT - 1) / NT;
  return (int)std::min<int64_t>(b, 148 * 8);
}

}  // namespace

// GMRES state bound to one device (buffers reused across solves).  The
// basis V holds complex128 or, in the FP32-inner solver, complex64 vectors;
// the residual t and the work vector w are always complex128.
struct Gmres {
  int m = 0, f32 = 0, mcap = 0;  // restart length and basis precision of this solve; capacity
  int64_t n = 0;
  void *V = nullptr;           // (mcap+1) x n basis vectors (sized for complex128)
  double2 *t = nullptr;        // residual / conversion buffer
  double2 *w = nullptr;
  double2 *partial = nullptr;  // (m+1) x nb
  double2 *h = nullptr;        // m+2: the least-squares solution y of a cycle
  double2 *hd = nullptr;       // RING slots of m+2: Hessenberg columns (projections, then the norm)
  double2 *h2 = nullptr;       // second-pass projections
  double *npart = nullptr;     // per-block partial norms
  double2 *hh = nullptr;       // pinned host copy of the RING slots
  cudaEvent_t ev[GMRES_RING] = {};
  // small n: one Arnoldi step as a CUDA graph (step index on the device)
  int *jdev = nullptr;
  cudaGraphExec_t gexec = nullptr;
  uint64_t gkey[6] = {};
  int64_t gkernels = 0;  // kernels per replay
  int nb = 0, chunk = CHUNK;  // multi-dot partials per projection, elements per partial
  bool small() const { return chunk == 256; }
  template <typename VT> VT *basis() const { return static_cast<VT *>(V); }
  // Buffers are kept across solves and reallocated only for a new n or a
  // longer restart, so solves that alternate settings reuse them.
  void ensure(int64_t n_, int m_, int f32_) {
    f32 = f32_;
    if (n_ == n && m_ <= mcap) {
      m = m_;
      return;
    }
    release();
    n = n_;
    m = mcap = m_;
    f32 = f32_;
    chunk = n <= (int64_t)FUSE_NB * 256 ? 256 : CHUNK;
    nb = (int)((n + chunk - 1) / chunk);
    QCUDA(cudaMalloc(&V, (size_t)(m + 1) * n * sizeof(double2)));
    QCUDA(cudaMalloc(&t, (size_t)n * sizeof(double2)));
    QCUDA(cudaMalloc(&w, (size_t)n * sizeof(double2)));
    QCUDA(cudaMalloc(&partial, (size_t)(m + 1) * nb * sizeof(double2)));
    QCUDA(cudaMalloc(&h, (size_t)(m + 2) * sizeof(double2)));
    QCUDA(cudaMalloc(&hd, (size_t)GMRES_RING * (m + 2) * sizeof(double2)));
    QCUDA(cudaMalloc(&h2, (size_t)(m + 1) * sizeof(double2)));
    QCUDA(cudaMalloc(&npart, (size_t)std::max<int64_t>(grid_for(n), (n + CGS_EB - 1) / CGS_EB) * sizeof(double)));
    QCUDA(cudaMallocHost(&hh, (size_t)GMRES_RING * (m + 2) * sizeof(double2)));
    QCUDA(cudaMalloc(&jdev, sizeof(int)));
    for (cudaEvent_t &e : ev) QCUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  void release() {
    if (V) {
      cudaFree(V); cudaFree(t); cudaFree(w); cudaFree(partial); cudaFree(h); cudaFree(hd); cudaFree(h2);
      cudaFree(npart);
      cudaFree(jdev);
      cudaFreeHost(hh);
      if (gexec) cudaGraphExecDestroy(gexec);
      for (cudaEvent_t &e : ev)
        if (e) cudaEventDestroy(e);
    }
    for (cudaEvent_t &e : ev) e = nullptr;
    V = nullptr;
    jdev = nullptr;
    gexec = nullptr;
    for (uint64_t &k : gkey) k = 0;
    t = w = partial = h = hd = h2 = hh = nullptr;
    npart = nullptr;
    n = 0;
    m = mcap = 0;
  }
};

// One solver workspace per device; the steady-state entry points hold its
// lock for the whole solve, so solves on one device run one at a time.
struct GmresSlot {
  Gmres g;
  std::mutex mu;
};


static GmresSlot &gmres_slot() {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<GmresSlot>> slots;
  int dev = 0;
  QCUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  std::unique_ptr<GmresSlot> &p = slots[dev];
  if (!p) p.reset(new GmresSlot());
  return *p;
}

static Gmres &gmres_for(qsystem) { return gmres_slot().g; }

struct SteadyPrecond;
SteadyPrecond *precond_for(qsystem qs, cudaStream_t s);
void precond_apply(SteadyPrecond &P, const double2 *x, double2 *y, cudaStream_t s);
void precond_apply_c64(SteadyPrecond &P, const float2 *x, double2 *y, cudaStream_t s);
double2 *precond_scratch(SteadyPrecond &P);

// A x with A = L + e0 vec(I)^T
static void apply_A(const DeviceProgram &PP, const double2 *x, double2 *y, cudaStream_t s) {
  Epi e;
  zero_epi(e);
  e.kout = y;
  launch_lrho_any(PP, x, e, s);
  k_trace_add<<<1, NT, 0, s>>>(x, y, PP.dev.D);
  count_launch();
}

static double norm2(const double2 *x, int64_t n, cudaStream_t s) {
  return std::sqrt(std::max(0.0, vdot(x, x, n, s).real()));
}

// Deflation by W = { vec(u_i u_j^H) } (Galerkin projection):
//   E = W^H A W,  Q = W E^-1 W^H,  P = I - A Q.
// GMRES runs on P A; the true residual of x + Q r + (I - Q A) y is
// P (r - A y), which is what the Arnoldi process minimises, so the components
// of the residual in A span W are removed exactly and restarted GMRES no
// longer stalls on the slow modes that W captures.  Unlike the right
// preconditioner I + W (E^-1 - I) W^H, the projected operator does not get
// worse conditioned than A when W is far from an invariant subspace.
struct Deflation {
  int D = 0, kd = 0, nbx = 0, nby = 0;
  double2 *U = nullptr, *Ei = nullptr, *partial = nullptr, *coef = nullptr, *t1 = nullptr, *t2 = nullptr;
  double2 *Y = nullptr, *Z = nullptr;    // D x KDMAX each (subspace refresh)
  double2 *Id = nullptr, *Ecol = nullptr;  // kd^2 x kd^2 each (assembly of E)
  // small n: W and AW stored (kd^2 x n each) and the multi-dot partials of W^H w
  double2 *W = nullptr, *AW = nullptr, *pw = nullptr;
  double2 *pe = nullptr;  // kd^4 x nbw multi-dot partials of W^H A W
  int nbw = 0;
  bool stored() const { return W != nullptr; }
  std::vector<std::complex<double>> Uh;  // host copy of U, column-major D x kd
  int cap = 0;                           // kd the buffers were sized for
  void release() {
    for (double2 *p : {U, Ei, partial, coef, t1, t2, Y, Z, Id, Ecol, W, AW, pw, pe})
      if (p) cudaFree(p);
    U = Ei = partial = coef = t1 = t2 = Y = Z = Id = Ecol = W = AW = pw = pe = nullptr;
  }
};

static void defl_project(const Deflation &F, const double2 *in, const double2 *Cm, double2 *coef, int mode,
                         cudaStream_t s) {
  dim3 g(F.nbx, F.nby);
  k_defl_proj<<<g, DR, 0, s>>>(in, F.U, F.D, F.kd, F.partial);
  k_defl_coef<<<1, 128, 0, s>>>(F.partial, F.nbx * F.nby, Cm, F.kd, coef, mode);
  count_launch(2);
}

// out = Q in   (out may not alias in)
static void apply_Q(const Deflation &F, const double2 *in, double2 *out, cudaStream_t s) {
  defl_project(F, in, F.Ei, F.coef, 1, s);
  k_defl_expand<<<dim3(F.nbx, F.nby), DR, 0, s>>>(nullptr, out, F.U, F.coef, F.D, F.kd);
  count_launch();
}

// w <- P w = w - A Q w   (uses t1, t2; small n: W^H w and AW from storage, two launches)
static void apply_P(const DeviceProgram &PP, const Deflation &F, double2 *w, int64_t n, cudaStream_t s) {
  if (F.stored()) {
    const int K2 = F.kd * F.kd;
    k_multidot<double2><<<dim3(F.nbw, (K2 + NT / 32 - 1) / (NT / 32)), NT, 0, s>>>(F.W, w, n, K2, F.pw, 256);
    k_defl_apply_small<<<(int)((n + CGS_EB - 1) / CGS_EB), CGS_EB * CGS_KG, 0, s>>>(F.AW, F.Ei, F.pw, F.nbw,
                                                                                     K2, n, w);
    count_launch(2);
    return;
  }
  apply_Q(F, w, F.t1, s);
  apply_A(PP, F.t1, F.t2, s);
  k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(w, F.t2, n, -1.0);
  count_launch();
}

// Inverse of a small dense complex matrix (row-major, Gauss-Jordan with partial pivoting).
static bool invert_small(std::vector<std::complex<double>> &A, int n) {
  std::vector<std::complex<double>> I((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) I[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::abs(A[(size_t)r * n + c]) > std::abs(A[(size_t)piv * n + c])) piv = r;
    if (std::abs(A[(size_t)piv * n + c]) < 1e-300) return false;
    if (piv != c)
      for (int k = 0; k < n; k++) {
        std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
        std::swap(I[(size_t)c * n + k], I[(size_t)piv * n + k]);
      }
    const std::complex<double> d = 1.0 / A[(size_t)c * n + c];
    for (int k = 0; k < n; k++) { A[(size_t)c * n + k] *= d; I[(size_t)c * n + k] *= d; }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const std::complex<double> f = A[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) { A[(size_t)r * n + k] -= f * A[(size_t)c * n + k]; I[(size_t)r * n + k] -= f * I[(size_t)c * n + k]; }
    }
  }
  A.swap(I);
  return true;
}

// Eigen-decomposition of a Hermitian n x n matrix (row-major; A is
// overwritten): cyclic Jacobi.  Each rotation first scales row and column q
// by a phase so that A[p][q] is real, then applies the real Jacobi rotation
// of the symmetric 2 x 2 problem (Rutishauser's form: t = sgn(th) /
// (|th| + sqrt(th^2 + 1)), th = (a_qq - a_pp) / (2 a_pq)).  Returns the
// eigenvalues in w and the eigenvectors as the columns of V (row-major).
static void herm_eig(std::vector<cplx> &A, int n, std::vector<double> &w, std::vector<cplx> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0, diag = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = 0; q < n; q++) (p == q ? diag : off) += std::norm(A[(size_t)p * n + q]);
    if (off <= 1e-30 * (diag + off)) break;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) {
        const cplx apq = A[(size_t)p * n + q];
        const double r = std::abs(apq);
        if (r <= 1e-300) continue;
        const cplx ph = apq / r, cph = std::conj(ph);
        for (int k = 0; k < n; k++) A[(size_t)k * n + q] *= cph;
        for (int k = 0; k < n; k++) A[(size_t)q * n + k] *= ph;
        for (int k = 0; k < n; k++) V[(size_t)k * n + q] *= cph;
        const double th = (A[(size_t)q * n + q].real() - A[(size_t)p * n + p].real()) / (2.0 * r);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < n; k++) {
          const cplx a = A[(size_t)k * n + p], b = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * a - sn * b;
          A[(size_t)k * n + q] = sn * a + c * b;
        }
        for (int k = 0; k < n; k++) {
          const cplx a = A[(size_t)p * n + k], b = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * a - sn * b;
          A[(size_t)q * n + k] = sn * a + c * b;
        }
        for (int k = 0; k < n; k++) {
          const cplx a = V[(size_t)k * n + p], b = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = c * a - sn * b;
          V[(size_t)k * n + q] = sn * a + c * b;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; i++) w[i] = A[(size_t)i * n + i].real();
}

// Sizes the buffers for rank kd; a workspace already sized for this D and
// at least this rank is reused as it is.
static bool alloc_deflation(const DeviceProgram &PP, int kd, Deflation &F) {
  const int D = PP.dev.D;
  const int64_t n = (int64_t)D * D;
  if (F.U && F.D == D && F.cap >= kd) {
    F.kd = kd;
    return true;
  }
  F.release();
  F.D = D;
  F.kd = F.cap = kd;
  F.nbx = (D + DR - 1) / DR;
  F.nby = (D + DC - 1) / DC;
  const int K2 = kd * kd;
  QCUDA(cudaMalloc(&F.U, (size_t)D * kd * sizeof(double2)));
  QCUDA(cudaMalloc(&F.Ei, (size_t)K2 * K2 * sizeof(double2)));
  QCUDA(cudaMalloc(&F.partial, (size_t)F.nbx * F.nby * K2 * sizeof(double2)));
  QCUDA(cudaMalloc(&F.coef, (size_t)K2 * sizeof(double2)));
  QCUDA(cudaMalloc(&F.t1, n * sizeof(double2)));
  QCUDA(cudaMalloc(&F.t2, n * sizeof(double2)));
  QCUDA(cudaMalloc(&F.Y, (size_t)D * KDMAX * sizeof(double2)));
  QCUDA(cudaMalloc(&F.Z, (size_t)D * KDMAX * sizeof(double2)));
  QCUDA(cudaMalloc(&F.Id, (size_t)K2 * K2 * sizeof(double2)));
  QCUDA(cudaMalloc(&F.Ecol, (size_t)K2 * K2 * sizeof(double2)));
  if (n <= (int64_t)FUSE_NB * 256) {
    F.nbw = (int)((n + 255) / 256);
    QCUDA(cudaMalloc(&F.W, (size_t)K2 * n * sizeof(double2)));
    QCUDA(cudaMalloc(&F.AW, (size_t)K2 * n * sizeof(double2)));
    QCUDA(cudaMalloc(&F.pw, (size_t)K2 * F.nbw * sizeof(double2)));
    QCUDA(cudaMalloc(&F.pe, (size_t)K2 * K2 * F.nbw * sizeof(double2)));
  }
  return !has_error();
}

// E = W^H A W for the U on the device and Ei = E^-1.  E[:, q] for
// q = k*kd + l is W^H A vec(u_k u_l^H); every column is queued on the
// stream (unit coefficients from an identity block), one copy back.
// Returns false, leaving Ei as it was, if E is singular.
static bool assemble_E(const DeviceProgram &PP, Deflation &F, cudaStream_t s) {
  const int kd = F.kd, K2 = kd * kd;
  std::vector<double2> hId((size_t)K2 * K2, make_double2(0.0, 0.0)), hE((size_t)K2 * K2);
  for (int q = 0; q < K2; q++) hId[(size_t)q * K2 + q] = make_double2(1.0, 0.0);
  QCUDA(cudaMemcpyAsync(F.Id, hId.data(), hId.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  const int64_t n = (int64_t)F.D * F.D;
  // stored basis on a generic program: W in one launch, A W batched, and
  // E = W^H A W as one batched multi-dot
  bool batched = false;
  if (F.stored() && !PP.has_qubit) {
    k_defl_formW<<<grid_for(n * K2), NT, 0, s>>>(F.U, F.D, kd, F.W);
    count_launch();
    if (launch_lrho_batch(PP, F.W, F.AW, K2, s)) {
      k_trace_add<<<dim3(1, 1, K2), NT, 0, s>>>(F.W, F.AW, F.D);
      k_multidot<double2><<<dim3(F.nbw, (K2 + NT / 32 - 1) / (NT / 32), K2), NT, 0, s>>>(F.W, F.AW, n, K2, F.pe,
                                                                                         256);
      k_reduce_rows<<<K2 * K2, NT, 0, s>>>(F.pe, F.nbw, F.Ecol, 0);
      count_launch(3);
      batched = true;
    }
  }
  if (!batched) {
    for (int q = 0; q < K2; q++) {  // small n: W_q and A W_q are kept
      double2 *wq = F.stored() ? F.W + (size_t)q * n : F.t1;
      double2 *awq = F.stored() ? F.AW + (size_t)q * n : F.t2;
      k_defl_expand<<<dim3(F.nbx, F.nby), DR, 0, s>>>(nullptr, wq, F.U, F.Id + (size_t)q * K2, F.D, kd);
      count_launch();
      apply_A(PP, wq, awq, s);
      defl_project(F, awq, nullptr, F.Ecol + (size_t)q * K2, 0, s);
    }
  }
  QCUDA(cudaMemcpyAsync(hE.data(), F.Ecol, hE.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  std::vector<cplx> E((size_t)K2 * K2);
  for (int q = 0; q < K2; q++)
    for (int p = 0; p < K2; p++) E[(size_t)p * K2 + q] = cplx(hE[(size_t)q * K2 + p].x, hE[(size_t)q * K2 + p].y);
  if (has_error() || !invert_small(E, K2)) return false;
  std::vector<double2> Ei((size_t)K2 * K2);
  for (size_t p = 0; p < Ei.size(); p++) Ei[p] = make_double2(E[p].real(), E[p].imag());
  QCUDA(cudaMemcpyAsync(F.Ei, Ei.data(), Ei.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  QCUDA(cudaStreamSynchronize(s));
  return !has_error();
}

static void upload_U(Deflation &F, cudaStream_t s) {
  std::vector<double2> h(F.Uh.size());
  for (size_t i = 0; i < h.size(); i++) h[i] = make_double2(F.Uh[i].real(), F.Uh[i].imag());
  QCUDA(cudaMemcpyAsync(F.U, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  QCUDA(cudaStreamSynchronize(s));
}

// Builds the deflation from host U (D x kd, column-major, orthonormal columns).
static bool build_deflation(const DeviceProgram &PP, const cplx *U_host, int kd, Deflation &F, cudaStream_t s) {
  if (!alloc_deflation(PP, kd, F)) return false;
  F.Uh.assign(U_host, U_host + (size_t)PP.dev.D * kd);
  upload_U(F, s);
  return assemble_E(PP, F, s);
}

// Y = Xh Z on the device for Xh = (X + X^H) / 2, Z (D x k) host, Y returned on the host.
static std::vector<cplx> herm_part_times(const double2 *x, Deflation &F, const std::vector<cplx> &Zh, int k,
                                         cudaStream_t s) {
  const int D = F.D;
  std::vector<double2> h((size_t)D * k);
  for (size_t i = 0; i < h.size(); i++) h[i] = make_double2(Zh[i].real(), Zh[i].imag());
  QCUDA(cudaMemcpyAsync(F.Z, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  QCUDA(cudaMemsetAsync(F.Y, 0, (size_t)D * k * sizeof(double2), s));
  k_x_mul<<<dim3((D + DR - 1) / DR, (D + XSEG - 1) / XSEG), DR, 0, s>>>(x, F.Z, D, k, F.Y);
  k_xh_mul<<<(int)(((int64_t)D * 32 + NT - 1) / NT), NT, 0, s>>>(x, F.Z, D, k, F.Y);
  count_launch(2);
  QCUDA(cudaMemcpyAsync(h.data(), F.Y, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  std::vector<cplx> Y(h.size());
  for (size_t i = 0; i < h.size(); i++) Y[i] = cplx(h[i].x, h[i].y);
  return Y;
}

// One Rayleigh-Ritz step toward the kd leading eigenvectors of the
// Hermitian part Xh of the current iterate: the search space is span{U, Xh U}
// (Xh U orthogonalised against U, directions below 1e-12 of the largest
// dropped), the new U the kd Ritz vectors of Xh with the largest Ritz
// values.  Warm-started from the previous U, one step per restart tracks
// the iterate's dominant subspace as it converges.  E is then reassembled;
// if that fails, the previous U and E are kept.
static bool refresh_deflation(const DeviceProgram &PP, const double2 *x, Deflation &F, cudaStream_t s) {
  const int D = F.D, kd = F.kd;
  const std::vector<cplx> U = F.Uh;
  auto col = [D](const std::vector<cplx> &M, int j) { return M.data() + (size_t)j * D; };
  std::vector<cplx> Y = herm_part_times(x, F, U, kd, s);
  if (has_error()) return false;
  // Y <- Y - U (U^H Y)
  for (int j = 0; j < kd; j++) {
    cplx *y = Y.data() + (size_t)j * D;
    for (int i = 0; i < kd; i++) {
      const cplx *u = col(U, i);
      cplx d = 0.0;
      for (int r = 0; r < D; r++) d += std::conj(u[r]) * y[r];
      for (int r = 0; r < D; r++) y[r] -= d * u[r];
    }
  }
  // orthonormal basis of span Y from the eigenvectors of its Gram matrix
  std::vector<cplx> G((size_t)kd * kd), Vg;
  std::vector<double> g;
  for (int i = 0; i < kd; i++)
    for (int j = 0; j < kd; j++) {
      cplx d = 0.0;
      for (int r = 0; r < D; r++) d += std::conj(Y[(size_t)i * D + r]) * Y[(size_t)j * D + r];
      G[(size_t)i * kd + j] = d;
    }
  herm_eig(G, kd, g, Vg);
  double gmax = 0.0;
  for (double v : g) gmax = std::max(gmax, v);
  std::vector<cplx> Yo;
  int k2 = 0;
  for (int j = 0; j < kd; j++) {
    if (!(g[j] > 1e-24 * gmax) || gmax <= 0.0) continue;
    const double sc = 1.0 / std::sqrt(g[j]);
    Yo.resize((size_t)(k2 + 1) * D, 0.0);
    for (int i = 0; i < kd; i++) {
      const cplx c = Vg[(size_t)i * kd + j] * sc;
      for (int r = 0; r < D; r++) Yo[(size_t)k2 * D + r] += c * Y[(size_t)i * D + r];
    }
    k2++;
  }
  // Ritz problem on Z = [U, Yo]: T = Z^H Xh Z with Xh U = Y + U (U^H Xh U)
  // recomputed from scratch for accuracy
  const int nz = kd + k2;
  std::vector<cplx> Z((size_t)nz * D);
  std::copy(U.begin(), U.end(), Z.begin());
  std::copy(Yo.begin(), Yo.end(), Z.begin() + (size_t)kd * D);
  std::vector<cplx> XZ = herm_part_times(x, F, std::vector<cplx>(Z.begin(), Z.begin() + (size_t)kd * D), kd, s);
  if (k2 > 0) {
    std::vector<cplx> XY = herm_part_times(x, F, Yo, k2, s);
    XZ.insert(XZ.end(), XY.begin(), XY.end());
  }
  if (has_error()) return false;
  std::vector<cplx> T((size_t)nz * nz), Vt;
  for (int i = 0; i < nz; i++)
    for (int j = 0; j < nz; j++) {
      cplx d = 0.0;
      for (int r = 0; r < D; r++) d += std::conj(Z[(size_t)i * D + r]) * XZ[(size_t)j * D + r];
      T[(size_t)i * nz + j] = d;
    }
  for (int i = 0; i < nz; i++)
    for (int j = i; j < nz; j++) {
      const cplx a = 0.5 * (T[(size_t)i * nz + j] + std::conj(T[(size_t)j * nz + i]));
      T[(size_t)i * nz + j] = a;
      T[(size_t)j * nz + i] = std::conj(a);
    }
  std::vector<double> w;
  herm_eig(T, nz, w, Vt);
  std::vector<int> order(nz);
  for (int i = 0; i < nz; i++) order[i] = i;
  std::sort(order.begin(), order.end(), [&w](int a, int b) { return w[a] > w[b]; });
  std::vector<cplx> Un((size_t)kd * D, 0.0);
  for (int j = 0; j < kd; j++) {
    cplx *u = Un.data() + (size_t)j * D;
    for (int i = 0; i < nz; i++) {
      const cplx c = Vt[(size_t)i * nz + order[j]];
      for (int r = 0; r < D; r++) u[r] += c * Z[(size_t)i * D + r];
    }
    // re-orthonormalise against the columns before it (modified Gram-Schmidt)
    for (int i = 0; i < j; i++) {
      const cplx *v = Un.data() + (size_t)i * D;
      cplx d = 0.0;
      for (int r = 0; r < D; r++) d += std::conj(v[r]) * u[r];
      for (int r = 0; r < D; r++) u[r] -= d * v[r];
    }
    double nn = 0.0;
    for (int r = 0; r < D; r++) nn += std::norm(u[r]);
    if (!(nn > 0.0)) return false;
    const double sc = 1.0 / std::sqrt(nn);
    for (int r = 0; r < D; r++) u[r] *= sc;
  }
  F.Uh = Un;
  upload_U(F, s);
  if (!assemble_E(PP, F, s)) {  // keep the previous subspace (and its stored W, AW, E^-1)
    F.Uh = U;
    upload_U(F, s);
    assemble_E(PP, F, s);
    return false;
  }
  return !has_error();
}

// Restarted GMRES with the basis stored as VT.  Every restart forms the
// true residual b - A x in complex128, so with a complex64 basis (FP32
// inner) the restarts are the iterative refinement that takes the solution
// to the complex128 tolerance.
// Captures one small-n Arnoldi step (the step index j lives in G.jdev and
// every kernel reads it): V_j into t, w = A t (then P w with deflation),
// the two Gram-Schmidt passes, the Hessenberg column into its ring slot and
// V_{j+1}; the whole ring of columns is copied to the pinned host ring and
// j is incremented.  The executable graph is kept for the next step, cycle
// and solve with the same program, deflation buffers, basis type and
// restart length.  Returns false (the caller launches the kernels itself)
// if capture or instantiation fails.
template <typename VT>
static bool step_graph(Gmres &G, const DeviceProgram &PP, Deflation *def, int m, cudaStream_t s) {
  const uint64_t key[6] = {PP.serial, (uint64_t)(uintptr_t)(def ? def->W : nullptr), (uint64_t)(def ? def->kd : 0),
                           (uint64_t)sizeof(VT), (uint64_t)m, (uint64_t)(uintptr_t)G.V};
  if (G.gexec && std::equal(key, key + 6, G.gkey)) return true;
  if (G.gexec) {
    cudaGraphExecDestroy(G.gexec);
    G.gexec = nullptr;
  }
  const int64_t n = G.n;
  VT *V = G.basis<VT>();
  const int nbl = (int)((n + CGS_EB - 1) / CGS_EB);
  const dim3 gd(G.nb, (m + NT / 32 - 1) / (NT / 32));
  const int64_t c0 = quac_kernel_launch_count();
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  k_load_vj<<<grid_for(n), NT, 0, s>>>(V, G.jdev, n, G.t);
  apply_A(PP, G.t, G.w, s);
  if (def) apply_P(PP, *def, G.w, n, s);
  k_multidot_j<<<gd, NT, 0, s>>>(V, G.w, n, G.jdev, G.partial, G.chunk);
  k_cgs_small_j<VT, false><<<nbl, CGS_EB * CGS_KG, 0, s>>>(V, G.partial, G.nb, G.jdev, n, G.w, G.hd, m + 2,
                                                             G.h2, nullptr);
  k_multidot_j<<<gd, NT, 0, s>>>(V, G.w, n, G.jdev, G.partial, G.chunk);
  k_cgs_small_j<VT, true><<<nbl, CGS_EB * CGS_KG, 0, s>>>(V, G.partial, G.nb, G.jdev, n, G.w, G.hd, m + 2,
                                                            G.h2, G.npart);
  k_finish_scale_j<<<grid_for(n), NT, 0, s>>>(G.hd, m + 2, G.h2, G.jdev, G.npart, nbl, G.w, V, n);
  cudaMemcpyAsync(G.hh, G.hd, (size_t)GMRES_RING * (m + 2) * sizeof(double2), cudaMemcpyDeviceToHost, s);
  k_step_inc<<<1, 32, 0, s>>>(G.jdev);
  count_launch(7);
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s, &graph);
  const int64_t kernels = quac_kernel_launch_count() - c0;
  count_launch((int)-kernels);  // nothing ran yet; each replay counts them
  if (ec != cudaSuccess || !graph) {
    cudaGetLastError();
    return false;
  }
  const cudaError_t ei = cudaGraphInstantiate(&G.gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    G.gexec = nullptr;
    return false;
  }
  std::copy(key, key + 6, G.gkey);
  G.gkernels = kernels;
  return true;
}

// With a complex64 basis the residual after a restart carries an error of
// about eps32 * ||H|| * ||y||, which on ill-conditioned systems (||y|| >>
// ||r||) can exceed what a cycle gains; *stalled is set (and the run
// returns) when the true residual has not fallen below 0.9x its value
// STALL_CYCLES restarts earlier, and the caller continues in complex128.
constexpr int STALL_CYCLES = 20;

// With pre (right preconditioning, no deflation): the Arnoldi process runs
// on A M^-1 and each cycle ends with x += M^-1 V y, so the residual it
// minimises is still the true residual b - A x.
template <typename VT>
static int64_t gmres_run(const DeviceProgram &PP, Gmres &G, double2 *x, double rtol, int m, int64_t maxit,
                         double *final_res, Deflation *def, bool refresh, cudaStream_t s,
                         bool *stalled = nullptr, SteadyPrecond *pre = nullptr) {
  const int64_t n = G.n;
  VT *V = G.basis<VT>();
  std::vector<std::complex<double>> H((size_t)(m + 1) * m), cs(m), sn(m), gvec(m + 1), y(m);
  int64_t it = 0;
  double res = 0;
  std::vector<double> hist;  // true residual at the start of every cycle
  for (int cycle = 0;; cycle++) {
    if (has_error()) break;
    if (def && refresh && cycle > 0) refresh_deflation(PP, x, *def, s);
    // r = b - A x
    apply_A(PP, x, G.t, s);
    k_e0_minus<<<grid_for(n), NT, 0, s>>>(G.t, n);
    count_launch();
    double beta = norm2(G.t, n, s);
    res = beta;
    if (beta <= rtol || it >= maxit) break;
    hist.push_back(beta);
    if (stalled && hist.size() > (size_t)STALL_CYCLES && !(beta < 0.9 * hist[hist.size() - 1 - STALL_CYCLES])) {
      *stalled = true;
      break;
    }
    if (def) {  // x += Q r, and the cycle starts from P r = r - A Q r
      apply_Q(*def, G.t, def->t1, s);
      k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(x, def->t1, n, 1.0);
      apply_A(PP, def->t1, def->t2, s);
      k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(G.t, def->t2, n, -1.0);
      count_launch(2);
      beta = norm2(G.t, n, s);
      if (!(beta > rtol)) { it++; continue; }  // re-check the true residual
    }
    k_scale<<<grid_for(n), NT, 0, s>>>(G.t, V, n, 1.0 / beta);
    count_launch();
    std::fill(gvec.begin(), gvec.end(), 0.0);
    gvec[0] = beta;
    // Arnoldi steps run ahead of the host by up to GMRES_LAG: step j needs
    // only V_j, which step j-1 scaled on the device, so the host queues
    // the next steps before it reads column j back and applies the Givens
    // rotations.  Steps queued past convergence are discarded.
    const bool graph = G.small() && !pre && step_graph<VT>(G, PP, def, m, s);
    if (graph) QCUDA(cudaMemsetAsync(G.jdev, 0, sizeof(int), s));
    auto launch_step = [&](int j) {
      if (graph) {  // the step index advances on the device
        QCUDA(cudaGraphLaunch(G.gexec, s));
        count_launch((int)G.gkernels);
        QCUDA(cudaEventRecord(G.ev[j % GMRES_RING], s));
        return;
      }
      const VT *vj = V + (size_t)j * n;
      const double2 *src;
      if constexpr (std::is_same<VT, double2>::value) {
        src = reinterpret_cast<const double2 *>(vj);
        if (pre) {  // w = A M^-1 v_j
          precond_apply(*pre, src, precond_scratch(*pre), s);
          src = precond_scratch(*pre);
        }
      } else if (pre) {  // complex64 basis: M^-1 applied in complex64
        precond_apply_c64(*pre, reinterpret_cast<const float2 *>(vj), precond_scratch(*pre), s);
        src = precond_scratch(*pre);
      } else {
        k_scale<<<grid_for(n), NT, 0, s>>>(vj, G.t, n, 1.0);
        count_launch();
        src = G.t;
      }
      apply_A(PP, src, G.w, s);
      if (def) apply_P(PP, *def, G.w, n, s);  // Arnoldi on P A
      // CGS2 on the device; the Hessenberg column (projections of both
      // passes summed, then ||w||) goes to ring slot j % GMRES_RING
      double2 *hj = G.hd + (size_t)(j % GMRES_RING) * (m + 2);
      const dim3 gd(G.nb, (j + 1 + NT / 32 - 1) / (NT / 32));
      if (G.small()) {  // few partials: 5 launches, reductions inside the CGS passes
        const int nbl = (int)((n + CGS_EB - 1) / CGS_EB);
        k_multidot<<<gd, NT, 0, s>>>(V, G.w, n, j + 1, G.partial, G.chunk);
        k_cgs_small<VT, false><<<nbl, CGS_EB * CGS_KG, 0, s>>>(V, G.partial, G.nb, j + 1, n, G.w, hj, nullptr);
        k_multidot<<<gd, NT, 0, s>>>(V, G.w, n, j + 1, G.partial, G.chunk);
        k_cgs_small<VT, true><<<nbl, CGS_EB * CGS_KG, 0, s>>>(V, G.partial, G.nb, j + 1, n, G.w, G.h2, G.npart);
        k_finish_scale<<<grid_for(n), NT, 0, s>>>(hj, G.h2, j + 1, G.npart, nbl, G.w, V + (size_t)(j + 1) * n, n);
        count_launch(5);
      } else {
        k_multidot<<<gd, NT, 0, s>>>(V, G.w, n, j + 1, G.partial, G.chunk);
        k_reduce_rows<<<j + 1, NT, 0, s>>>(G.partial, G.nb, hj, 0);
        k_multiaxpy<<<grid_for(n), NT, 0, s>>>(V, hj, n, j + 1, G.w, -1.0);
        k_multidot<<<gd, NT, 0, s>>>(V, G.w, n, j + 1, G.partial, G.chunk);
        k_reduce_rows<<<j + 1, NT, 0, s>>>(G.partial, G.nb, G.h2, 0);
        k_multiaxpy_norm<<<grid_for(n), NT, 0, s>>>(V, G.h2, n, j + 1, G.w, G.npart);
        k_arnoldi_finish<<<1, NT, 0, s>>>(hj, G.h2, j + 1, G.npart, grid_for(n));
        k_scale_by_norm<<<grid_for(n), NT, 0, s>>>(G.w, V + (size_t)(j + 1) * n, n, hj + j + 1);
        count_launch(8);
      }
      QCUDA(cudaMemcpyAsync(G.hh + (size_t)(j % GMRES_RING) * (m + 2), hj, (j + 2) * sizeof(double2),
                            cudaMemcpyDeviceToHost, s));
      QCUDA(cudaEventRecord(G.ev[j % GMRES_RING], s));
    };
    int jl = 0, j = 0;  // steps launched, steps processed
    while (true) {
      while (jl < m && jl - j <= GMRES_LAG && it + (jl - j) < maxit) launch_step(jl++);
      if (j >= jl || has_error()) break;
      QCUDA(cudaEventSynchronize(G.ev[j % GMRES_RING]));
      const double2 *hc = G.hh + (size_t)(j % GMRES_RING) * (m + 2);
      const double hn = hc[j + 1].x;
      for (int k = 0; k <= j; k++) H[(size_t)k * m + j] = std::complex<double>(hc[k].x, hc[k].y);
      H[(size_t)(j + 1) * m + j] = hn;
      for (int k = 0; k < j; k++) {
        auto a = H[(size_t)k * m + j], b = H[(size_t)(k + 1) * m + j];
        H[(size_t)k * m + j] = std::conj(cs[k]) * a + std::conj(sn[k]) * b;
        H[(size_t)(k + 1) * m + j] = -sn[k] * a + cs[k] * b;
      }
      auto a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
      const double r = std::sqrt(std::norm(a) + std::norm(b));
      if (r == 0) { cs[j] = 1; sn[j] = 0; }
      else { cs[j] = a / r; sn[j] = b / r; }
      H[(size_t)j * m + j] = r;
      H[(size_t)(j + 1) * m + j] = 0;
      gvec[j + 1] = -sn[j] * gvec[j];
      gvec[j] = std::conj(cs[j]) * gvec[j];
      j++;
      it++;
      if (std::abs(gvec[j]) <= rtol || hn == 0) break;
    }
    // solve the triangular system and update x += V y
    for (int k = j - 1; k >= 0; k--) {
      auto sum = gvec[k];
      for (int q = k + 1; q < j; q++) sum -= H[(size_t)k * m + q] * y[q];
      y[k] = sum / H[(size_t)k * m + k];
    }
    if (j > 0) {
      std::vector<double2> yh(j);
      for (int k = 0; k < j; k++) yh[k] = make_double2(y[k].real(), y[k].imag());
      QCUDA(cudaMemcpyAsync(G.h, yh.data(), j * sizeof(double2), cudaMemcpyHostToDevice, s));
      if (def) {  // x += (I - Q A) V y
        QCUDA(cudaMemsetAsync(G.w, 0, n * sizeof(double2), s));
        k_multiaxpy<<<grid_for(n), NT, 0, s>>>(V, G.h, n, j, G.w, 1.0);
        k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(x, G.w, n, 1.0);
        count_launch(2);
        apply_A(PP, G.w, def->t2, s);
        apply_Q(*def, def->t2, def->t1, s);
        k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(x, def->t1, n, -1.0);
        count_launch();
      } else if (pre) {  // x += M^-1 V y
        QCUDA(cudaMemsetAsync(G.w, 0, n * sizeof(double2), s));
        k_multiaxpy<<<grid_for(n), NT, 0, s>>>(V, G.h, n, j, G.w, 1.0);
        count_launch();
        precond_apply(*pre, G.w, precond_scratch(*pre), s);
        k_axpy_inplace<<<grid_for(n), NT, 0, s>>>(x, precond_scratch(*pre), n, 1.0);
        count_launch();
      } else {
        k_multiaxpy<<<grid_for(n), NT, 0, s>>>(V, G.h, n, j, x, 1.0);
        count_launch();
      }
      QCUDA(cudaStreamSynchronize(s));
    }
  }
  QCUDA(cudaStreamSynchronize(s));
  if (final_res) *final_res = res;
  return it;
}

// Returns iterations, fills x (device, length n).  rtol is relative to ||b|| = 1.
// The basis precision follows quac_set_gmres_precision.
int64_t gmres_solve(qsystem qs, double2 *x, double rtol, int m, int64_t maxit, bool x_is_guess,
                    double *final_res, Deflation *def = nullptr, bool refresh = false) {
  ensure_program(qs);
  const DeviceProgram &PP = *qs->impl->prog;
  const DevProg &P = PP.dev;
  const int64_t n = (int64_t)P.D * P.ncols;
  cudaStream_t s = stream_of(qs);
  if (m < 1 || m > GMRES_MAXM) { fail(9, "ERROR! GMRES restart must be in [1, %d]\n", GMRES_MAXM); return -1; }
  Gmres &G = gmres_for(qs);
  const int f32 = options().gmres_f32;
  G.ensure(n, m, f32);
  if (has_error()) return -1;
  if (!x_is_guess) {
    QCUDA(cudaMemsetAsync(x, 0, n * sizeof(double2), s));
    const double2 one = make_double2(1.0, 0.0);
    QCUDA(cudaMemcpyAsync(x, &one, sizeof(double2), cudaMemcpyHostToDevice, s));
  }
  // the no-jump preconditioner (quac_set_gmres_preconditioner) in runs
  // without a deflation space
  SteadyPrecond *pre = nullptr;
  if (options().gmres_precond && !def) {
    pre = precond_for(qs, s);
    if (!pre) return -1;
  }
  if (!f32) return gmres_run<double2>(PP, G, x, rtol, m, maxit, final_res, def, refresh, s, nullptr, pre);
  bool stalled = false;
  int64_t its = gmres_run<float2>(PP, G, x, rtol, m, maxit, final_res, def, refresh, s, &stalled, pre);
  if (!stalled || its < 0) return its;
  const int64_t more = gmres_run<double2>(PP, G, x, rtol, m, maxit - its, final_res, def, refresh, s, nullptr, pre);
  return more < 0 ? -1 : its + more;
}

}  // namespace quac

using namespace quac;

extern "C" PetscInt steady_state_sys(qsystem qs, qvec x) {
  if (!qs->dm_equations) { fail(0, "ERROR! steady_state_sys needs Lindblad terms\n"); return -1; }
  if (!qs->impl->td.empty()) { fail(0, "ERROR! a steady state needs a time-independent system\n"); return -1; }
  if (!qs->mat_allocated) construct_matrix(qs);
  if (has_error()) return -1;
  vec_sync_to_device(x->data);
  std::lock_guard<std::mutex> lk(gmres_slot().mu);
  double res = 0;
  const int64_t its = gmres_solve(qs, x->data->d, options().gmres_rtol, options().gmres_restart, 200000, false, &res);
  return has_error() ? -1 : its;
}

// Deflation workspace of one device, kept across guided solves (used under
// the lock of the device's GMRES workspace).
static Deflation &deflation_slot() {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<Deflation>> slots;
  int dev = 0;
  QCUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  std::unique_ptr<Deflation> &p = slots[dev];
  if (!p) p.reset(new Deflation());
  return *p;
}

// Steady state from a proposed initial state (x on entry) and a proposed
// dominant subspace U (D x kd, orthonormal columns, column-major host array;
// kd = 0: no deflation).  Deflated GMRES runs for at most maxit_guided
// iterations; if it has not converged, plain GMRES(100) continues from its
// iterate.  Returns the total number of iterations (-1 on error).
extern "C" PetscInt quac_steady_state_guided(qsystem qs, qvec x, const PetscScalar *U_host, PetscInt kd,
                                             PetscInt maxit_guided, PetscReal *residual) {
  if (!qs->dm_equations) { fail(0, "ERROR! steady state needs Lindblad terms\n"); return -1; }
  if (!qs->impl->td.empty()) { fail(0, "ERROR! a steady state needs a time-independent system\n"); return -1; }
  if (kd < 0 || kd > KDMAX) { fail(0, "ERROR! deflation rank must be in [0, %d]\n", KDMAX); return -1; }
  if (!qs->mat_allocated) construct_matrix(qs);
  if (has_error()) return -1;
  vec_sync_to_device(x->data);
  ensure_program(qs);
  const DeviceProgram &PP = *qs->impl->prog;
  cudaStream_t s = stream_of(qs);
  std::lock_guard<std::mutex> lk(gmres_slot().mu);
  Deflation &F = deflation_slot();
  const bool use = kd > 0;
  if (use && !build_deflation(PP, reinterpret_cast<const std::complex<double> *>(U_host), (int)kd, F, s)) {
    if (!has_error()) fail(0, "ERROR! W^H A W is singular for the proposed deflation space\n");
    return -1;
  }
  // start from whichever of the proposal and e0 has the smaller residual
  {
    Gmres &G = gmres_for(qs);
    const int64_t n = (int64_t)PP.dev.D * PP.dev.D;
    G.ensure(n, options().gmres_restart, options().gmres_f32);
    apply_A(PP, x->data->d, G.w, s);
    k_e0_minus<<<grid_for(n), NT, 0, s>>>(G.w, n);
    count_launch();
    const double r_guess = norm2(G.w, n, s);
    QCUDA(cudaMemsetAsync(G.t, 0, n * sizeof(double2), s));
    const double2 one = make_double2(1.0, 0.0);
    QCUDA(cudaMemcpyAsync(G.t, &one, sizeof(double2), cudaMemcpyHostToDevice, s));
    apply_A(PP, G.t, G.w, s);
    k_e0_minus<<<grid_for(n), NT, 0, s>>>(G.w, n);
    count_launch();
    const double r_e0 = norm2(G.w, n, s);
    if (!(r_guess <= r_e0)) QCUDA(cudaMemcpyAsync(x->data->d, G.t, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  }
  double res = 0;
  const int m = options().gmres_restart;
  const double rtol = options().gmres_rtol;
  int64_t its = gmres_solve(qs, x->data->d, rtol, m, maxit_guided, true, &res, use ? &F : nullptr,
                            options().defl_refresh != 0);
  if (its < 0) return -1;
  if (res > rtol) {
    const int64_t more = gmres_solve(qs, x->data->d, rtol, m, 200000, true, &res);
    if (more < 0) return -1;
    its += more;
  }
  if (residual) *residual = res;
  return has_error() ? -1 : its;
}
