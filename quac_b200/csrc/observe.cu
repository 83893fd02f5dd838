// Observables as single-pass device reductions: Tr(O rho), trace, <psi|rho|psi>,
// vector dot products.  The reference gathers them element by element with
// one MPI_Allreduce per element (qvec_utilities.c:322-392, 1197-1283,
// 2271-2337); here each is one kernel plus an 16-byte read-back.
#include <mutex>

#include "runtime.h"

namespace quac {

namespace {

constexpr int NT = 256;
constexpr int MAXB = 1024;

__device__ __forceinline__ double2 cmulr(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__device__ void block_reduce_store(double2 v, double2 *out) {
  __shared__ double2 red[NT / 32];
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = make_double2(0.0, 0.0);
    for (int w = 0; w < NT / 32; w++) { s.x += red[w].x; s.y += red[w].y; }
    out[blockIdx.x] = s;
  }
}

// sum_c val[c] * rho[map[c], c]   (map[c] < 0: no contribution)
__global__ void k_dm_expect(const double2 *__restrict__ rho, int64_t D,
                            const int *__restrict__ map, const double2 *__restrict__ val,
                            double2 *partial) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t c = (int64_t)blockIdx.x * NT + threadIdx.x; c < D; c += (int64_t)gridDim.x * NT) {
    const int j = map[c];
    if (j >= 0) {
      const double2 v = cmulr(val[c], rho[c * D + j]);
      acc.x += v.x; acc.y += v.y;
    }
  }
  block_reduce_store(acc, partial);
}

// sum_r conj(psi[r]) * val[r] * psi[map[r]]
__global__ void k_wf_expect(const double2 *__restrict__ psi, int64_t D,
                            const int *__restrict__ map, const double2 *__restrict__ val,
                            double2 *partial) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t r = (int64_t)blockIdx.x * NT + threadIdx.x; r < D; r += (int64_t)gridDim.x * NT) {
    const int j = map[r];
    if (j >= 0) {
      double2 p = psi[r];
      p.y = -p.y;
      const double2 v = cmulr(p, cmulr(val[r], psi[j]));
      acc.x += v.x; acc.y += v.y;
    }
  }
  block_reduce_store(acc, partial);
}

__global__ void k_trace(const double2 *__restrict__ rho, int64_t D, double2 *partial) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < D; i += (int64_t)gridDim.x * NT) {
    const double2 v = rho[i * (D + 1)];
    acc.x += v.x; acc.y += v.y;
  }
  block_reduce_store(acc, partial);
}

// sum_{r,c} conj(psi[r]) rho[c*D + r] psi[c]
__global__ void k_dm_wf(const double2 *__restrict__ rho, const double2 *__restrict__ psi,
                        int64_t D, double2 *partial) {
  double2 acc = make_double2(0.0, 0.0);
  const int64_t n = D * D;
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    const int64_t c = i / D, r = i - c * D;
    double2 pr = psi[r];
    pr.y = -pr.y;
    const double2 v = cmulr(cmulr(pr, rho[i]), psi[c]);
    acc.x += v.x; acc.y += v.y;
  }
  block_reduce_store(acc, partial);
}

// sum conj(a) b
__global__ void k_vdot(const double2 *__restrict__ a, const double2 *__restrict__ b, int64_t n,
                       double2 *partial) {
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t i = (int64_t)blockIdx.x * NT + threadIdx.x; i < n; i += (int64_t)gridDim.x * NT) {
    double2 x = a[i];
    x.y = -x.y;
    const double2 v = cmulr(x, b[i]);
    acc.x += v.x; acc.y += v.y;
  }
  block_reduce_store(acc, partial);
}

__global__ void k_final(const double2 *partial, int nb, double2 *out) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nb; i += NT) { acc.x += partial[i].x; acc.y += partial[i].y; }
  block_reduce_store(acc, out);
}

struct Scratch {
  double2 *partial = nullptr;
  double2 *result = nullptr;
  double2 *host = nullptr;
};

Scratch &scratch() {
  static std::mutex mu;
  static Scratch per_dev[64];
  int dev = 0;
  QCUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  Scratch &S = per_dev[dev & 63];
  if (!S.partial) {
    QCUDA(cudaMalloc(&S.partial, MAXB * sizeof(double2)));
    QCUDA(cudaMalloc(&S.result, sizeof(double2)));
    QCUDA(cudaMallocHost(&S.host, sizeof(double2)));
  }
  return S;
}

int nblocks(int64_t n) {
  int64_t b = (n + NT - 1) / NT;
  if (b > MAXB) b = MAXB;
  if (b < 1) b = 1;
  return (int)b;
}

cplx finish(Scratch &S, int nb, cudaStream_t s) {
  k_final<<<1, NT, 0, s>>>(S.partial, nb, S.result);
  count_launch(2);
  QCUDA(cudaGetLastError());
  QCUDA(cudaMemcpyAsync(S.host, S.result, sizeof(double2), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  return cplx(S.host->x, S.host->y);
}

}  // namespace

cplx dm_expectation(const double2 *rho, int64_t D, const int *map, const double2 *val,
                    cudaStream_t s) {
  Scratch &S = scratch();
  const int nb = nblocks(D);
  k_dm_expect<<<nb, NT, 0, s>>>(rho, D, map, val, S.partial);
  return finish(S, nb, s);
}

cplx wf_expectation(const double2 *psi, int64_t D, const int *map, const double2 *val,
                    cudaStream_t s) {
  Scratch &S = scratch();
  const int nb = nblocks(D);
  k_wf_expect<<<nb, NT, 0, s>>>(psi, D, map, val, S.partial);
  return finish(S, nb, s);
}

cplx dm_trace(const double2 *rho, int64_t D, cudaStream_t s) {
  Scratch &S = scratch();
  const int nb = nblocks(D);
  k_trace<<<nb, NT, 0, s>>>(rho, D, S.partial);
  return finish(S, nb, s);
}

double dm_wf_fidelity(const double2 *rho, const double2 *psi, int64_t D, cudaStream_t s) {
  Scratch &S = scratch();
  const int nb = nblocks(D * D);
  k_dm_wf<<<nb, NT, 0, s>>>(rho, psi, D, S.partial);
  return finish(S, nb, s).real();
}

cplx vdot(const double2 *a, const double2 *b, int64_t n, cudaStream_t s) {
  Scratch &S = scratch();
  const int nb = nblocks(n);
  k_vdot<<<nb, NT, 0, s>>>(a, b, n, S.partial);
  return finish(S, nb, s);
}

}  // namespace quac
