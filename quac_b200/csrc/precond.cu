// Right preconditioner of the steady-state GMRES: the exact inverse of the
// no-jump part of the Liouvillian.
//
// The reference preconditions its GMRES with PCASM / ILU(0) on the
// assembled matrix (solver.c:167-198).  Here nothing is assembled; instead
// the Liouvillian is split as L = L0 + J with
//   L0 X = -i (H_eff X - X H_eff^H),   H_eff = H - i/2 sum_k a_k C_k^dag C_k,
//   J  X = sum_k a_k C_k X C_k^dag          (the jumps),
// and L0 is inverted exactly through the eigen-decomposition
// H_eff = V diag(lam) V^-1 (a Sylvester equation in the eigenbasis):
//   L0^-1 Y = V [ (V^-1 Y V^-H) ./ (-i (lam_j - conj(lam_k))) ] V^H.
// Every eigenvalue of a dissipative H_eff has Im(lam) < 0, so the divisor
// never vanishes; modes without decay get a small shift.  One application
// is four D x D complex GEMMs (cuBLAS) and an element-wise scaling.  The
// decomposition is computed once per system on the GPU (cuSOLVER geev and
// an LU inverse of V) and cached by program serial number.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "runtime.h"

namespace quac {

bool compile_host(qsystem qs, int mode, HostProg &hp);

struct SteadyPrecond {
  uint64_t serial = 0;
  int D = 0;
  double2 *V = nullptr, *Vi = nullptr, *den = nullptr, *T = nullptr, *Z = nullptr;
  cublasHandle_t blas = nullptr;
  void release() {
    for (double2 *p : {V, Vi, den, T, Z})
      if (p) cudaFree(p);
    V = Vi = den = T = Z = nullptr;
    serial = 0;
  }
};

namespace {

constexpr int PT = 256;

__global__ void k_hadamard(double2 *__restrict__ y, const double2 *__restrict__ den, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT) {
    const double2 a = y[i], b = den[i];
    y[i] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
}

bool blas_ok(cublasStatus_t st, const char *what) {
  if (st == CUBLAS_STATUS_SUCCESS) return true;
  fail(9, "ERROR! %s failed (cuBLAS status %d)\n", what, (int)st);
  return false;
}

bool solver_ok(cusolverStatus_t st, const char *what) {
  if (st == CUSOLVER_STATUS_SUCCESS) return true;
  fail(9, "ERROR! %s failed (cuSOLVER status %d)\n", what, (int)st);
  return false;
}

std::mutex g_mu;
std::map<qsystem, SteadyPrecond> g_pre;

}  // namespace

// Decomposes H_eff of qs (cached); nullptr on failure.
SteadyPrecond *precond_for(qsystem qs, cudaStream_t s) {
  ensure_program(qs);
  if (has_error() || !qs->impl->prog) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  SteadyPrecond &P = g_pre[qs];
  const uint64_t serial = qs->impl->prog->serial;
  if (P.serial == serial && P.V) return &P;
  P.release();
  HostProg hp;
  if (!compile_host(qs, 2, hp)) return nullptr;  // -i H_eff in Schroedinger form
  const int D = hp.D;
  const size_t n2 = (size_t)D * D;
  // dense H_eff, column-major: H_eff = i (-i H_eff)
  std::vector<std::complex<double>> H(n2, 0.0);
  const std::complex<double> I(0.0, 1.0);
  for (int r = 0; r < D; r++) H[(size_t)r * D + r] += I * hp.dr[r];
  for (size_t t = 0; t < hp.Lmap.size(); t++)
    for (int r = 0; r < D; r++) {
      const int c = hp.Lmap[t][r];
      if (c >= 0) H[(size_t)c * D + r] += I * hp.Lval[t][r];
    }
  double2 *A = nullptr, *W = nullptr;
  int64_t *ipiv = nullptr;
  int *info = nullptr;
  void *dwork = nullptr;
  QCUDA(cudaMalloc(&P.V, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P.Vi, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P.den, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P.T, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P.Z, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&A, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&W, D * sizeof(double2)));
  QCUDA(cudaMalloc(&ipiv, D * sizeof(int64_t)));
  QCUDA(cudaMalloc(&info, sizeof(int)));
  QCUDA(cudaMemcpyAsync(A, H.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
  cusolverDnHandle_t sol = nullptr;
  cusolverDnParams_t par = nullptr;
  bool ok = solver_ok(cusolverDnCreate(&sol), "cusolverDnCreate") && solver_ok(cusolverDnSetStream(sol, s), "stream") &&
            solver_ok(cusolverDnCreateParams(&par), "params");
  size_t dsz = 0, hsz = 0, dsz2 = 0, hsz2 = 0;
  if (ok)
    ok = solver_ok(cusolverDnXgeev_bufferSize(sol, par, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, D,
                                              CUDA_C_64F, A, D, CUDA_C_64F, W, CUDA_C_64F, nullptr, D, CUDA_C_64F,
                                              P.V, D, CUDA_C_64F, &dsz, &hsz),
                   "geev buffer size") &&
         solver_ok(cusolverDnXgetrf_bufferSize(sol, par, D, D, CUDA_C_64F, P.Vi, D, CUDA_C_64F, &dsz2, &hsz2),
                   "getrf buffer size");
  std::vector<char> hwork(std::max(hsz, hsz2) + 1);
  if (ok) QCUDA(cudaMalloc(&dwork, std::max(dsz, dsz2) + 16));
  int hinfo = 0;
  if (ok && !has_error())
    ok = solver_ok(cusolverDnXgeev(sol, par, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, D, CUDA_C_64F, A,
                                   D, CUDA_C_64F, W, CUDA_C_64F, nullptr, D, CUDA_C_64F, P.V, D, CUDA_C_64F, dwork,
                                   dsz, hwork.data(), hsz, info),
                   "geev");
  if (ok) {
    QCUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    QCUDA(cudaStreamSynchronize(s));
    if (hinfo != 0) { fail(9, "ERROR! eigen-decomposition of H_eff failed (info %d)\n", hinfo); ok = false; }
  }
  // V^-1: LU of V (in Vi), then solve with the identity on the right
  std::vector<std::complex<double>> Id(n2, 0.0);
  for (int k = 0; k < D; k++) Id[(size_t)k * D + k] = 1.0;
  if (ok) {
    QCUDA(cudaMemcpyAsync(P.Vi, P.V, n2 * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    QCUDA(cudaMemcpyAsync(P.T, Id.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
    ok = solver_ok(cusolverDnXgetrf(sol, par, D, D, CUDA_C_64F, P.Vi, D, ipiv, CUDA_C_64F, dwork, dsz2, hwork.data(),
                                    hsz2, info),
                   "getrf") &&
         solver_ok(cusolverDnXgetrs(sol, par, CUBLAS_OP_N, D, D, CUDA_C_64F, P.Vi, D, ipiv, CUDA_C_64F, P.T, D, info),
                   "getrs");
  }
  if (ok) {
    QCUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    QCUDA(cudaStreamSynchronize(s));
    if (hinfo != 0) { fail(9, "ERROR! eigenvector matrix of H_eff is singular (info %d)\n", hinfo); ok = false; }
    std::swap(P.Vi, P.T);  // Vi = V^-1
  }
  if (ok) {
    std::vector<std::complex<double>> lam(D), den(n2);
    QCUDA(cudaMemcpy(lam.data(), W, D * sizeof(double2), cudaMemcpyDeviceToHost));
    double scale = 0.0;
    for (auto &l : lam) scale = std::max(scale, std::abs(l));
    const double shift = 1e-8 * std::max(scale, 1e-300);  // modes without decay
    for (int k = 0; k < D; k++)
      for (int j = 0; j < D; j++) den[(size_t)k * D + j] = 1.0 / (-I * (lam[j] - std::conj(lam[k])) - shift);
    QCUDA(cudaMemcpy(P.den, den.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice));
  }
  for (void *p : {(void *)A, (void *)W, (void *)ipiv, (void *)info, dwork})
    if (p) cudaFree(p);
  if (par) cusolverDnDestroyParams(par);
  if (sol) cusolverDnDestroy(sol);
  if (ok && !P.blas) ok = blas_ok(cublasCreate(&P.blas), "cublasCreate");
  if (!ok || has_error()) {
    P.release();
    return nullptr;
  }
  P.D = D;
  P.serial = serial;
  return &P;
}

// y = L0^-1 x (vec of D x D, column stacking); x and y distinct
void precond_apply(SteadyPrecond &P, const double2 *x, double2 *y, cudaStream_t s) {
  const int D = P.D;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  auto *cx = reinterpret_cast<const cuDoubleComplex *>(x);
  auto *cy = reinterpret_cast<cuDoubleComplex *>(y);
  auto *cT = reinterpret_cast<cuDoubleComplex *>(P.T);
  auto *cV = reinterpret_cast<const cuDoubleComplex *>(P.V);
  auto *cVi = reinterpret_cast<const cuDoubleComplex *>(P.Vi);
  blas_ok(cublasSetStream(P.blas, s), "cublasSetStream");
  // T = V^-1 X ;  Y = T V^-H ;  Y ./= den ;  T = V Y ;  Y = T V^H
  blas_ok(cublasZgemm(P.blas, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cVi, D, cx, D, &zero, cT, D), "zgemm");
  blas_ok(cublasZgemm(P.blas, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cVi, D, &zero, cy, D), "zgemm");
  const int64_t n2 = (int64_t)D * D;
  k_hadamard<<<(int)std::min<int64_t>((n2 + PT - 1) / PT, 148 * 8), PT, 0, s>>>(y, P.den, n2);
  count_launch();
  blas_ok(cublasZgemm(P.blas, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cV, D, cy, D, &zero, cT, D), "zgemm");
  blas_ok(cublasZgemm(P.blas, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cV, D, &zero, cy, D), "zgemm");
}

double2 *precond_scratch(SteadyPrecond &P) { return P.Z; }

void precond_release_system(qsystem qs) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_pre.find(qs);
  if (it == g_pre.end()) return;
  it->second.release();
  if (it->second.blas) cublasDestroy(it->second.blas);
  g_pre.erase(it);
}

}  // namespace quac
