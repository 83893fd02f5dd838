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
// decomposition is computed on the GPU (cuSOLVER geev and an LU inverse of
// V) once per system and cached by program serial number; at D = 512 it
// takes about 0.14 s, most of a preconditioned solve.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "runtime.h"

namespace quac {

bool compile_host(qsystem qs, int mode, HostProg &hp);

// V, V^-1 and the eigenvalues of one H_eff (device memory)
struct Decomp {
  int D = 0;
  int kind = 1;  // 1: eigen-decomposition of H_eff; 2: of its Hermitian part
  int device = 0;
  double shift = 0.0;
  double2 *V = nullptr, *Vi = nullptr, *lam = nullptr;
  float2 *V32 = nullptr, *Vi32 = nullptr;  // complex64 copies for the complex64-basis GMRES
  ~Decomp() {
    for (double2 *p : {V, Vi, lam})
      if (p) cudaFree(p);
    for (float2 *p : {V32, Vi32})
      if (p) cudaFree(p);
  }
};

// per-device library handles and the scratch of precond_apply
struct DeviceCtx {
  cusolverDnHandle_t sol = nullptr;
  cusolverDnParams_t par = nullptr;
  cublasHandle_t blas = nullptr;
  double2 *T = nullptr, *Z = nullptr;
  float2 *T32 = nullptr, *U32 = nullptr;
  size_t cap = 0;  // elements of T and Z (and of T32, U32)
};

struct SteadyPrecond {
  uint64_t serial = 0;
  std::shared_ptr<Decomp> dec;
  DeviceCtx *ctx = nullptr;
};

namespace {

constexpr int PT = 256;

// y[k D + j] /= -i (lam_j - conj(lam_k)) - shift
__global__ void k_sylvester_scale(double2 *__restrict__ y, const double2 *__restrict__ lam, int D, double shift) {
  const int64_t n = (int64_t)D * D;
  for (int64_t i = (int64_t)blockIdx.x * PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT) {
    const int k = (int)(i / D), j = (int)(i - (int64_t)k * D);
    const double2 a = lam[j], b = lam[k];
    // -i (a - conj(b)) = (a.y + b.y) - i (a.x - b.x)
    const double dr = a.y + b.y - shift, di = b.x - a.x;
    const double inv = 1.0 / (dr * dr + di * di);
    const double2 v = y[i];
    y[i] = make_double2((v.x * dr + v.y * di) * inv, (v.y * dr - v.x * di) * inv);
  }
}

// lam[k] = w[k] - i/2 Re(sum_i conj(U[i, k]) T[i, k]), T = G U (column-major)
__global__ void k_herm_eigs(const double2 *__restrict__ U, const double2 *__restrict__ T, const double *__restrict__ w,
                            double2 *__restrict__ lam, int D) {
  const int k = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < D; i += PT) {
    const double2 u = U[(size_t)k * D + i], t = T[(size_t)k * D + i];
    s += u.x * t.x + u.y * t.y;
  }
  __shared__ double red[PT];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = PT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) lam[k] = make_double2(w[k], -0.5 * red[0]);
}

__global__ void k_to_c64(const double2 *__restrict__ x, float2 *__restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT)
    y[i] = make_float2((float)x[i].x, (float)x[i].y);
}

__global__ void k_to_c128(const float2 *__restrict__ x, double2 *__restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT)
    y[i] = make_double2((double)x[i].x, (double)x[i].y);
}

// complex64 form of k_sylvester_scale (divisor in double)
__global__ void k_sylvester_scale32(float2 *__restrict__ y, const double2 *__restrict__ lam, int D, double shift) {
  const int64_t n = (int64_t)D * D;
  for (int64_t i = (int64_t)blockIdx.x * PT + threadIdx.x; i < n; i += (int64_t)gridDim.x * PT) {
    const int k = (int)(i / D), j = (int)(i - (int64_t)k * D);
    const double2 a = lam[j], b = lam[k];
    const double dr = a.y + b.y - shift, di = b.x - a.x;
    const double inv = 1.0 / (dr * dr + di * di);
    const float2 v = y[i];
    y[i] = make_float2((float)((v.x * dr + v.y * di) * inv), (float)((v.y * dr - v.x * di) * inv));
  }
}

int grid_of(int64_t n) { return (int)std::min<int64_t>((n + PT - 1) / PT, 148 * 8); }

// complex64 copies of V and V^-1
bool add_c64_copies(Decomp &P, cudaStream_t s) {
  const int64_t n2 = (int64_t)P.D * P.D;
  QCUDA(cudaMalloc(&P.V32, n2 * sizeof(float2)));
  QCUDA(cudaMalloc(&P.Vi32, n2 * sizeof(float2)));
  if (has_error()) return false;
  k_to_c64<<<grid_of(n2), PT, 0, s>>>(P.V, P.V32, n2);
  k_to_c64<<<grid_of(n2), PT, 0, s>>>(P.Vi, P.Vi32, n2);
  count_launch(2);
  QCUDA(cudaStreamSynchronize(s));
  return !has_error();
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
std::map<int, DeviceCtx> g_ctx;
int64_t g_builds = 0;
double g_build_seconds = 0.0;

DeviceCtx *device_ctx() {
  int dev = 0;
  QCUDA(cudaGetDevice(&dev));
  DeviceCtx &C = g_ctx[dev];
  if (!C.sol) {
    if (!solver_ok(cusolverDnCreate(&C.sol), "cusolverDnCreate")) { C.sol = nullptr; return nullptr; }
    if (!solver_ok(cusolverDnCreateParams(&C.par), "cusolverDnCreateParams")) return nullptr;
  }
  if (!C.blas && !blas_ok(cublasCreate(&C.blas), "cublasCreate")) { C.blas = nullptr; return nullptr; }
  return &C;
}

bool ensure_scratch(DeviceCtx &C, size_t n2) {
  if (C.cap >= n2) return true;
  for (double2 *p : {C.T, C.Z})
    if (p) cudaFree(p);
  for (float2 *p : {C.T32, C.U32})
    if (p) cudaFree(p);
  C.T = C.Z = nullptr;
  C.T32 = C.U32 = nullptr;
  C.cap = 0;
  QCUDA(cudaMalloc(&C.T, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&C.Z, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&C.T32, n2 * sizeof(float2)));
  QCUDA(cudaMalloc(&C.U32, n2 * sizeof(float2)));
  if (has_error()) return false;
  C.cap = n2;
  return true;
}

// Mode 2: H_eff = H - i/2 G with H, G Hermitian; H = U diag(w) U^H by the
// Hermitian eigensolver, and the eigenvalues of H_eff approximated by
// w_k - i/2 (U^H G U)_kk.  V = U is unitary (V^-1 = U^H), so the setup needs
// no LU; the preconditioner is exact when G commutes with H and otherwise a
// fixed approximation of L0^-1, which GMRES tolerates (it still minimises
// the true residual).
std::shared_ptr<Decomp> decompose_hermitian(int D, const std::vector<std::complex<double>> &Heff, DeviceCtx &C,
                                            cudaStream_t s) {
  const size_t n2 = (size_t)D * D;
  std::vector<std::complex<double>> H(n2), G(n2);
  const std::complex<double> I(0.0, 1.0);
  for (int c = 0; c < D; c++)
    for (int r = 0; r < D; r++) {
      const std::complex<double> a = Heff[(size_t)c * D + r], b = std::conj(Heff[(size_t)r * D + c]);
      H[(size_t)c * D + r] = 0.5 * (a + b);
      G[(size_t)c * D + r] = I * (a - b);
    }
  auto P = std::make_shared<Decomp>();
  P->D = D;
  P->kind = 2;
  QCUDA(cudaGetDevice(&P->device));
  double2 *Gd = nullptr, *T = nullptr;
  double *w = nullptr;
  int *info = nullptr;
  void *dwork = nullptr;
  QCUDA(cudaMalloc(&P->V, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P->Vi, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P->lam, D * sizeof(double2)));
  QCUDA(cudaMalloc(&Gd, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&T, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&w, D * sizeof(double)));
  QCUDA(cudaMalloc(&info, sizeof(int)));
  bool ok = !has_error();
  if (ok) {
    QCUDA(cudaMemcpyAsync(P->V, H.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
    QCUDA(cudaMemcpyAsync(Gd, G.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
  }
  ok = ok && !has_error() && solver_ok(cusolverDnSetStream(C.sol, s), "cusolverDnSetStream");
  size_t dsz = 0, hsz = 0;
  ok = ok && solver_ok(cusolverDnXsyevd_bufferSize(C.sol, C.par, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D,
                                                   CUDA_C_64F, P->V, D, CUDA_R_64F, w, CUDA_C_64F, &dsz, &hsz),
                       "syevd buffer size");
  std::vector<char> hwork(hsz + 1);
  if (ok) QCUDA(cudaMalloc(&dwork, dsz + 16));
  ok = ok && !has_error() &&
       solver_ok(cusolverDnXsyevd(C.sol, C.par, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, D, CUDA_C_64F, P->V,
                                  D, CUDA_R_64F, w, CUDA_C_64F, dwork, dsz, hwork.data(), hsz, info),
                 "syevd");
  int hinfo = 0;
  if (ok) {
    QCUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    QCUDA(cudaStreamSynchronize(s));
    if (hinfo != 0) { fail(9, "ERROR! eigen-decomposition of the Hermitian part of H_eff failed (info %d)\n", hinfo); ok = false; }
  }
  if (ok && !C.blas) ok = blas_ok(cublasCreate(&C.blas), "cublasCreate");
  if (ok) {
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    auto *cU = reinterpret_cast<cuDoubleComplex *>(P->V);
    ok = blas_ok(cublasSetStream(C.blas, s), "cublasSetStream") &&
         blas_ok(cublasZgemm(C.blas, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one,
                             reinterpret_cast<const cuDoubleComplex *>(Gd), D, cU, D, &zero,
                             reinterpret_cast<cuDoubleComplex *>(T), D),
                 "zgemm") &&
         blas_ok(cublasZgeam(C.blas, CUBLAS_OP_C, CUBLAS_OP_N, D, D, &one, cU, D, &zero, cU, D,
                             reinterpret_cast<cuDoubleComplex *>(P->Vi), D),
                 "zgeam");
  }
  if (ok) {
    k_herm_eigs<<<D, PT, 0, s>>>(P->V, T, w, P->lam, D);
    count_launch();
    QCUDA(cudaGetLastError());
    std::vector<std::complex<double>> lam(D);
    QCUDA(cudaMemcpyAsync(lam.data(), P->lam, D * sizeof(double2), cudaMemcpyDeviceToHost, s));
    QCUDA(cudaStreamSynchronize(s));
    double scale = 0.0;
    for (auto &l : lam) scale = std::max(scale, std::abs(l));
    P->shift = 1e-8 * std::max(scale, 1e-300);
  }
  for (void *p : {(void *)Gd, (void *)T, (void *)w, (void *)info, dwork})
    if (p) cudaFree(p);
  if (!ok || has_error()) return nullptr;
  return P;
}

// eigen-decomposition of H_eff of qs (caller holds g_mu); nullptr on failure
std::shared_ptr<Decomp> decompose(qsystem qs, DeviceCtx &C, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
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
  if (options().gmres_precond == 2) {
    if (!ensure_scratch(C, n2)) return nullptr;
    auto Q = decompose_hermitian(D, H, C, s);
    if (!Q || !add_c64_copies(*Q, s)) return nullptr;
    g_builds++;
    g_build_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return Q;
  }
  auto P = std::make_shared<Decomp>();
  P->D = D;
  QCUDA(cudaGetDevice(&P->device));
  double2 *A = nullptr;
  int64_t *ipiv = nullptr;
  int *info = nullptr;
  void *dwork = nullptr;
  QCUDA(cudaMalloc(&P->V, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P->Vi, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&P->lam, D * sizeof(double2)));
  QCUDA(cudaMalloc(&A, n2 * sizeof(double2)));
  QCUDA(cudaMalloc(&ipiv, D * sizeof(int64_t)));
  QCUDA(cudaMalloc(&info, sizeof(int)));
  bool ok = !has_error() && ensure_scratch(C, n2);
  if (ok) QCUDA(cudaMemcpyAsync(A, H.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
  ok = ok && solver_ok(cusolverDnSetStream(C.sol, s), "cusolverDnSetStream");
  size_t dsz = 0, hsz = 0, dsz2 = 0, hsz2 = 0;
  if (ok)
    ok = solver_ok(cusolverDnXgeev_bufferSize(C.sol, C.par, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, D,
                                              CUDA_C_64F, A, D, CUDA_C_64F, P->lam, CUDA_C_64F, nullptr, D,
                                              CUDA_C_64F, P->V, D, CUDA_C_64F, &dsz, &hsz),
                   "geev buffer size") &&
         solver_ok(cusolverDnXgetrf_bufferSize(C.sol, C.par, D, D, CUDA_C_64F, P->Vi, D, CUDA_C_64F, &dsz2, &hsz2),
                   "getrf buffer size");
  std::vector<char> hwork(std::max(hsz, hsz2) + 1);
  if (ok) QCUDA(cudaMalloc(&dwork, std::max(dsz, dsz2) + 16));
  int hinfo = 0;
  if (ok && !has_error())
    ok = solver_ok(cusolverDnXgeev(C.sol, C.par, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, D, CUDA_C_64F,
                                   A, D, CUDA_C_64F, P->lam, CUDA_C_64F, nullptr, D, CUDA_C_64F, P->V, D, CUDA_C_64F,
                                   dwork, dsz, hwork.data(), hsz, info),
                   "geev");
  if (ok) {
    QCUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
    QCUDA(cudaStreamSynchronize(s));
    if (hinfo != 0) { fail(9, "ERROR! eigen-decomposition of H_eff failed (info %d)\n", hinfo); ok = false; }
  }
  // V^-1: LU of V (in A), then solve with the identity on the right (in Vi)
  if (ok) {
    std::vector<std::complex<double>> Id(n2, 0.0);
    for (int k = 0; k < D; k++) Id[(size_t)k * D + k] = 1.0;
    QCUDA(cudaMemcpyAsync(A, P->V, n2 * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    QCUDA(cudaMemcpyAsync(P->Vi, Id.data(), n2 * sizeof(double2), cudaMemcpyHostToDevice, s));
    ok = solver_ok(cusolverDnXgetrf(C.sol, C.par, D, D, CUDA_C_64F, A, D, ipiv, CUDA_C_64F, dwork, dsz2,
                                    hwork.data(), hsz2, info),
                   "getrf") &&
         solver_ok(cusolverDnXgetrs(C.sol, C.par, CUBLAS_OP_N, D, D, CUDA_C_64F, A, D, ipiv, CUDA_C_64F, P->Vi, D,
                                    info),
                   "getrs");
    if (ok) {
      QCUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, s));
      QCUDA(cudaStreamSynchronize(s));  // also keeps Id alive until the copy is done
      if (hinfo != 0) { fail(9, "ERROR! eigenvector matrix of H_eff is singular (info %d)\n", hinfo); ok = false; }
    }
  }
  if (ok) {
    std::vector<std::complex<double>> lam(D);
    QCUDA(cudaMemcpy(lam.data(), P->lam, D * sizeof(double2), cudaMemcpyDeviceToHost));
    double scale = 0.0;
    for (auto &l : lam) scale = std::max(scale, std::abs(l));
    P->shift = 1e-8 * std::max(scale, 1e-300);  // modes without decay
  }
  for (void *p : {(void *)A, (void *)ipiv, (void *)info, dwork})
    if (p) cudaFree(p);
  if (!ok || has_error() || !add_c64_copies(*P, s)) return nullptr;
  g_builds++;
  g_build_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return P;
}

// the entry of qs, its decomposition valid for the current program
SteadyPrecond *entry_for(qsystem qs, cudaStream_t s) {
  ensure_program(qs);
  if (has_error() || !qs->impl->prog) return nullptr;
  DeviceCtx *C = device_ctx();
  if (!C) return nullptr;
  SteadyPrecond &P = g_pre[qs];
  P.ctx = C;
  const uint64_t serial = qs->impl->prog->serial;
  if (P.serial == serial && P.dec && P.dec->kind == options().gmres_precond)
    return ensure_scratch(*C, (size_t)P.dec->D * P.dec->D) ? &P : nullptr;
  P.dec.reset();
  P.serial = 0;
  auto d = decompose(qs, *C, s);
  if (!d) return nullptr;
  P.dec = d;
  P.serial = serial;
  return &P;
}

}  // namespace

// The preconditioner of qs (decomposed on first use)
SteadyPrecond *precond_for(qsystem qs, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  return entry_for(qs, s);
}

// y = L0^-1 x (vec of D x D, column stacking); x and y distinct
void precond_apply(SteadyPrecond &P, const double2 *x, double2 *y, cudaStream_t s) {
  const Decomp &M = *P.dec;
  const int D = M.D;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  auto *cx = reinterpret_cast<const cuDoubleComplex *>(x);
  auto *cy = reinterpret_cast<cuDoubleComplex *>(y);
  auto *cT = reinterpret_cast<cuDoubleComplex *>(P.ctx->T);
  auto *cV = reinterpret_cast<const cuDoubleComplex *>(M.V);
  auto *cVi = reinterpret_cast<const cuDoubleComplex *>(M.Vi);
  cublasHandle_t h = P.ctx->blas;
  blas_ok(cublasSetStream(h, s), "cublasSetStream");
  // T = V^-1 X ;  Y = T V^-H ;  Y ./= den ;  T = V Y ;  Y = T V^H
  blas_ok(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cVi, D, cx, D, &zero, cT, D), "zgemm");
  blas_ok(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cVi, D, &zero, cy, D), "zgemm");
  const int64_t n2 = (int64_t)D * D;
  k_sylvester_scale<<<(int)std::min<int64_t>((n2 + PT - 1) / PT, 148 * 8), PT, 0, s>>>(y, M.lam, D, M.shift);
  count_launch();
  blas_ok(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cV, D, cy, D, &zero, cT, D), "zgemm");
  blas_ok(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cV, D, &zero, cy, D), "zgemm");
}

// y = L0^-1 x with x a complex64 vector and the four GEMMs in complex64
// (the complex64-basis GMRES: its Arnoldi vectors are complex64 already,
// and GMRES only needs the preconditioner to be a fixed map)
void precond_apply_c64(SteadyPrecond &P, const float2 *x, double2 *y, cudaStream_t s) {
  const Decomp &M = *P.dec;
  const int D = M.D;
  const cuComplex one = make_cuComplex(1.0f, 0.0f), zero = make_cuComplex(0.0f, 0.0f);
  auto *cx = reinterpret_cast<const cuComplex *>(x);
  auto *cT = reinterpret_cast<cuComplex *>(P.ctx->T32);
  auto *cU = reinterpret_cast<cuComplex *>(P.ctx->U32);
  auto *cV = reinterpret_cast<const cuComplex *>(M.V32);
  auto *cVi = reinterpret_cast<const cuComplex *>(M.Vi32);
  cublasHandle_t h = P.ctx->blas;
  blas_ok(cublasSetStream(h, s), "cublasSetStream");
  blas_ok(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cVi, D, cx, D, &zero, cT, D), "cgemm");
  blas_ok(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cVi, D, &zero, cU, D), "cgemm");
  const int64_t n2 = (int64_t)D * D;
  k_sylvester_scale32<<<grid_of(n2), PT, 0, s>>>(P.ctx->U32, M.lam, D, M.shift);
  blas_ok(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, D, D, D, &one, cV, D, cU, D, &zero, cT, D), "cgemm");
  blas_ok(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, D, D, D, &one, cT, D, cV, D, &zero, cU, D), "cgemm");
  k_to_c128<<<grid_of(n2), PT, 0, s>>>(P.ctx->U32, y, n2);
  count_launch(2);
}

double2 *precond_scratch(SteadyPrecond &P) { return P.ctx->Z; }

void precond_release_system(qsystem qs) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_pre.erase(qs);
}

}  // namespace quac

using namespace quac;

// Builds the steady-state preconditioner of qs now (the first
// preconditioned solve would otherwise do it), like PCSetUp.
extern "C" int quac_steady_precond_setup(qsystem qs) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!qs->mat_allocated) construct_matrix(qs);
  if (has_error()) return 1;
  return entry_for(qs, stream_of(qs)) ? 0 : 1;
}

// Decompositions computed in this process and their total host wall time.
extern "C" void quac_steady_precond_stats(int64_t *builds, double *seconds) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (builds) *builds = g_builds;
  if (seconds) *seconds = g_build_seconds;
}
