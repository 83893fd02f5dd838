// Matrix-free Liouvillian action y = L x with fused Runge-Kutta stage
// updates.  Replaces the assembled MPIAIJ superoperator of construct_matrix
// (qsystem.c:593-676) and the PETSc MatMult inside every TSRK stage
// (qsystem.c:937, 954).
//
// One CTA owns a TR x TC tile of the column-stacked matrix x (element (r,c)
// at c*D + r), staged in shared memory.  A thread owns one row r of the
// tile and K of its columns, so the per-row tables of a term (partner row,
// coefficient) are read once and reused for K elements, while the
// per-column tables are warp-uniform broadcasts.  Partners that fall inside
// the tile come from shared memory, the others from global memory (L2).
#include <map>
#include <mutex>
#include "common.h"

namespace quac {

namespace {

constexpr int NT = 256;

__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ double cabs2(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

// Batched form (gridDim.z > 1, epilogue writing kout only): slice z reads
// X + z*D*ncols and writes kout + z*D*ncols.
template <int K>
__global__ void __launch_bounds__(NT) k_lrho(const DevProg P, const double2 *__restrict__ X,
                                             Epi E, const int TR, const int CG) {
  extern __shared__ double2 tile[];
  __shared__ double red[NT / 32];
  const int D = P.D, NC = P.ncols;
  if (blockIdx.z) {
    const size_t zoff = (size_t)blockIdx.z * D * NC;
    X += zoff;
    E.kout += zoff;
  }
  const int TC = CG * K;
  const int R0 = blockIdx.x * TR;
  const int C0 = blockIdx.y * TC;
  for (int idx = threadIdx.x; idx < TR * TC; idx += NT) {
    const int cc = idx / TR, rr = idx - cc * TR;
    const int r = R0 + rr, c = C0 + cc;
    tile[idx] = (r < D && c < NC) ? __ldg(X + (size_t)c * D + r) : make_double2(0.0, 0.0);
  }
  __syncthreads();

  const int rr = threadIdx.x % TR;
  const int g = threadIdx.x / TR;
  const int r = R0 + rr;
  const bool row_ok = (g < CG) && (r < D);
  double nloc = 0.0;

  if (row_ok) {
    int cidx[K];
    bool cok[K];
    double2 acc[K], xs[K];
    const double2 drr = __ldg(P.dr + r);
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int c = C0 + g + k * CG;
      cidx[k] = c;
      cok[k] = c < NC;
      xs[k] = cok[k] ? tile[(c - C0) * TR + rr] : make_double2(0.0, 0.0);
      const double2 d = cok[k] ? cadd(drr, __ldg(P.dc + (NC == 1 ? 0 : c))) : drr;
      acc[k] = NC == 1 ? cmul(drr, xs[k]) : cmul(d, xs[k]);
    }
    // diagonal jumps: a v(r) conj(v(c)) x[r,c]
    for (int t = 0; t < P.nJd; t++) {
      const double2 f = __ldg(P.Jdrow + (size_t)t * D + r);
      if (f.x == 0.0 && f.y == 0.0) continue;
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (!cok[k]) continue;
        const double2 h = __ldg(P.Jdcol + (size_t)t * D + cidx[k]);
        cfma(acc[k], cmul(f, h), xs[k]);
      }
    }
    // left Hamiltonian terms: -i a G[r,p] x[p,c]
    for (int t = 0; t < P.nL; t++) {
      const int p = __ldg(P.Lmap + (size_t)t * D + r);
      if (p < 0) continue;
      const double2 v = __ldg(P.Lval + (size_t)t * D + r);
      const unsigned pr = (unsigned)(p - R0);
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (!cok[k]) continue;
        const double2 xp = (pr < (unsigned)TR) ? tile[(cidx[k] - C0) * TR + pr]
                                               : __ldg(X + (size_t)cidx[k] * D + p);
        cfma(acc[k], v, xp);
      }
    }
    // right Hamiltonian terms: +i a x[r,q] G[q,c]
    for (int t = 0; t < P.nR; t++) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (!cok[k]) continue;
        const int q = __ldg(P.Rmap + (size_t)t * D + cidx[k]);
        if (q < 0) continue;
        const double2 v = __ldg(P.Rval + (size_t)t * D + cidx[k]);
        const unsigned qc = (unsigned)(q - C0);
        const double2 xq = (qc < (unsigned)TC) ? tile[qc * TR + rr] : __ldg(X + (size_t)q * D + r);
        cfma(acc[k], v, xq);
      }
    }
    // jumps: a v(r) conj(v(c)) x[j(r), j(c)]
    for (int t = 0; t < P.nJ; t++) {
      const int p = __ldg(P.Jmap + (size_t)t * D + r);
      if (p < 0) continue;
      const double2 f = __ldg(P.Jrow + (size_t)t * D + r);
      const unsigned pr = (unsigned)(p - R0);
#pragma unroll
      for (int k = 0; k < K; k++) {
        if (!cok[k]) continue;
        const int q = __ldg(P.Jmap + (size_t)t * D + cidx[k]);
        if (q < 0) continue;
        const double2 h = __ldg(P.Jcol + (size_t)t * D + cidx[k]);
        const unsigned qc = (unsigned)(q - C0);
        const double2 xpq = (pr < (unsigned)TR && qc < (unsigned)TC)
                                ? tile[qc * TR + pr]
                                : __ldg(X + (size_t)q * D + p);
        cfma(acc[k], cmul(f, h), xpq);
      }
    }
    // fused stage epilogue
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (!cok[k]) continue;
      const size_t i = (size_t)cidx[k] * D + r;
      const double2 Kv = acc[k];
      if (E.kout) E.kout[i] = Kv;
      double2 upd[3];
#pragma unroll
      for (int u = 0; u < 3; u++) {
        if (u < E.nupd) {
          double2 b = E.base[u] ? E.base[u][i] : make_double2(0.0, 0.0);
          b.x = fma(E.coef[u], Kv.x, b.x);
          b.y = fma(E.coef[u], Kv.y, b.y);
          E.out[u][i] = b;
          upd[u] = b;
        }
      }
      if (E.nsum) {
        const double2 e = upd[E.err_upd];
        const double2 y = E.ny[i];
        const double2 yn = E.yn_upd >= 0 ? upd[E.yn_upd] : E.nyn[i];
        const double q = cabs2(e) / (E.atol + E.rtol * fmax(cabs2(y), cabs2(yn)));
        nloc += q * q;
      }
    }
  }
  if (E.nsum) {
    for (int o = 16; o > 0; o >>= 1) nloc += __shfl_down_sync(0xffffffffu, nloc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nloc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < NT / 32; w++) s += red[w];
      atomicAdd(E.nsum, s);
    }
  }
}

// Small systems (D * ncols <= 16384, every partner in L2): S threads share
// one element.  Lane s takes terms t = s, s + S, ... of every term list, the
// S partial sums are combined by a butterfly of shuffles (fixed order) and
// lane 0 applies the same epilogue as k_lrho.  S times more CTAs and S times
// shorter dependent chains than one thread per element.
template <int S>
__global__ void __launch_bounds__(NT) k_lrho_split(const DevProg P, const double2 *__restrict__ X, Epi E) {
  __shared__ double red[NT / 32];
  const int D = P.D, NC = P.ncols;
  if (blockIdx.z) {
    const size_t zoff = (size_t)blockIdx.z * D * NC;
    X += zoff;
    E.kout += zoff;
  }
  const int64_t n = (int64_t)D * NC;
  const int64_t el = ((int64_t)blockIdx.x * NT + threadIdx.x) / S;
  const int s = threadIdx.x % S;
  const bool ok = el < n;
  const int c = ok ? (int)(el / D) : 0;
  const int r = ok ? (int)(el - (int64_t)c * D) : 0;
  double2 acc = make_double2(0.0, 0.0);
  if (ok) {
    const double2 xs = __ldg(X + el);
    if (s == 0) {
      const double2 drr = __ldg(P.dr + r);
      acc = NC == 1 ? cmul(drr, xs) : cmul(cadd(drr, __ldg(P.dc + c)), xs);
    }
    // diagonal jumps: a v(r) conj(v(c)) x[r,c]
    for (int t = s; t < P.nJd; t += S) {
      const double2 f = __ldg(P.Jdrow + (size_t)t * D + r);
      if (f.x == 0.0 && f.y == 0.0) continue;
      cfma(acc, cmul(f, __ldg(P.Jdcol + (size_t)t * D + c)), xs);
    }
    // left Hamiltonian terms: -i a G[r,p] x[p,c]
    for (int t = s; t < P.nL; t += S) {
      const int p = __ldg(P.Lmap + (size_t)t * D + r);
      if (p < 0) continue;
      cfma(acc, __ldg(P.Lval + (size_t)t * D + r), __ldg(X + (size_t)c * D + p));
    }
    // right Hamiltonian terms: +i a x[r,q] G[q,c]
    for (int t = s; t < P.nR; t += S) {
      const int q = __ldg(P.Rmap + (size_t)t * D + c);
      if (q < 0) continue;
      cfma(acc, __ldg(P.Rval + (size_t)t * D + c), __ldg(X + (size_t)q * D + r));
    }
    // jumps: a v(r) conj(v(c)) x[j(r), j(c)]
    for (int t = s; t < P.nJ; t += S) {
      const int p = __ldg(P.Jmap + (size_t)t * D + r);
      if (p < 0) continue;
      const int q = __ldg(P.Jmap + (size_t)t * D + c);
      if (q < 0) continue;
      const double2 f = cmul(__ldg(P.Jrow + (size_t)t * D + r), __ldg(P.Jcol + (size_t)t * D + c));
      cfma(acc, f, __ldg(X + (size_t)q * D + p));
    }
  }
#pragma unroll
  for (int o = S / 2; o > 0; o >>= 1) {  // every lane of the group ends with the same sum
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  double nloc = 0.0;
  if (ok && s == 0) {
    const size_t i = (size_t)el;
    const double2 Kv = acc;
    if (E.kout) E.kout[i] = Kv;
    double2 upd[3];
#pragma unroll
    for (int u = 0; u < 3; u++) {
      if (u < E.nupd) {
        double2 b = E.base[u] ? E.base[u][i] : make_double2(0.0, 0.0);
        b.x = fma(E.coef[u], Kv.x, b.x);
        b.y = fma(E.coef[u], Kv.y, b.y);
        E.out[u][i] = b;
        upd[u] = b;
      }
    }
    if (E.nsum) {
      const double2 e = upd[E.err_upd];
      const double2 y = E.ny[i];
      const double2 yn = E.yn_upd >= 0 ? upd[E.yn_upd] : E.nyn[i];
      const double qv = cabs2(e) / (E.atol + E.rtol * fmax(cabs2(y), cabs2(yn)));
      nloc = qv * qv;
    }
  }
  if (E.nsum) {
    for (int o = 16; o > 0; o >>= 1) nloc += __shfl_down_sync(0xffffffffu, nloc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nloc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; w++) t += red[w];
      atomicAdd(E.nsum, t);
    }
  }
}

}  // namespace

void ensure_smem(const void *func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  int dev = 0;
  QCUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t &have = done[std::make_pair(func, dev)];
  if (have >= bytes) return;
  QCUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  if (!has_error()) have = bytes;
}

void preload_generic_lrho_kernels() {
  cudaFuncAttributes fa;
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho_split<8>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho<1>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho<2>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho<4>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho<8>));
}

void zero_epi(Epi &e) {
  memset(&e, 0, sizeof(Epi));
  e.err_upd = 0;
  e.yn_upd = -1;
}

void launch_lrho(const DevProg &P, const double2 *x, const Epi &e, cudaStream_t s, int nbatch) {
  int TR, CG, K;
  if (P.ncols == 1) {
    TR = P.D < NT ? P.D : NT;
    CG = NT / TR;
    K = 1;
  } else {
    TR = P.D < 64 ? P.D : 64;
    CG = NT / TR;
    K = 8;
    while (K > 1 && (int64_t)CG * (K / 2) >= P.ncols) K /= 2;
  }
  // small systems: several threads per element (k_lrho_split)
  if ((int64_t)P.D * P.ncols <= (int64_t)NT * 64) {
    constexpr int S = 8;
    const int64_t threads = (int64_t)P.D * P.ncols * S;
    k_lrho_split<S><<<dim3((unsigned)((threads + NT - 1) / NT), 1, nbatch), NT, 0, s>>>(P, x, e);
    count_launch();
    QCUDA(cudaGetLastError());
    return;
  }
  const int TC = CG * K;
  dim3 grid((P.D + TR - 1) / TR, (P.ncols + TC - 1) / TC, nbatch);
  const size_t smem = (size_t)TR * TC * sizeof(double2);
  switch (K) {
    case 1: k_lrho<1><<<grid, NT, smem, s>>>(P, x, e, TR, CG); break;
    case 2: k_lrho<2><<<grid, NT, smem, s>>>(P, x, e, TR, CG); break;
    case 4: k_lrho<4><<<grid, NT, smem, s>>>(P, x, e, TR, CG); break;
    default: k_lrho<8><<<grid, NT, smem, s>>>(P, x, e, TR, CG); break;
  }
  count_launch();
  QCUDA(cudaGetLastError());
}

}  // namespace quac
