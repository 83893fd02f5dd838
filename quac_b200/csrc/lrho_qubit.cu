// Matrix-free L.x for qubit systems (every subsystem two-level).
//
// Terms arrive as bit masks (QTerm, built by qubit_terms.cpp) in the kernel
// parameter block, so every thread reads them through the constant bank.
// A CTA owns a 64-row x TC-column tile of the column-stacked state (the low
// six row bits and the low log2(TC) column bits, i.e. the last-created
// qubits), staged in shared memory; partners across those bits come from
// the tile, the others from global memory (L2).  A thread owns rows
// lane and lane+32 of the tile and M columns; term data that depends only
// on the row (or the column) is evaluated once and reused across the block.
// With all Hamiltonian coefficients purely imaginary and all jump rates
// real (real couplings, Pauli X/Z and ladder operators) each partner costs
// two FMAs instead of four.
#include "runtime.h"

namespace quac {

namespace {

constexpr int QNT = 256;

struct QParams {
  QubitProg prog;
  QTerm t[QMAX_TERMS];
};

__device__ __forceinline__ double2 cmulq(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ void cfmaq(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ double cabsq(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

template <int M, bool REAL>
__global__ void __launch_bounds__(QNT) k_lrho_qubit(const __grid_constant__ QParams Qp,
                                                    const double2 *__restrict__ X, const Epi E) {
  constexpr int TC = 8 * M;
  extern __shared__ double2 sm[];
  double2 *tile = sm;               // TC * 64, column-major (64 rows per column)
  double2 *drs = tile + TC * 64;    // 64
  double2 *dcs = drs + 64;          // TC
  double2 *gts = dcs + TC;          // ngroups * 64
  __shared__ double red[QNT / 32];
  const QubitProg &Q = Qp.prog;
  const int n = Q.n;
  const int D = 1 << n;
  const int R0 = blockIdx.x * 64;
  const int C0 = blockIdx.y * TC;
  for (int idx = threadIdx.x; idx < TC * 64; idx += QNT) {
    const int cc = idx >> 6, rr = idx & 63;
    tile[idx] = __ldg(X + (size_t)(C0 + cc) * D + R0 + rr);
  }
  if (threadIdx.x < 64) drs[threadIdx.x] = __ldg(Q.dr + R0 + threadIdx.x);
  if (threadIdx.x < TC) dcs[threadIdx.x] = __ldg(Q.dc + C0 + threadIdx.x);
  for (int i = threadIdx.x; i < Q.ngroups * 64; i += QNT) gts[i] = __ldg(Q.gtab + i);
  __syncthreads();

  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int rl[2], r[2], cl[M], c[M];
  rl[0] = lane;
  rl[1] = lane + 32;
  r[0] = R0 + rl[0];
  r[1] = R0 + rl[1];
#pragma unroll
  for (int m = 0; m < M; m++) {
    cl[m] = w + 8 * m;
    c[m] = C0 + cl[m];
  }
  double2 acc[2][M], xs[2][M];
#pragma unroll
  for (int i = 0; i < 2; i++) {
#pragma unroll
    for (int m = 0; m < M; m++) {
      xs[i][m] = tile[cl[m] * 64 + rl[i]];
      double2 d = drs[rl[i]];
      const double2 dc = dcs[cl[m]];
      d.x += dc.x;
      d.y += dc.y;
      for (int g = 0; g < Q.ngroups; g++) {
        const double2 v = gts[g * 64 + (((r[i] >> (3 * g)) & 7) << 3) + ((c[m] >> (3 * g)) & 7)];
        d.x += v.x;
        d.y += v.y;
      }
      acc[i][m] = cmulq(d, xs[i][m]);
    }
  }
  int t = 0;
  // left (row) terms
  for (int e = t + Q.nL; t < e; t++) {
    const QTerm T = Qp.t[t];
    const bool local = (T.fmask >> 6) == 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      if ((r[i] & T.cmask) != T.cval) continue;
      const bool neg = __popc(r[i] & T.smask) & 1;
      const int pr = r[i] ^ T.fmask;
      if (REAL) {
        const double wv = neg ? -T.coef.y : T.coef.y;
#pragma unroll
        for (int m = 0; m < M; m++) {
          const double2 p = local ? tile[cl[m] * 64 + (pr - R0)] : __ldg(X + (size_t)c[m] * D + pr);
          acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
          acc[i][m].y = fma(wv, p.x, acc[i][m].y);
        }
      } else {
        const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
#pragma unroll
        for (int m = 0; m < M; m++) {
          const double2 p = local ? tile[cl[m] * 64 + (pr - R0)] : __ldg(X + (size_t)c[m] * D + pr);
          cfmaq(acc[i][m], wv, p);
        }
      }
    }
  }
  // right (column) terms
  for (int e = t + Q.nR; t < e; t++) {
    const QTerm T = Qp.t[t];
    const bool local = (T.fmask / TC) == 0;
#pragma unroll
    for (int m = 0; m < M; m++) {
      if ((c[m] & T.cmask) != T.cval) continue;
      const bool neg = __popc(c[m] & T.smask) & 1;
      const int pc = c[m] ^ T.fmask;
      if (REAL) {
        const double wv = neg ? -T.coef.y : T.coef.y;
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const double2 p = local ? tile[(pc - C0) * 64 + rl[i]] : __ldg(X + (size_t)pc * D + r[i]);
          acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
          acc[i][m].y = fma(wv, p.x, acc[i][m].y);
        }
      } else {
        const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const double2 p = local ? tile[(pc - C0) * 64 + rl[i]] : __ldg(X + (size_t)pc * D + r[i]);
          cfmaq(acc[i][m], wv, p);
        }
      }
    }
  }
  // jumps: partner (r ^ f, c ^ f)
  for (int e = t + Q.nJ; t < e; t++) {
    const QTerm T = Qp.t[t];
    const bool local = (T.fmask >> 6) == 0 && (T.fmask / TC) == 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
      if ((r[i] & T.cmask) != T.cval) continue;
      const int sr = __popc(r[i] & T.smask);
      const int pr = r[i] ^ T.fmask;
#pragma unroll
      for (int m = 0; m < M; m++) {
        if ((c[m] & T.cmask) != T.cval) continue;
        const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
        const int pc = c[m] ^ T.fmask;
        const double2 p = local ? tile[(pc - C0) * 64 + (pr - R0)] : __ldg(X + (size_t)pc * D + pr);
        if (REAL) {
          const double wv = neg ? -T.coef.x : T.coef.x;
          acc[i][m].x = fma(wv, p.x, acc[i][m].x);
          acc[i][m].y = fma(wv, p.y, acc[i][m].y);
        } else {
          const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
          cfmaq(acc[i][m], wv, p);
        }
      }
    }
  }
  // multi-qubit diagonal jumps
  for (int e = t + Q.nJx; t < e; t++) {
    const QTerm T = Qp.t[t];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      if ((r[i] & T.cmask) != T.cval) continue;
      const int sr = __popc(r[i] & T.smask);
#pragma unroll
      for (int m = 0; m < M; m++) {
        if ((c[m] & T.cmask) != T.cval) continue;
        const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
        const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
        cfmaq(acc[i][m], wv, xs[i][m]);
      }
    }
  }
  // fused stage epilogue
  double nloc = 0.0;
#pragma unroll
  for (int i = 0; i < 2; i++) {
#pragma unroll
    for (int m = 0; m < M; m++) {
      const size_t idx = (size_t)c[m] * D + r[i];
      const double2 Kv = acc[i][m];
      if (E.kout) E.kout[idx] = Kv;
      double2 upd[3];
#pragma unroll
      for (int u = 0; u < 3; u++) {
        if (u < E.nupd) {
          double2 b = E.base[u] ? E.base[u][idx] : make_double2(0.0, 0.0);
          b.x = fma(E.coef[u], Kv.x, b.x);
          b.y = fma(E.coef[u], Kv.y, b.y);
          E.out[u][idx] = b;
          upd[u] = b;
        }
      }
      if (E.nsum) {
        const double2 ev = upd[E.err_upd];
        const double2 y = E.ny[idx];
        const double2 yn = E.yn_upd >= 0 ? upd[E.yn_upd] : E.nyn[idx];
        const double q = cabsq(ev) / (E.atol + E.rtol * fmax(cabsq(y), cabsq(yn)));
        nloc += q * q;
      }
    }
  }
  if (E.nsum) {
    for (int o = 16; o > 0; o >>= 1) nloc += __shfl_down_sync(0xffffffffu, nloc, o);
    if (lane == 0) red[w] = nloc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int k = 0; k < QNT / 32; k++) s += red[k];
      atomicAdd(E.nsum, s);
    }
  }
}

template <int M, bool REAL>
void launch_q(const QParams &qp, const double2 *x, const Epi &e, cudaStream_t s) {
  constexpr int TC = 8 * M;
  const int D = 1 << qp.prog.n;
  const size_t smem = (size_t)(TC * 64 + 64 + TC + qp.prog.ngroups * 64) * sizeof(double2);
  ensure_smem((const void *)k_lrho_qubit<M, REAL>, smem + 4096);
  dim3 grid(D / 64, D / TC);
  k_lrho_qubit<M, REAL><<<grid, QNT, smem, s>>>(qp, x, e);
}

}  // namespace

void preload_single_pass_qubit_kernels() {
  cudaFuncAttributes fa;
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho_qubit<4, true>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho_qubit<4, false>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho_qubit<8, true>));
  QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_lrho_qubit<8, false>));
}

void launch_lrho_qubit(const DeviceProgram &P, const double2 *x, const Epi &e, cudaStream_t s) {
  static QParams qp;  // assembled on the host per launch (5-6 KB parameter block)
  qp.prog = P.qdev;
  const size_t nt = P.qterms.size();
  for (size_t k = 0; k < nt; k++) qp.t[k] = P.qterms[k];
  const int D = 1 << P.qdev.n;
  const bool real = P.qdev.real != 0;
  if (D >= 64 * 64) {
    if (real) launch_q<8, true>(qp, x, e, s);
    else launch_q<8, false>(qp, x, e, s);
  } else {
    if (real) launch_q<4, true>(qp, x, e, s);
    else launch_q<4, false>(qp, x, e, s);
  }
  count_launch();
  QCUDA(cudaGetLastError());
}

void launch_lrho_any(const DeviceProgram &P, const double2 *x, const Epi &e, cudaStream_t s) {
  if (P.has_qubit && !P.passes.empty()) {
    DeviceProgram &M = const_cast<DeviceProgram &>(P);
    if (!M.scratch) {
      const size_t n = (size_t)P.dev.D * P.dev.ncols;
      QCUDA(cudaMalloc(&M.scratch, n * sizeof(double2)));
      M.allocations.push_back(M.scratch);
    }
    launch_qubit_passes(M.passes, x, M.scratch, e, s, options().lrho_f32 != 0);
  } else if (P.has_qubit) {
    launch_lrho_qubit(P, x, e, s);
  } else {
    launch_lrho(P.dev, x, e, s);
  }
}

bool launch_lrho_batch(const DeviceProgram &P, const double2 *x, double2 *y, int nbatch, cudaStream_t s) {
  if (P.has_qubit || nbatch < 1 || nbatch > 65535) return false;  // qubit kernels: one vector per launch
  Epi e;
  zero_epi(e);
  e.kout = y;
  launch_lrho(P.dev, x, e, s, nbatch);
  return true;
}

}  // namespace quac
