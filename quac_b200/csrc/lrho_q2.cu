// Multi-pass matrix-free L.x for qubit systems (n >= 7 qubits).
//
// The 2n bits of the column-stacked index (row bits r_0..r_{n-1}, column
// bits c_0..c_{n-1}) are covered by groups of six bit positions [lo, lo+6),
// applied to rows and columns alike.  Pass p owns 64 x 64 tiles whose free
// bits are group p for rows and columns; every term whose flip mask lies in
// group p (left: row flips, right: column flips, jumps: both) finds its
// partners inside the tile.  The high groups run first and accumulate into a
// running-sum vector; the pass over group 0 (contiguous rows) also applies
// the diagonal and runs the fused stage epilogue.  CTAs are persistent (one
// per SM), claim work items from a queue in global memory and stream tiles
// through three shared-memory stages filled by TMA, so the next tiles' loads
// overlap the current tile's arithmetic.
//
// Hermitian mode (x Hermitian, L Hermiticity-preserving): the last pass
// computes only the 64 x 64 blocks I <= J of the bits above group 0 and
// writes each off-diagonal block's conjugate transpose as well.  In a
// two-pass program the first pass then works on tile pairs: tile (b, a) of
// its fixed low bits is the conjugate transpose of tile (a, b), so one load
// serves both, halving that pass's reads of x.
#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <atomic>

#include <cuda.h>

#include "common.h"

namespace quac {

namespace {

constexpr int TILE = 64;           // tile rows = tile columns
constexpr int NEL = TILE * TILE;   // elements per tile
__device__ __forceinline__ void cfma2(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma2(float2 &acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
template <typename V2>
__device__ __forceinline__ V2 to_v2(double2 v);
template <>
__device__ __forceinline__ double2 to_v2<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 to_v2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double cabs2d(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_u32(bar))
      : "memory");
}

// triangular work index t = b (b + 1) / 2 + a  ->  (a, b), a <= b
__device__ __forceinline__ void tri_index(long long t, unsigned &a, unsigned &b) {
  long long J = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((J + 1) * (J + 2) / 2 <= t) J++;
  while (J * (J + 1) / 2 > t) J--;
  a = (unsigned)(t - J * (J + 1) / 2);
  b = (unsigned)J;
}

// fixed (non-tile) bits of a work item: rows then columns
__device__ __forceinline__ void tile_origin(const PassParams &P, long long t, unsigned &rfix, unsigned &cfix) {
  if (P.herm_tiles) {
    // blocks I <= J of the bits above the low group (lo == 0)
    unsigned I, J;
    tri_index(t, I, J);
    rfix = I << 6;
    cfix = J << 6;
    return;
  }
  if (P.pair_tiles) {
    // tile pairs a <= b of the fixed low bits [0, lo) (lo + 6 == n)
    tri_index(t, rfix, cfix);
    return;
  }
  const int n = P.n, lo = P.lo;
  const int hi = lo + 6;
  const unsigned lowmask = (1u << lo) - 1u;
  const int nhigh = n - hi;
  const unsigned r_lo = (unsigned)(t & lowmask);
  t >>= lo;
  const unsigned r_hi = (unsigned)(t & ((1ll << nhigh) - 1));
  t >>= nhigh;
  const unsigned c_lo = (unsigned)(t & lowmask);
  t >>= lo;
  const unsigned c_hi = (unsigned)t;
  rfix = r_lo | (r_hi << hi);
  cfix = c_lo | (c_hi << hi);
}

__device__ __forceinline__ void load_tile(double2 *buf, const double2 *__restrict__ X, long long t,
                                          const PassParams &P) {
  unsigned rfix, cfix;
  tile_origin(P, t, rfix, cfix);
  const size_t D = (size_t)1 << P.n;
  for (int e = threadIdx.x; e < NEL; e += blockDim.x) {
    const unsigned cl = e >> 6, rl = e & 63;
    const size_t r = rfix | (rl << P.lo), c = cfix | (cl << P.lo);
    cp_async16(buf + e, X + c * D + r);
  }
}

// issues the TMA load of work item t into buf (thread 0 only)
__device__ __forceinline__ void tma_tile(const PassParams &P, const CUtensorMap *map, double2 *buf,
                                         uint64_t *bar, long long t) {
  unsigned rfix, cfix;
  tile_origin(P, t, rfix, cfix);
  const unsigned long long F = (unsigned long long)rfix | ((unsigned long long)cfix << P.n);
  int c[5] = {0, 0, 0, 0, 0};
  // a fixed run merged into dim 0: two doubles per element
  if (!P.tfree[0]) c[0] = (int)(2ull * (F & ((1ull << P.tlen[0]) - 1ull)));
#pragma unroll
  for (int d = 1; d < 5; d++)
    c[d] = P.tfree[d] ? 0 : (int)((F >> P.tstart[d]) & ((1ull << P.tlen[d]) - 1ull));
  mbar_expect_tx(bar, NEL * sizeof(double2));
  tma_load_5d(buf, map, bar, c[0], c[1], c[2], c[3], c[4]);
}

// waits for phase `parity` of bar for at most `limit_ns`; false on time-out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}

// stage value base_u + coef_u K of the epilogue (base of update 0 from registers)
__device__ __forceinline__ double2 stage_value(const Epi &E, int u, size_t idx, double2 Kv, double2 b0) {
  double2 b = u == 0 ? b0 : (E.base[u] ? E.base[u][idx] : make_double2(0.0, 0.0));
  return make_double2(fma(E.coef[u], Kv.x, b.x), fma(E.coef[u], Kv.y, b.y));
}

#ifndef QUAC_QPASS_THREADS
#define QUAC_QPASS_THREADS 512
#endif
constexpr int QT = QUAC_QPASS_THREADS;  // threads of the pass kernel (256, 512 or 1024)
constexpr int QNW = QT / 32;            // warps
constexpr int QMC = 64 / QNW;           // tile columns per thread
static_assert(QMC == 2 || QMC == 4 || QMC == 8, "pass kernel runs 256, 512 or 1024 threads");
// thread column m holds tile column w + QNW m: bit 0 of m is column bit
// QCB, so flips of column bits >= QCB are register moves
constexpr int QCB = QMC == 8 ? 3 : (QMC == 4 ? 4 : 5);
__host__ __device__ constexpr int qcol_flip(int b) { return b >= QCB ? 1 << (b - QCB) : 0; }

// One pass over 64 x 64 tiles.  Thread (lane, w) owns tile rows lane,
// lane + 32 and columns w + QNW m (512 threads: w, w + 16, w + 32, w + 48);
// its values sit in registers, so flips of row bit 5 and of the column bits
// >= QCB need no shared-memory read.  CANON (real mode only) is a compile-time mask of the
// canonical single-bit kinds present: 1 = left X, 2 = right X, 4 = lowering
// jump, 8 = raising jump; CANON < 0 means the kinds are decided at run
// time.  With TMA the CTAs are persistent, claim work items from a queue
// when they issue the load (two items ahead, three stages), and prefetch
// the running sum and the first stage base into registers before waiting
// for the tile.
template <bool REAL, bool TMA, int CANON, bool F32>
__global__ void __launch_bounds__(QT, 1) k_qpass(const __grid_constant__ PassParams P,
                                                 const __grid_constant__ CUtensorMap tmap,
                                                 const __grid_constant__ CUtensorMap bmap,
                                                 const double2 *__restrict__ X, const Epi E) {
  constexpr int NST = TMA ? 3 : 2;   // shared-memory buffers of NEL values
  // complex128 contraction, or (F32) complex64 contraction of tiles
  // converted in shared memory, accumulated in complex64
  using V2 = typename std::conditional<F32, float2, double2>::type;
  using S = typename std::conditional<F32, float, double>::type;
  extern __shared__ __align__(128) double2 sm[];
  double2 *gts = sm + NST * NEL;     // ngroups * 64, layout [g][col bits][row bits]
  __shared__ double red[QNW];
  __shared__ __align__(8) uint64_t bars[4];
  __shared__ long long tids[3];
  // last pass with TMA: the first stage base of each tile comes by TMA into
  // the third buffer, and the tiles of x use two stages
  const bool bt = TMA && P.last && E.nupd > 0 && E.base[0] != nullptr;
  // a middle pass (running sum in and out, complex128): its running-sum tile
  // comes by TMA into the third buffer (the tensor map in bmap) and is added
  // after the pass's own terms, instead of single 16-byte loads per thread
  const bool at = TMA && !F32 && !P.last && P.accin != nullptr;
  const int nst = TMA ? ((bt || at) ? 2 : 3) : 2;
  const double2 *bbuf = sm + 2 * NEL;
  const int n = P.n, lo = P.lo;
  const size_t D = (size_t)1 << n;
  if (P.diag)
    for (int i = threadIdx.x; i < P.ngroups * 64; i += QT) {
      const int g = i >> 6, rb = (i >> 3) & 7, cb = i & 7;  // source layout [g][rb][cb]
      gts[(g << 6) | (cb << 3) | rb] = P.gtab[i];
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double nloc = 0.0;
  bool timed_out = false;
  int it = 0;
  if (TMA) {
    if (threadIdx.x == 0) {
      for (int q = 0; q < 4; q++) mbar_init(&bars[q], 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
      for (int q = 0; q < nst - 1; q++) {
        const long long tq = (long long)atomicAdd(P.claim, 1ull);
        tids[q] = tq;
        if (tq < P.ntiles) tma_tile(P, &tmap, sm + q * NEL, &bars[q], tq);
      }
    }
  } else {
    if (blockIdx.x < P.ntiles) load_tile(sm, X, blockIdx.x, P);
    cp_commit();
  }
  __syncthreads();
  long long t_static = blockIdx.x;
  for (;; it++) {
    const long long t = TMA ? tids[it % nst] : t_static;
    if (t >= P.ntiles) break;
    double2 *cur = sm + (it % nst) * NEL;
    if (TMA && threadIdx.x == 0) {
      const int q2 = (it + nst - 1) % nst;
      const long long t2 = (long long)atomicAdd(P.claim, 1ull);
      tids[q2] = t2;
      if (t2 < P.ntiles) tma_tile(P, &tmap, sm + q2 * NEL, &bars[q2], t2);
      if (bt || at) tma_tile(P, &bmap, sm + 2 * NEL, &bars[3], t);
    }
    unsigned rfix, cfix;
    tile_origin(P, t, rfix, cfix);
    // an off-diagonal block also stands for its conjugate transpose
    const bool mirror = P.herm_tiles && rfix != cfix;
    unsigned rl[2] = {(unsigned)lane, (unsigned)lane + 32u};
    unsigned cl[QMC];
#pragma unroll
    for (int m = 0; m < QMC; m++) cl[m] = (unsigned)(w + QNW * m);
    unsigned r[2], c[QMC];
#pragma unroll
    for (int i = 0; i < 2; i++) r[i] = rfix | (rl[i] << lo);
#pragma unroll
    for (int m = 0; m < QMC; m++) c[m] = cfix | (cl[m] << lo);
    // loads that do not depend on the tile go out before the wait
    V2 acc[2][QMC];
    if (P.accin && !at) {
      const V2 *ain = reinterpret_cast<const V2 *>(P.accin);
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < QMC; m++) acc[i][m] = ain[(size_t)c[m] * D + r[i]];
    } else {
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < QMC; m++) acc[i][m] = to_v2<V2>(make_double2(0.0, 0.0));
    }
    if (TMA) {
      const bool ok = mbar_wait_bounded(&bars[it % nst], (unsigned)((it / nst) & 1), 2000000000ull);
      if (__syncthreads_or(!ok)) { timed_out = true; break; }
    } else {
      const long long tn = t + gridDim.x;
      if (tn < P.ntiles) load_tile(sm + ((it + 1) & 1) * NEL, X, tn, P);
      cp_commit();
      cp_wait<1>();
      __syncthreads();
    }
    const V2 *tile = reinterpret_cast<const V2 *>(cur);
    if (F32) {
      // in place: every thread reads its complex128 elements before any
      // complex64 value is written over them
      double2 tmp[NEL / QT];
#pragma unroll
      for (int k2 = 0; k2 < NEL / QT; k2++) tmp[k2] = cur[threadIdx.x + k2 * QT];
      __syncthreads();
      float2 *c32 = reinterpret_cast<float2 *>(cur);
#pragma unroll
      for (int k2 = 0; k2 < NEL / QT; k2++)
        c32[threadIdx.x + k2 * QT] = make_float2((float)tmp[k2].x, (float)tmp[k2].y);
      __syncthreads();
    }
    V2 xo[2][QMC];  // own values
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int m = 0; m < QMC; m++) xo[i][m] = tile[cl[m] * 64 + rl[i]];
    if (P.diag) {
      // groups 0 and 1 vary inside the tile (lo == 0 here); the others are
      // fixed by the tile origin
      double2 gconst = make_double2(0.0, 0.0);
      for (int g = 2; g < P.ngroups; g++) {
        const double2 v = gts[(g << 6) | (((cfix >> (3 * g)) & 7u) << 3) | ((rfix >> (3 * g)) & 7u)];
        gconst.x += v.x;
        gconst.y += v.y;
      }
#pragma unroll
      for (int i = 0; i < 2; i++) {
        double2 dri = __ldg(P.dr + r[i]);
        dri.x += gconst.x;
        dri.y += gconst.y;
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          double2 d = __ldg(P.dc + c[m]);
          d.x += dri.x;
          d.y += dri.y;
          const double2 v0 = gts[((c[m] & 7u) << 3) | (r[i] & 7u)];
          d.x += v0.x;
          d.y += v0.y;
          if (P.ngroups > 1) {
            const double2 v1 = gts[64 | (((c[m] >> 3) & 7u) << 3) | ((r[i] >> 3) & 7u)];
            d.x += v1.x;
            d.y += v1.y;
          }
          cfma2(acc[i][m], to_v2<V2>(d), xo[i][m]);
        }
      }
    }
    if (REAL && (CANON > 0 || (CANON < 0 && P.ncanon))) {
      constexpr bool C_HL = CANON < 0 || (CANON & 1), C_HR = CANON < 0 || (CANON & 2);
      constexpr bool C_GL = CANON < 0 || (CANON & 4), C_GU = CANON < 0 || (CANON & 8);
      // canonical single-bit terms: partner offsets are compile-time
      // constants; absent kinds are compiled out, zero coefficients are
      // applied as zeros (no branches between terms).  Partners across row
      // bit 5 or column bits 4, 5 come from the thread's own registers.
#pragma unroll
      for (int b = 0; b < 6; b++) {
        const unsigned f = 1u << b;
        if (C_HL) {
          const S hl = (S)P.hl[b];
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < QMC; m++) {
              const V2 p = b == 5 ? xo[i ^ 1][m] : tile[cl[m] * 64 + (rl[i] ^ f)];
              acc[i][m].x = fma(-hl, p.y, acc[i][m].x);
              acc[i][m].y = fma(hl, p.x, acc[i][m].y);
            }
        }
        if (C_HR) {
          const S hr = (S)P.hr[b];
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < QMC; m++) {
              const V2 p = b >= QCB ? xo[i][m ^ qcol_flip(b)] : tile[(cl[m] ^ f) * 64 + rl[i]];
              acc[i][m].x = fma(-hr, p.y, acc[i][m].x);
              acc[i][m].y = fma(hr, p.x, acc[i][m].y);
            }
        }
        if (C_GL || C_GU) {
          const S gl = C_GL ? (S)P.gl[b] : (S)0, gu = C_GU ? (S)P.gu[b] : (S)0;
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < QMC; m++) {
              const bool rb = rl[i] & f, cb = cl[m] & f;
              const S g = (rb != cb) ? (S)0 : (rb ? gu : gl);
              const V2 p = b == 5 ? xo[i ^ 1][m ^ qcol_flip(5)] : tile[(cl[m] ^ f) * 64 + (rl[i] ^ f)];
              acc[i][m].x = fma(g, p.x, acc[i][m].x);
              acc[i][m].y = fma(g, p.y, acc[i][m].y);
            }
        }
      }
    }
    int k = 0;
    for (int e = k + P.nL; k < e; k++) {
      const PassTerm T = P.t[k];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        if ((r[i] & T.cmask) != T.cval) continue;
        const bool neg = __popc(r[i] & T.smask) & 1;
        const unsigned pr = rl[i] ^ T.fl;
        if (REAL) {
          const S wv = (S)(neg ? -T.coef.y : T.coef.y);
#pragma unroll
          for (int m = 0; m < QMC; m++) {
            const V2 p = tile[cl[m] * 64 + pr];
            acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
            acc[i][m].y = fma(wv, p.x, acc[i][m].y);
          }
        } else {
          const V2 wv = to_v2<V2>(neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef);
#pragma unroll
          for (int m = 0; m < QMC; m++) cfma2(acc[i][m], wv, tile[cl[m] * 64 + pr]);
        }
      }
    }
    for (int e = k + P.nR; k < e; k++) {
      const PassTerm T = P.t[k];
#pragma unroll
      for (int m = 0; m < QMC; m++) {
        if ((c[m] & T.cmask) != T.cval) continue;
        const bool neg = __popc(c[m] & T.smask) & 1;
        const unsigned pc = cl[m] ^ T.fl;
        if (REAL) {
          const S wv = (S)(neg ? -T.coef.y : T.coef.y);
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const V2 p = tile[pc * 64 + rl[i]];
            acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
            acc[i][m].y = fma(wv, p.x, acc[i][m].y);
          }
        } else {
          const V2 wv = to_v2<V2>(neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef);
#pragma unroll
          for (int i = 0; i < 2; i++) cfma2(acc[i][m], wv, tile[pc * 64 + rl[i]]);
        }
      }
    }
    for (int e = k + P.nJ; k < e; k++) {
      const PassTerm T = P.t[k];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        if ((r[i] & T.cmask) != T.cval) continue;
        const int sr = __popc(r[i] & T.smask);
        const unsigned pr = rl[i] ^ T.fl;
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          if ((c[m] & T.cmask) != T.cval) continue;
          const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
          const V2 p = tile[(cl[m] ^ T.fl) * 64 + pr];
          if (REAL) {
            const S wv = (S)(neg ? -T.coef.x : T.coef.x);
            acc[i][m].x = fma(wv, p.x, acc[i][m].x);
            acc[i][m].y = fma(wv, p.y, acc[i][m].y);
          } else {
            cfma2(acc[i][m], to_v2<V2>(neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef), p);
          }
        }
      }
    }
    for (int e = k + P.nJx; k < e; k++) {  // multi-qubit diagonal jumps (diagonal pass)
      const PassTerm T = P.t[k];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        if ((r[i] & T.cmask) != T.cval) continue;
        const int sr = __popc(r[i] & T.smask);
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          if ((c[m] & T.cmask) != T.cval) continue;
          const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
          cfma2(acc[i][m], to_v2<V2>(neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef), xo[i][m]);
        }
      }
    }
    // cross-group terms (flip bits in two groups): global loads.  Stored
    // after the pass's own terms with fl holding the full flip mask and the
    // kind (L, R, J) in its top bits.
    for (int s = 0; s < P.nspill; s++, k++) {
      const PassTerm T = P.t[k];
      const int kind = (int)(T.fl >> 29);
      const unsigned f = T.fl & 0x1fffffffu;
#pragma unroll
      for (int i = 0; i < 2; i++) {
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          const bool okr = (r[i] & T.cmask) == T.cval, okc = (c[m] & T.cmask) == T.cval;
          size_t pidx;
          int sg;
          if (kind == 0) {
            if (!okr) continue;
            pidx = (size_t)c[m] * D + (r[i] ^ f);
            sg = __popc(r[i] & T.smask);
          } else if (kind == 1) {
            if (!okc) continue;
            pidx = (size_t)(c[m] ^ f) * D + r[i];
            sg = __popc(c[m] & T.smask);
          } else {
            if (!okr || !okc) continue;
            pidx = (size_t)(c[m] ^ f) * D + (r[i] ^ f);
            sg = __popc(r[i] & T.smask) + __popc(c[m] & T.smask);
          }
          cfma2(acc[i][m], to_v2<V2>((sg & 1) ? make_double2(-T.coef.x, -T.coef.y) : T.coef),
                to_v2<V2>(__ldg(X + pidx)));
        }
      }
    }
    if (bt || at) {
      const bool ok = mbar_wait_bounded(&bars[3], (unsigned)(it & 1), 2000000000ull);
      if (__syncthreads_or(!ok)) { timed_out = true; break; }
    }
    if (at) {
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          const double2 v = bbuf[cl[m] * 64 + rl[i]];
          acc[i][m].x += v.x;
          acc[i][m].y += v.y;
        }
    }
    // first stage base of element (i, m)
    auto base0 = [&](int i, int m, size_t idx) -> double2 {
      if (bt) return bbuf[cl[m] * 64 + rl[i]];
      return (E.nupd > 0 && E.base[0]) ? E.base[0][idx] : make_double2(0.0, 0.0);
    };
    if (!P.last) {
      // running sum for the later passes
      V2 *aout = reinterpret_cast<V2 *>(P.accout);
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          if (!P.pair_tiles) {
            aout[(size_t)c[m] * D + r[i]] = acc[i][m];
            continue;
          }
          // tile (a, b) at its own positions, and its conjugate transpose at
          // the transposed positions (those of tile (b, a)), wherever the
          // last pass reads the running sum
          if ((r[i] >> 6) <= (c[m] >> 6)) aout[(size_t)c[m] * D + r[i]] = acc[i][m];
          if (rfix != cfix && (c[m] >> 6) <= (r[i] >> 6)) {
            V2 v = acc[i][m];
            v.y = -v.y;
            aout[(size_t)r[i] * D + c[m]] = v;
          }
        }
    } else if (!P.herm_tiles) {
#pragma unroll
      for (int i = 0; i < 2; i++) {
#pragma unroll
        for (int m = 0; m < QMC; m++) {
          const size_t idx = (size_t)c[m] * D + r[i];
          const double2 Kv = make_double2((double)acc[i][m].x, (double)acc[i][m].y);
          if (E.kout) E.kout[idx] = Kv;
          double2 u0 = make_double2(0.0, 0.0), u1 = u0, u2 = u0;
          const double2 b0 = base0(i, m, idx);
          if (E.nupd > 0) E.out[0][idx] = u0 = stage_value(E, 0, idx, Kv, b0);
          if (E.nupd > 1) E.out[1][idx] = u1 = stage_value(E, 1, idx, Kv, b0);
          if (E.nupd > 2) E.out[2][idx] = u2 = stage_value(E, 2, idx, Kv, b0);
          if (E.nsum) {
            const double2 ev = E.err_upd == 0 ? u0 : (E.err_upd == 1 ? u1 : u2);
            const double2 y = E.ny[idx];
            const double2 yn = E.yn_upd == 0 ? u0 : (E.yn_upd == 1 ? u1 : (E.yn_upd == 2 ? u2 : E.nyn[idx]));
            const double q = cabs2d(ev) / (E.atol + E.rtol * fmax(cabs2d(y), cabs2d(yn)));
            nloc += q * q;
          }
        }
      }
    } else {
      // Hermitian blocks: every output is written at its own position and,
      // through the tile buffer, conjugate-transposed at block (J, I); a
      // diagonal block rewrites its strictly lower triangle as the conjugate
      // of the upper one and zeroes the imaginary part of its diagonal, so
      // the state stays exactly Hermitian.  Element (r, c) is staged at
      // c*64 + (r ^ c): both the staging stores and the transposed reads are
      // conflict-free.
      double2 *stg = cur;
      const int nd = (E.kout ? 1 : 0) + E.nupd;
      for (int o = 0; o < nd; o++) {
        const int u = E.kout ? o - 1 : o;
        double2 *dst = u < 0 ? E.kout : E.out[u];
        __syncthreads();  // the tile (o == 0) or the previous staging has been read
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
          for (int m = 0; m < QMC; m++) {
            const size_t idx = (size_t)c[m] * D + r[i];
            const double2 Kv = make_double2((double)acc[i][m].x, (double)acc[i][m].y);
            const double2 b0 = u == 0 || E.yn_upd == 0 ? base0(i, m, idx) : make_double2(0.0, 0.0);
            const double2 v = u < 0 ? Kv : stage_value(E, u, idx, Kv, b0);
            dst[idx] = v;
            stg[cl[m] * 64 + (rl[i] ^ cl[m])] = v;
            if (E.nsum && u == E.err_upd) {
              const double2 y = E.ny[idx];
              const double2 yn = E.yn_upd >= 0 ? stage_value(E, E.yn_upd, idx, Kv, b0) : E.nyn[idx];
              const double q = cabs2d(v) / (E.atol + E.rtol * fmax(cabs2d(y), cabs2d(yn)));
              nloc += mirror ? 2.0 * q * q : q * q;
            }
          }
        __syncthreads();
        for (int e2 = threadIdx.x; e2 < NEL; e2 += QT) {
          const unsigned a = e2 & 63u, b = e2 >> 6;
          double2 v = stg[a * 64 + (b ^ a)];  // value at (row b, column a) of block (I, J)
          v.y = -v.y;
          if (mirror || a > b) dst[(size_t)(rfix | b) * D + (cfix | a)] = v;
          else if (a == b) dst[(size_t)(rfix | b) * D + (cfix | a)] = make_double2(v.x, 0.0);
        }
      }
    }
    __syncthreads();  // every thread is done with cur before it is refilled
    if (!TMA) t_static += gridDim.x;
  }
  if (!TMA) cp_wait<0>();
  if (TMA && threadIdx.x == 0) {
    if (timed_out) {
      // no new loads were issued after the time-out; give every load still
      // outstanding (this stage and the two prefetched ones) a bounded wait
      // so the CTA does not exit with copies in flight (if these waits run
      // out as well, it exits anyway and the error word reports the run)
      if (P.errflag) atomicExch(P.errflag, 1);
      for (int k2 = 0; k2 < nst; k2++) {
        const int q = (it + k2) % nst;
        if (tids[q] < P.ntiles) mbar_wait_bounded(&bars[q], (unsigned)(((it + k2) / nst) & 1), 500000000ull);
      }
      if (bt || at) mbar_wait_bounded(&bars[3], (unsigned)(it & 1), 500000000ull);
    }
    // queue reset by the last CTA: every CTA has made its final claim
    // before it counts itself here
    __threadfence();
    if (atomicAdd(P.done, 1u) == gridDim.x - 1) {
      atomicExch(P.claim, 0ull);
      atomicExch(P.done, 0u);
    }
  }
  if (P.last && E.nsum) {
    for (int o = 16; o > 0; o >>= 1) nloc += __shfl_down_sync(0xffffffffu, nloc, o);
    if (lane == 0) red[w] = nloc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < QNW; q++) s += red[q];
      atomicAdd(E.nsum, s);
    }
  }
}

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    QCUDA(cudaGetDevice(&dev));
    QCUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    QCUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) fail(9, "ERROR! cuTensorMapEncodeTiled unavailable\n");
    fn = (EncodeTiledFn)p;
  }
  return fn;
}

// Describes the 64x64 tile of a pass as a 5-D box over the flat index.
// Returns false when the runs of fixed and free bits need more than five
// dimensions (then the cp.async path is used).
bool describe_tma(PassParams &pp) {
  const int n = pp.n, lo = pp.lo;
  struct Run { int start, len; bool free; };
  std::vector<Run> runs;
  auto add = [&](int start, int len, bool fr) {
    if (len <= 0) return;
    if (!runs.empty() && runs.back().free == fr && runs.back().start + runs.back().len == start)
      runs.back().len += len;
    else
      runs.push_back({start, len, fr});
  };
  add(0, lo, false);
  add(lo, 6, true);
  add(lo + 6, n - lo - 6, false);
  add(n, lo, false);
  add(n + lo, 6, true);
  add(n + lo + 6, n - lo - 6, false);
  // dim 0 = the element (two doubles), merged with a leading free run; when
  // the runs need more than five dimensions (a middle group: fixed bits on
  // both sides of the free ones in rows and columns), a leading fixed run
  // is merged into dim 0 as well, its value selected by the dim-0
  // coordinate (an even number of doubles, so 16-byte aligned) with a box
  // of one element
  int first = 0;
  bool first_fixed = false;
  if (!runs.empty() && runs[0].start == 0) {
    if (runs[0].free) {
      first = 1;
    } else if (1 + (int)runs.size() > 5) {
      first = 1;
      first_fixed = true;
    }
  }
  const int ndims = 1 + (int)runs.size() - first;
  if (ndims > 5) return false;
  pp.tstart[0] = 0;
  pp.tlen[0] = first ? runs[0].len : 0;
  pp.tfree[0] = first_fixed ? 0 : 1;
  int d = 1;
  for (size_t k = first; k < runs.size(); k++, d++) {
    pp.tstart[d] = runs[k].start;
    pp.tlen[d] = runs[k].len;
    pp.tfree[d] = runs[k].free ? 1 : 0;
  }
  for (; d < 5; d++) {  // padding dims of size one
    pp.tstart[d] = 2 * n;
    pp.tlen[d] = 0;
    pp.tfree[d] = 1;
  }
  return true;
}

void encode_tma(const PassParams &pp, const double2 *x, CUtensorMap *map) {
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  dims[0] = 2ull << pp.tlen[0];
  box[0] = pp.tfree[0] ? (2u << pp.tlen[0]) : 2u;
  for (int d = 1; d < 5; d++) {
    dims[d] = 1ull << pp.tlen[d];
    box[d] = pp.tfree[d] ? (1u << pp.tlen[d]) : 1u;
    strides[d - 1] = 16ull << pp.tstart[d];
  }
  CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, (void *)x, dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(9, "ERROR! cuTensorMapEncodeTiled failed (%d)\n", (int)r);
}

template <bool REAL, bool TMA, int CANON, bool F32>
void launch_pass(const PassParams &pp, const CUtensorMap &map, const CUtensorMap &bmap, const double2 *x,
                 const Epi &e, int grid, size_t smem, cudaStream_t s, bool dry) {
  ensure_smem((const void *)k_qpass<REAL, TMA, CANON, F32>, smem);
  if (dry) {
    cudaFuncAttributes fa;
    QCUDA(cudaFuncGetAttributes(&fa, (const void *)k_qpass<REAL, TMA, CANON, F32>));
    return;
  }
  k_qpass<REAL, TMA, CANON, F32><<<grid, QT, smem, s>>>(pp, map, bmap, x, e);
}

template <bool TMA, bool F32>
struct Canon {
  template <int CANON>
  static void launch(const PassParams &pp, const CUtensorMap &map, const CUtensorMap &bmap, const double2 *x,
                     const Epi &e, int grid, size_t smem, cudaStream_t s, bool dry) {
    launch_pass<true, TMA, CANON, F32>(pp, map, bmap, x, e, grid, smem, s, dry);
  }
};

// canonical fast path: real mode, no general terms in this pass
template <bool TMA, bool F32>
void launch_canon_mask(int mask, const PassParams &pp, const CUtensorMap &map, const CUtensorMap &bmap,
                       const double2 *x, const Epi &e, int grid, size_t smem, cudaStream_t s, bool dry) {
#define launch_canon Canon<TMA, F32>::template launch
  switch (mask) {
    case 0: launch_canon<0>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 1: launch_canon<1>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 2: launch_canon<2>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 3: launch_canon<3>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 4: launch_canon<4>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 5: launch_canon<5>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 6: launch_canon<6>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 7: launch_canon<7>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 8: launch_canon<8>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 9: launch_canon<9>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 10: launch_canon<10>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 11: launch_canon<11>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 12: launch_canon<12>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 13: launch_canon<13>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    case 14: launch_canon<14>(pp, map, bmap, x, e, grid, smem, s, dry); break;
    default: launch_canon<15>(pp, map, bmap, x, e, grid, smem, s, dry); break;
  }
#undef launch_canon
}

int canon_mask(const PassParams &pp) {
  int m = 0;
  for (int b = 0; b < 6; b++) {
    if (pp.hl[b] != 0) m |= 1;
    if (pp.hr[b] != 0) m |= 2;
    if (pp.gl[b] != 0) m |= 4;
    if (pp.gu[b] != 0) m |= 8;
  }
  return m;
}

template <bool F32>
void launch_any_pass(const PassParams &pp, const CUtensorMap &map, const CUtensorMap &bmap, const double2 *x,
                     const Epi &e, int grid, size_t smem, cudaStream_t s, bool dry) {
  const bool tma = pp.tma != 0;
  const bool only_canon = pp.real && pp.nL == 0 && pp.nR == 0 && pp.nJ == 0 && pp.nJx == 0 && pp.nspill == 0;
  if (only_canon && tma) launch_canon_mask<true, F32>(canon_mask(pp), pp, map, bmap, x, e, grid, smem, s, dry);
  else if (only_canon) launch_canon_mask<false, F32>(canon_mask(pp), pp, map, bmap, x, e, grid, smem, s, dry);
  else if (pp.real && tma) launch_pass<true, true, -1, F32>(pp, map, bmap, x, e, grid, smem, s, dry);
  else if (pp.real) launch_pass<true, false, -1, F32>(pp, map, bmap, x, e, grid, smem, s, dry);
  else if (tma) launch_pass<false, true, -1, F32>(pp, map, bmap, x, e, grid, smem, s, dry);
  else launch_pass<false, false, -1, F32>(pp, map, bmap, x, e, grid, smem, s, dry);
}

// A pass whose terms are canonical single-bit ones that map Hermitian
// inputs to Hermitian outputs (left and right X with opposite
// coefficients, real jumps): its tile (b, a) result is the conjugate
// transpose of its tile (a, b) result.
bool hermitian_canonical_pass(const PassParams &pp) {
  if (!(pp.real && pp.nL == 0 && pp.nR == 0 && pp.nJ == 0 && pp.nJx == 0 && pp.nspill == 0 && !pp.diag))
    return false;
  for (int b = 0; b < 6; b++)
    if (pp.hl[b] != -pp.hr[b]) return false;
  return true;
}

size_t pass_smem(const PassParams &pp) {
  return (size_t)((pp.tma ? 3 : 2) * NEL + QMAX_GROUPS * 64) * sizeof(double2);
}

}  // namespace


// Splits a compiled qubit program into passes.  Returns false if the
// system does not suit the multi-pass kernel (n < 7 or too many terms).
bool plan_qubit_passes(const DeviceProgram &P, std::vector<PassParams> &out) {
  const QubitProg &Q = P.qdev;
  const int n = Q.n;
  if (n < 7 || n > 16) return false;
  // groups of six bit positions; the last may overlap its neighbour
  std::vector<int> los;
  for (int lo = 0; lo < n; lo += 6) los.push_back(std::min(lo, n - 6));
  const int ng = (int)los.size();
  std::vector<std::vector<PassTerm>> L(ng), R(ng), J(ng);
  std::vector<PassTerm> Jx, spill;
  std::vector<std::array<double, 24>> canon(ng);
  for (auto &cv : canon) cv.fill(0.0);
  auto group_of = [&](uint32_t f) -> int {
    for (int p = 0; p < ng; p++) {
      const uint32_t gm = 0x3fu << los[p];
      if ((f & ~gm) == 0) return p;
    }
    return -1;
  };
  auto mk = [&](const QTerm &q, uint32_t fl) {
    PassTerm t;
    t.fl = fl;
    t.cmask = q.cmask;
    t.cval = q.cval;
    t.smask = q.smask;
    t.coef = q.coef;
    return t;
  };
  const bool real = Q.real != 0;
  const auto &qt = P.qterms;
  size_t k = 0;
  for (int kind = 0; kind < 4; kind++) {
    const int cnt = kind == 0 ? Q.nL : kind == 1 ? Q.nR : kind == 2 ? Q.nJ : Q.nJx;
    for (int j = 0; j < cnt; j++, k++) {
      const QTerm &q = qt[k];
      if (kind == 3) { Jx.push_back(mk(q, 0)); continue; }
      const int p = group_of(q.fmask);
      if (p < 0) {
        spill.push_back(mk(q, q.fmask | ((uint32_t)kind << 29)));
        continue;
      }
      const uint32_t fl = q.fmask >> los[p];
      if (real && __builtin_popcount(fl) == 1) {
        int b = 0;
        while ((1u << b) != fl) b++;
        if (kind < 2 && q.cmask == 0 && q.smask == 0) {
          canon[p][kind * 6 + b] += q.coef.y;
          continue;
        }
        if (kind == 2 && q.cmask == q.fmask && q.smask == 0) {
          canon[p][(q.cval ? 18 : 12) + b] += q.coef.x;
          continue;
        }
      }
      (kind == 0 ? L : kind == 1 ? R : J)[p].push_back(mk(q, fl));
    }
  }
  // pass order: the high groups first, group 0 (contiguous rows, diagonal,
  // stage epilogue) last
  const long long ntiles = 1ll << (2 * n - 12);
  out.clear();
  for (int p = ng - 1; p >= 0; p--) {
    PassParams pp;
    memset(&pp, 0, sizeof(pp));
    pp.n = n;
    pp.lo = los[p];
    pp.diag = p == 0;
    pp.last = p == 0;
    pp.real = Q.real;
    pp.ngroups = Q.ngroups;
    pp.ntiles = ntiles;
    pp.dr = Q.dr;
    pp.dc = Q.dc;
    pp.gtab = Q.gtab;
    for (int b = 0; b < 6; b++) {
      pp.hl[b] = canon[p][b];
      pp.hr[b] = canon[p][6 + b];
      pp.gl[b] = canon[p][12 + b];
      pp.gu[b] = canon[p][18 + b];
      if (pp.hl[b] != 0 || pp.hr[b] != 0 || pp.gl[b] != 0 || pp.gu[b] != 0) pp.ncanon = 1;
    }
    std::vector<PassTerm> all;
    all.insert(all.end(), L[p].begin(), L[p].end());
    all.insert(all.end(), R[p].begin(), R[p].end());
    all.insert(all.end(), J[p].begin(), J[p].end());
    pp.nL = (int)L[p].size();
    pp.nR = (int)R[p].size();
    pp.nJ = (int)J[p].size();
    if (p == 0) {
      all.insert(all.end(), Jx.begin(), Jx.end());
      pp.nJx = (int)Jx.size();
      all.insert(all.end(), spill.begin(), spill.end());
      pp.nspill = (int)spill.size();
    }
    if (all.size() > (size_t)MAXPT) return false;
    for (size_t i = 0; i < all.size(); i++) pp.t[i] = all[i];
    pp.tma = describe_tma(pp) ? 1 : 0;
    pp.errflag = P.errflag;
    pp.claim = P.tile_claim;
    pp.done = P.tile_done;
    out.push_back(pp);
  }
  return true;
}

bool check_program_error(DeviceProgram &P, cudaStream_t s) {
  if (!P.errflag) return true;
  int h = 0;
  QCUDA(cudaMemcpyAsync(&h, P.errflag, sizeof(int), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  if (h) {
    // error word and tile-queue words start again from zero
    QCUDA(cudaMemsetAsync(P.errflag, 0, 16, s));
    QCUDA(cudaStreamSynchronize(s));
    fail(9, "ERROR! a tile load did not complete within its time limit; results are invalid\n");
    return false;
  }
  return true;
}

// Runs the passes; `scratch` holds D^2 complex values when there are at
// least two passes.
static std::atomic<int64_t> g_herm_applications{0};

void launch_qubit_passes(std::vector<PassParams> &passes, const double2 *x, double2 *scratch,
                         const Epi &e, cudaStream_t s, bool f32) {
  const int np = (int)passes.size();
  const int n = passes[0].n;
  // Hermitian mode: the last pass (low group) works on the blocks I <= J of
  // the bits above it and mirrors them; a two-pass program whose first pass
  // is a Hermitian canonical pass over the top six bits runs that pass on
  // tile pairs
  const bool herm = e.herm && passes.back().lo == 0 && passes.back().last;
  const bool pair = herm && np == 2 && passes[0].lo + 6 == n && hermitian_canonical_pass(passes[0]);
  if (herm) g_herm_applications++;
  const long long T = 1ll << (n - 6);
  for (int p = 0; p < np; p++) {
    PassParams &pp = passes[p];
    pp.accin = p > 0 ? scratch : nullptr;
    pp.accout = (p < np - 1) ? scratch : nullptr;
    const long long ntiles_full = pp.ntiles;
    if (herm && p == np - 1) {
      pp.herm_tiles = 1;
      pp.ntiles = T * (T + 1) / 2;
    }
    if (pair && p == 0) {
      pp.pair_tiles = 1;
      pp.ntiles = T * (T + 1) / 2;
    }
    CUtensorMap map, bmap;
    memset(&map, 0, sizeof(map));
    memset(&bmap, 0, sizeof(bmap));
    if (pp.tma) encode_tma(pp, x, &map);
    // the kernel loads the first stage base by TMA in a last pass with TMA
    if (pp.tma && pp.last && e.nupd > 0 && e.base[0]) encode_tma(pp, e.base[0], &bmap);
    // a middle pass with TMA reads its running sum through bmap (complex128)
    if (pp.tma && !pp.last && pp.accin && !f32) encode_tma(pp, pp.accin, &bmap);
    const int g = (int)std::min<long long>(pp.ntiles, num_sms());
    if (f32) launch_any_pass<true>(pp, map, bmap, x, e, g, pass_smem(pp), s, false);
    else launch_any_pass<false>(pp, map, bmap, x, e, g, pass_smem(pp), s, false);
    pp.herm_tiles = 0;
    pp.pair_tiles = 0;
    pp.ntiles = ntiles_full;
    count_launch();
    QCUDA(cudaGetLastError());
  }
}

void preload_lrho_kernels(const DeviceProgram &P) {
  if (P.has_qubit && !P.passes.empty()) {
    CUtensorMap map;
    memset(&map, 0, sizeof(map));
    Epi e;
    zero_epi(e);
    for (const PassParams &pp : P.passes) {
      launch_any_pass<false>(pp, map, map, nullptr, e, 1, pass_smem(pp), 0, true);
      launch_any_pass<true>(pp, map, map, nullptr, e, 1, pass_smem(pp), 0, true);
    }
  } else if (P.has_qubit) {
    preload_single_pass_qubit_kernels();
  } else {
    preload_generic_lrho_kernels();
  }
}

}  // namespace quac

// Number of L.x applications that ran in Hermitian mode (diagnostics).
extern "C" int64_t quac_hermitian_apply_count(void) { return quac::g_herm_applications.load(); }
