// Multi-pass matrix-free L.x for qubit systems (n >= 7 qubits).
//
// The 2n bits of the column-stacked index (row bits r_0..r_{n-1}, column
// bits c_0..c_{n-1}) are covered by groups of six bit positions [lo, lo+6),
// applied to rows and columns alike.  Pass p owns 64 x 64 tiles whose free
// bits are group p for rows and columns; every term whose flip mask lies in
// group p (left: row flips, right: column flips, jumps: both) finds its
// partners inside the tile.  Pass 0 also applies the diagonal.  Passes
// accumulate into a scratch vector; the last one runs the fused stage
// epilogue.  A CTA is persistent (one per SM) and streams tiles through two
// shared-memory buffers filled by cp.async, so the next tile's loads overlap
// the current tile's arithmetic.
//
// Consecutive work items differ in the lowest fixed row bit, so in passes
// whose tiles have single-element rows the two halves of every 32-byte
// sector are requested by neighbouring CTAs at the same time.
#include <algorithm>
#include <array>
#include <cstring>

#include "common.h"

namespace quac {

namespace {

constexpr int PT = 512;            // threads per CTA (16 warps)
constexpr int TILE = 64;           // tile rows = tile columns
constexpr int NEL = TILE * TILE;   // elements per tile
__device__ __forceinline__ void cfma2(double2 &acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double cabs2d(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// fixed (non-tile) bits of a work item: rows then columns
__device__ __forceinline__ void tile_origin(long long t, int n, int lo, unsigned &rfix, unsigned &cfix) {
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
                                          int n, int lo) {
  unsigned rfix, cfix;
  tile_origin(t, n, lo, rfix, cfix);
  const size_t D = (size_t)1 << n;
  for (int e = threadIdx.x; e < NEL; e += PT) {
    const unsigned cl = e >> 6, rl = e & 63;
    const size_t r = rfix | (rl << lo), c = cfix | (cl << lo);
    cp_async16(buf + e, X + c * D + r);
  }
}

template <bool REAL>
__global__ void __launch_bounds__(PT, 1) k_qpass(const __grid_constant__ PassParams P,
                                                 const double2 *__restrict__ X, const Epi E) {
  extern __shared__ double2 sm[];
  double2 *buf0 = sm, *buf1 = sm + NEL;
  double2 *gts = sm + 2 * NEL;                 // ngroups * 64, layout [g][col bits][row bits]
  __shared__ double red[PT / 32];
  const int n = P.n, lo = P.lo;
  const size_t D = (size_t)1 << n;
  if (P.diag)
    for (int i = threadIdx.x; i < P.ngroups * 64; i += PT) {
      const int g = i >> 6, rb = (i >> 3) & 7, cb = i & 7;  // source layout [g][rb][cb]
      gts[(g << 6) | (cb << 3) | rb] = P.gtab[i];
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double nloc = 0.0;
  long long t = blockIdx.x;
  if (t < P.ntiles) load_tile(buf0, X, t, n, lo);
  cp_commit();
  for (int it = 0; t < P.ntiles; it++, t += gridDim.x) {
    const long long tn = t + gridDim.x;
    double2 *cur = (it & 1) ? buf1 : buf0;
    double2 *nxt = (it & 1) ? buf0 : buf1;
    if (tn < P.ntiles) load_tile(nxt, X, tn, n, lo);
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    unsigned rfix, cfix;
    tile_origin(t, n, lo, rfix, cfix);
    // thread elements: rows lane, lane+32; columns w, w+16, w+32, w+48
    unsigned rl[2] = {(unsigned)lane, (unsigned)lane + 32u};
    unsigned cl[4] = {(unsigned)w, (unsigned)w + 16u, (unsigned)w + 32u, (unsigned)w + 48u};
    unsigned r[2], c[4];
#pragma unroll
    for (int i = 0; i < 2; i++) r[i] = rfix | (rl[i] << lo);
#pragma unroll
    for (int m = 0; m < 4; m++) c[m] = cfix | (cl[m] << lo);
    double2 acc[2][4];
    if (P.accin) {
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < 4; m++) acc[i][m] = P.accin[(size_t)c[m] * D + r[i]];
    } else {
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int m = 0; m < 4; m++) acc[i][m] = make_double2(0.0, 0.0);
    }
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
        for (int m = 0; m < 4; m++) {
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
          cfma2(acc[i][m], d, cur[cl[m] * 64 + rl[i]]);
        }
      }
    }
    if (REAL && P.ncanon) {
      // canonical single-bit terms: partner offsets are compile-time constants
#pragma unroll
      for (int b = 0; b < 6; b++) {
        const unsigned f = 1u << b;
        const double hl = P.hl[b], hr = P.hr[b], gl = P.gl[b], gu = P.gu[b];
        if (hl != 0.0) {
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < 4; m++) {
              const double2 p = cur[cl[m] * 64 + (rl[i] ^ f)];
              acc[i][m].x = fma(-hl, p.y, acc[i][m].x);
              acc[i][m].y = fma(hl, p.x, acc[i][m].y);
            }
        }
        if (hr != 0.0) {
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < 4; m++) {
              const double2 p = cur[(cl[m] ^ f) * 64 + rl[i]];
              acc[i][m].x = fma(-hr, p.y, acc[i][m].x);
              acc[i][m].y = fma(hr, p.x, acc[i][m].y);
            }
        }
        if (gl != 0.0 || gu != 0.0) {
#pragma unroll
          for (int i = 0; i < 2; i++)
#pragma unroll
            for (int m = 0; m < 4; m++) {
              const bool rb = rl[i] & f, cb = cl[m] & f;
              if (rb == cb) {
                const double g = rb ? gu : gl;
                const double2 p = cur[(cl[m] ^ f) * 64 + (rl[i] ^ f)];
                acc[i][m].x = fma(g, p.x, acc[i][m].x);
                acc[i][m].y = fma(g, p.y, acc[i][m].y);
              }
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
          const double wv = neg ? -T.coef.y : T.coef.y;
#pragma unroll
          for (int m = 0; m < 4; m++) {
            const double2 p = cur[cl[m] * 64 + pr];
            acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
            acc[i][m].y = fma(wv, p.x, acc[i][m].y);
          }
        } else {
          const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
#pragma unroll
          for (int m = 0; m < 4; m++) cfma2(acc[i][m], wv, cur[cl[m] * 64 + pr]);
        }
      }
    }
    for (int e = k + P.nR; k < e; k++) {
      const PassTerm T = P.t[k];
#pragma unroll
      for (int m = 0; m < 4; m++) {
        if ((c[m] & T.cmask) != T.cval) continue;
        const bool neg = __popc(c[m] & T.smask) & 1;
        const unsigned pc = cl[m] ^ T.fl;
        if (REAL) {
          const double wv = neg ? -T.coef.y : T.coef.y;
#pragma unroll
          for (int i = 0; i < 2; i++) {
            const double2 p = cur[pc * 64 + rl[i]];
            acc[i][m].x = fma(-wv, p.y, acc[i][m].x);
            acc[i][m].y = fma(wv, p.x, acc[i][m].y);
          }
        } else {
          const double2 wv = neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef;
#pragma unroll
          for (int i = 0; i < 2; i++) cfma2(acc[i][m], wv, cur[pc * 64 + rl[i]]);
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
        for (int m = 0; m < 4; m++) {
          if ((c[m] & T.cmask) != T.cval) continue;
          const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
          const double2 p = cur[(cl[m] ^ T.fl) * 64 + pr];
          if (REAL) {
            const double wv = neg ? -T.coef.x : T.coef.x;
            acc[i][m].x = fma(wv, p.x, acc[i][m].x);
            acc[i][m].y = fma(wv, p.y, acc[i][m].y);
          } else {
            cfma2(acc[i][m], neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef, p);
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
        for (int m = 0; m < 4; m++) {
          if ((c[m] & T.cmask) != T.cval) continue;
          const bool neg = (sr + __popc(c[m] & T.smask)) & 1;
          cfma2(acc[i][m], neg ? make_double2(-T.coef.x, -T.coef.y) : T.coef, cur[cl[m] * 64 + rl[i]]);
        }
      }
    }
    // cross-group terms (flip bits in two groups): global loads.  Stored
    // after the pass's own terms with fl holding the full flip mask and the
    // kind in cval's top bits is not needed: kind order L, R, J.
    for (int s = 0; s < P.nspill; s++, k++) {
      const PassTerm T = P.t[k];
      const int kind = (int)(T.fl >> 29);
      const unsigned f = T.fl & 0x1fffffffu;
#pragma unroll
      for (int i = 0; i < 2; i++) {
#pragma unroll
        for (int m = 0; m < 4; m++) {
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
          cfma2(acc[i][m], (sg & 1) ? make_double2(-T.coef.x, -T.coef.y) : T.coef, __ldg(X + pidx));
        }
      }
    }
    // outputs
#pragma unroll
    for (int i = 0; i < 2; i++) {
#pragma unroll
      for (int m = 0; m < 4; m++) {
        const size_t idx = (size_t)c[m] * D + r[i];
        const double2 Kv = acc[i][m];
        if (!P.last) {
          P.accout[idx] = Kv;
          continue;
        }
        if (E.kout) E.kout[idx] = Kv;
        double2 u0 = make_double2(0.0, 0.0), u1 = u0, u2 = u0;
        if (E.nupd > 0) {
          double2 b = E.base[0] ? E.base[0][idx] : make_double2(0.0, 0.0);
          u0 = make_double2(fma(E.coef[0], Kv.x, b.x), fma(E.coef[0], Kv.y, b.y));
          E.out[0][idx] = u0;
        }
        if (E.nupd > 1) {
          double2 b = E.base[1] ? E.base[1][idx] : make_double2(0.0, 0.0);
          u1 = make_double2(fma(E.coef[1], Kv.x, b.x), fma(E.coef[1], Kv.y, b.y));
          E.out[1][idx] = u1;
        }
        if (E.nupd > 2) {
          double2 b = E.base[2] ? E.base[2][idx] : make_double2(0.0, 0.0);
          u2 = make_double2(fma(E.coef[2], Kv.x, b.x), fma(E.coef[2], Kv.y, b.y));
          E.out[2][idx] = u2;
        }
        if (E.nsum) {
          const double2 ev = E.err_upd == 0 ? u0 : (E.err_upd == 1 ? u1 : u2);
          const double2 y = E.ny[idx];
          const double2 yn = E.yn_upd == 0 ? u0 : (E.yn_upd == 1 ? u1 : (E.yn_upd == 2 ? u2 : E.nyn[idx]));
          const double q = cabs2d(ev) / (E.atol + E.rtol * fmax(cabs2d(y), cabs2d(yn)));
          nloc += q * q;
        }
      }
    }
    __syncthreads();  // cur is refilled two iterations later
  }
  cp_wait<0>();
  if (P.last && E.nsum) {
    for (int o = 16; o > 0; o >>= 1) nloc += __shfl_down_sync(0xffffffffu, nloc, o);
    if (lane == 0) red[w] = nloc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int q = 0; q < PT / 32; q++) s += red[q];
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
    out.push_back(pp);
  }
  return true;
}

// Runs the passes; `scratch` holds D^2 complex values when there are at
// least two passes.
void launch_qubit_passes(std::vector<PassParams> &passes, const double2 *x, double2 *scratch,
                         const Epi &e, cudaStream_t s) {
  const int np = (int)passes.size();
  const size_t smem = (size_t)(2 * NEL + QMAX_GROUPS * 64) * sizeof(double2);
  static bool attr = false;
  if (!attr) {
    QCUDA(cudaFuncSetAttribute(k_qpass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    QCUDA(cudaFuncSetAttribute(k_qpass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const long long nt = passes[0].ntiles;
  const int grid = (int)std::min<long long>(nt, num_sms());
  for (int p = 0; p < np; p++) {
    PassParams &pp = passes[p];
    pp.accin = p > 0 ? scratch : nullptr;
    pp.accout = (p < np - 1) ? scratch : nullptr;
    if (pp.real) k_qpass<true><<<grid, PT, smem, s>>>(pp, x, e);
    else k_qpass<false><<<grid, PT, smem, s>>>(pp, x, e);
    count_launch();
    QCUDA(cudaGetLastError());
  }
}

}  // namespace quac
