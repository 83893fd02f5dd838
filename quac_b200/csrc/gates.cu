// Gates on a state: rho <- U rho W^T on selected binary digits of the
// column-stacked vector, in one pass over the affected element groups.
//
// Both reference engines reduce to this form:
//  - the superoperator engine (_apply_gate_sys, quantum_circuits.c:435-481)
//    builds U* (x) U with qubit q = subsystem q (digit stride n_after), i.e.
//    W = conj(U) on the column digit;
//  - the in-place engine (_apply_gate2, quantum_circuits.c:696-772) runs a
//    state-vector kernel on the row digits, then again (conjugated, except
//    RZ, quantum_circuits.c:2114-2147) on the column digits.
// The caller passes the strides of the digits inside the flat vector index
// (a column digit of stride s has vector stride D*s) and the row / column
// matrices in the kernel's basis: index = 2*d(first digit) + d(second).
#include "common.h"

namespace quac {

namespace {

constexpr int NT = 256;

struct Mat4 {
  double2 m[8];
};
struct Mat32 {
  double2 m[32];
};

__device__ __forceinline__ double2 cmulg(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ int64_t insert0(int64_t t, int64_t s) {
  return (t / s) * 2 * s + (t % s);
}

// One row digit (stride sr) and optionally one column digit (stride sc > sr).
__global__ void k_gate1(double2 *__restrict__ a, int64_t nquads, int64_t sr, int64_t sc,
                        const Mat4 UW) {
  const int64_t t = (int64_t)blockIdx.x * NT + threadIdx.x;
  if (t >= nquads) return;
  const double2 *U = UW.m, *W = UW.m + 4;
  if (sc == 0) {
    const int64_t i0 = insert0(t, sr), i1 = i0 + sr;
    const double2 x0 = a[i0], x1 = a[i1];
    double2 y0 = cmulg(U[0], x0), y1 = cmulg(U[2], x0);
    const double2 p = cmulg(U[1], x1), q = cmulg(U[3], x1);
    y0.x += p.x; y0.y += p.y; y1.x += q.x; y1.y += q.y;
    a[i0] = y0; a[i1] = y1;
    return;
  }
  const int64_t i00 = insert0(insert0(t, sr), sc);
  const int64_t idx[4] = {i00, i00 + sr, i00 + sc, i00 + sr + sc};
  double2 x[4];
#pragma unroll
  for (int k = 0; k < 4; k++) x[k] = a[idx[k]];
  // element (ra, cb) at idx[ra + 2 cb]; new = sum U[ra,ra'] W[cb,cb'] x
#pragma unroll
  for (int cb = 0; cb < 2; cb++) {
#pragma unroll
    for (int ra = 0; ra < 2; ra++) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int cb2 = 0; cb2 < 2; cb2++) {
#pragma unroll
        for (int ra2 = 0; ra2 < 2; ra2++) {
          const double2 f = cmulg(U[ra * 2 + ra2], W[cb * 2 + cb2]);
          const double2 v = cmulg(f, x[ra2 + 2 * cb2]);
          acc.x += v.x; acc.y += v.y;
        }
      }
      a[idx[ra + 2 * cb]] = acc;
    }
  }
}

// Two row digits (strides r0, r1) and optionally two column digits.
struct Gate2Args {
  int64_t s[4];      // strides: row A, row B, col A, col B (cols 0 if absent)
  int64_t sorted[4];
  int nsort;
};

__global__ void k_gate2(double2 *__restrict__ a, int64_t ngroups, const Gate2Args G,
                        const Mat32 UW) {
  const int64_t t = (int64_t)blockIdx.x * NT + threadIdx.x;
  if (t >= ngroups) return;
  int64_t base = t;
  for (int k = 0; k < G.nsort; k++) base = insert0(base, G.sorted[k]);
  const double2 *U = UW.m, *W = UW.m + 16;
  if (G.s[2] == 0) {
    double2 x[4];
    int64_t idx[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      idx[k] = base + ((k >> 1) & 1) * G.s[0] + (k & 1) * G.s[1];
      x[k] = a[idx[k]];
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const double2 v = cmulg(U[r * 4 + c], x[c]);
        acc.x += v.x; acc.y += v.y;
      }
      a[idx[r]] = acc;
    }
    return;
  }
  double2 x[16];
  int64_t idx[16];
#pragma unroll
  for (int k = 0; k < 16; k++) {
    const int ri = k & 3, ci = k >> 2;
    idx[k] = base + ((ri >> 1) & 1) * G.s[0] + (ri & 1) * G.s[1] + ((ci >> 1) & 1) * G.s[2] +
             (ci & 1) * G.s[3];
    x[k] = a[idx[k]];
  }
  // rows first: y[ri,ci] = sum_ri' U[ri,ri'] x[ri',ci]
  double2 y[16];
#pragma unroll
  for (int ci = 0; ci < 4; ci++) {
#pragma unroll
    for (int ri = 0; ri < 4; ri++) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int r2 = 0; r2 < 4; r2++) {
        const double2 v = cmulg(U[ri * 4 + r2], x[r2 + 4 * ci]);
        acc.x += v.x; acc.y += v.y;
      }
      y[ri + 4 * ci] = acc;
    }
  }
#pragma unroll
  for (int ci = 0; ci < 4; ci++) {
#pragma unroll
    for (int ri = 0; ri < 4; ri++) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int c2 = 0; c2 < 4; c2++) {
        const double2 v = cmulg(W[ci * 4 + c2], y[ri + 4 * c2]);
        acc.x += v.x; acc.y += v.y;
      }
      a[idx[ri + 4 * ci]] = acc;
    }
  }
}

}  // namespace

// Applies U on the row digit of stride sr and W on the column digit of
// vector stride sc (sc = 0: no column part).  U, W row-major 2x2.
void launch_gate1(double2 *a, int64_t n, int64_t sr, int64_t sc, const cplx *U, const cplx *W,
                  cudaStream_t s) {
  Mat4 m;
  for (int k = 0; k < 4; k++) {
    m.m[k] = make_double2(U[k].real(), U[k].imag());
    m.m[4 + k] = W ? make_double2(W[k].real(), W[k].imag()) : make_double2(0, 0);
  }
  // every digit must be a binary digit of the index space: the group
  // enumeration below then stays inside [0, n)
  if (sr < 1 || n % (2 * sr) != 0 || (sc && (sc % (2 * sr) != 0 || n % (2 * sc) != 0))) {
    fail(0, "ERROR! gate digit strides (%ld, %ld) do not address binary digits of a %ld-vector\n",
         (long)sr, (long)sc, (long)n);
    return;
  }
  const int64_t nq = sc ? n / 4 : n / 2;
  if (nq <= 0) return;
  k_gate1<<<(unsigned)((nq + NT - 1) / NT), NT, 0, s>>>(a, nq, sr, sc, m);
  count_launch();
  QCUDA(cudaGetLastError());
}

// Two-qubit form: strides {rowA, rowB, colA, colB} (cols 0 if absent),
// U / W row-major 4x4 in the basis 2*d(A) + d(B).
void launch_gate2(double2 *a, int64_t n, const int64_t strides[4], const cplx *U, const cplx *W,
                  cudaStream_t s) {
  Gate2Args G;
  int ns = 0;
  for (int k = 0; k < 4; k++) {
    G.s[k] = strides[k];
    if (strides[k] > 0) G.sorted[ns++] = strides[k];
  }
  for (int i = 1; i < ns; i++)
    for (int j = i; j > 0 && G.sorted[j] < G.sorted[j - 1]; j--) std::swap(G.sorted[j], G.sorted[j - 1]);
  G.nsort = ns;
  bool ok = ns >= 2 && G.sorted[0] >= 1 && n % (2 * G.sorted[ns - 1]) == 0;
  for (int k = 1; k < ns; k++) ok = ok && (G.sorted[k] % (2 * G.sorted[k - 1]) == 0);
  if (!ok) {
    fail(0, "ERROR! two-qubit gate digits are not distinct binary digits of the state\n");
    return;
  }
  Mat32 h;
  for (int k = 0; k < 16; k++) {
    h.m[k] = make_double2(U[k].real(), U[k].imag());
    h.m[16 + k] = W ? make_double2(W[k].real(), W[k].imag()) : make_double2(0, 0);
  }
  const int64_t ng = n >> ns;
  if (ng <= 0) return;
  k_gate2<<<(unsigned)((ng + NT - 1) / NT), NT, 0, s>>>(a, ng, G, h);
  count_launch();
  QCUDA(cudaGetLastError());
}

}  // namespace quac
