// Qubit-path compiler: recognises systems made only of two-level subsystems
// and rewrites every term as bit masks (see QTerm in common.h).
//
// Per qubit, a product of QuaC basic operators (kron.c:294-538 restricted to
// two levels) is a partial injection of {0,1}: identity, flip, a condition
// on the bit (one surviving row), or zero, with values whose ratio is +-1
// when both rows survive (Pauli products).  Qubit q = subsystem q sits at
// bit n-1-q of the Hilbert index (subsystem 0 is the most significant
// digit, kron.c:308).
#include <cmath>

#include "runtime.h"

namespace quac {

namespace {

struct QFactor {
  int m[2];     // row -> column map, -1 = empty row
  cplx v[2];
};

// two-level basic operator (the two-level case of kron.c:294-538)
bool basic2(op_handle o, QFactor &f) {
  f.m[0] = f.m[1] = -1;
  f.v[0] = f.v[1] = 0.0;
  switch (o->my_op_type) {
    case LOWER: f.m[0] = 1; f.v[0] = 1.0; break;
    case RAISE: f.m[1] = 0; f.v[1] = 1.0; break;
    case SIGMA_X: f.m[0] = 1; f.v[0] = 1.0; f.m[1] = 0; f.v[1] = 1.0; break;
    case SIGMA_Y: f.m[0] = 1; f.v[0] = cplx(0, -1); f.m[1] = 0; f.v[1] = cplx(0, 1); break;
    case NUMBER: f.m[1] = 1; f.v[1] = 1.0; break;
    case IDENTITY: f.m[0] = 0; f.v[0] = 1.0; f.m[1] = 1; f.v[1] = 1.0; break;
    case SIGMA_Z: f.m[0] = 0; f.v[0] = 1.0; f.m[1] = 1; f.v[1] = -1.0; break;
    case OTHER: break;
    default: return false;
  }
  return true;
}

int qubit_index(qsystem qs, op_handle o) {
  int64_t nb = o->n_before;
  int s = 0;
  while ((int64_t(1) << s) < nb) s++;
  if ((int64_t(1) << s) != nb || s >= qs->num_subsystems) return -1;
  return s;
}

struct Masks {
  uint32_t f = 0, cm = 0, cv = 0, sm = 0;
  cplx coef = 1.0;
  bool zero = false;
};

// Composes the op chain per qubit and reduces it to masks.
bool term_masks(qsystem qs, const Term &t, Masks &M) {
  const int n = (int)qs->num_subsystems;
  std::vector<QFactor> fac(n);
  std::vector<bool> touched(n, false);
  for (int q = 0; q < n; q++) {
    fac[q].m[0] = 0; fac[q].m[1] = 1; fac[q].v[0] = 1.0; fac[q].v[1] = 1.0;
  }
  for (size_t k = 0; k < t.ops.size(); k++) {
    op_handle o = t.ops[k];
    QFactor b;
    if (o->my_op_type == VEC) {
      if (k + 1 >= t.ops.size()) return false;
      op_handle o2 = t.ops[k + 1];
      b.m[0] = b.m[1] = -1;
      b.v[0] = b.v[1] = 0.0;
      if (o->position < 0 || o->position > 1 || o2->position < 0 || o2->position > 1) return false;
      b.m[o->position] = (int)o2->position;
      b.v[o->position] = 1.0;
      k++;
    } else if (!basic2(o, b)) {
      return false;
    }
    int q = qubit_index(qs, o);
    if (q < 0) return false;
    touched[q] = true;
    QFactor &f = fac[q];
    for (int d = 0; d < 2; d++) {
      if (f.m[d] < 0) continue;
      int e = f.m[d];
      if (b.m[e] < 0) { f.m[d] = -1; f.v[d] = 0.0; }
      else { f.m[d] = b.m[e]; f.v[d] = f.v[d] * b.v[e]; }
    }
  }
  for (int q = 0; q < n; q++) {
    if (!touched[q]) continue;
    const uint32_t bit = 1u << (n - 1 - q);
    QFactor &f = fac[q];
    if (f.m[0] < 0 && f.m[1] < 0) { M.zero = true; return true; }
    const bool flip = (f.m[0] == 1) || (f.m[1] == 0);
    if (flip) M.f |= bit;
    if (f.m[0] >= 0 && f.m[1] >= 0) {
      const cplx ratio = f.v[1] / f.v[0];
      if (std::abs(ratio - 1.0) < 1e-15) { M.coef *= f.v[0]; }
      else if (std::abs(ratio + 1.0) < 1e-15) { M.coef *= f.v[0]; M.sm |= bit; }
      else return false;
    } else {
      const int d = f.m[0] >= 0 ? 0 : 1;
      M.cm |= bit;
      if (d) M.cv |= bit;
      M.coef *= f.v[d];
    }
  }
  return true;
}

}  // namespace

bool compile_qubit(qsystem qs, const HostProg &hp, DeviceProgram *P) {
  const int n = (int)qs->num_subsystems;
  if (n < 6 || n > 24 || hp.ncols == 1) return false;
  for (int s = 0; s < n; s++)
    if (qs->subsystem_list[s]->my_levels != 2) return false;
  const cplx I(0, 1);
  std::vector<QTerm> L, R, J, Jx;
  // per-qubit single-qubit diagonal-jump tables T[q][br][bc]
  std::vector<cplx> T(n * 4, 0.0);
  bool real = true;
  auto push = [](std::vector<QTerm> &v, const Masks &M, cplx coef) {
    QTerm q;
    q.fmask = M.f; q.cmask = M.cm; q.cval = M.cv; q.smask = M.sm;
    q.coef = make_double2(coef.real(), coef.imag());
    v.push_back(q);
  };
  for (auto &t : qs->impl->terms) {
    if (t.a == cplx(0.0, 0.0)) continue;
    Masks M;
    if (!term_masks(qs, t, M)) return false;
    if (M.zero) continue;
    if (t.kind == 1) {
      if (M.f == 0) continue;  // diagonal: already folded into dr / dc
      const cplx wl = -I * t.a * M.coef;
      push(L, M, wl);
      // right action: partner c ^ f, condition on c ^ f
      Masks Mr = M;
      Mr.cv = M.cv ^ (M.f & M.cm);
      const double sgn = (__builtin_popcount(M.f & M.sm) & 1) ? -1.0 : 1.0;
      const cplx wr = I * t.a * M.coef * sgn;
      push(R, Mr, wr);
      if (std::abs(wl.real()) > 0 || std::abs(wr.real()) > 0) real = false;
    } else {
      const cplx w = t.a * std::norm(M.coef);
      if (std::abs(w.imag()) > 0) real = false;
      if (M.f == 0) {
        const int nb = __builtin_popcount(M.cm | M.sm);
        if (nb == 1) {
          const uint32_t bit = M.cm | M.sm;
          int b = 0;
          while ((1u << b) != bit) b++;
          const int q = n - 1 - b;
          for (int br = 0; br < 2; br++)
            for (int bc = 0; bc < 2; bc++) {
              auto ok = [&](int x) { return !(M.cm & bit) || ((x ? bit : 0u) == (M.cv & bit)); };
              if (!ok(br) || !ok(bc)) continue;
              double s = 1.0;
              if ((M.sm & bit) && br) s = -s;
              if ((M.sm & bit) && bc) s = -s;
              T[q * 4 + br * 2 + bc] += w * s;
            }
        } else {
          push(Jx, M, w);
        }
      } else {
        push(J, M, w);
      }
    }
  }
  const size_t total = L.size() + R.size() + J.size() + Jx.size();
  if (total > (size_t)QMAX_TERMS) return false;
  // group tables over bits [3g, 3g+3)
  const int ng = (n + 2) / 3;
  if (ng > QMAX_GROUPS) return false;
  std::vector<double2> g(ng * 64, make_double2(0, 0));
  for (int gi = 0; gi < ng; gi++)
    for (int rb = 0; rb < 8; rb++)
      for (int cb = 0; cb < 8; cb++) {
        cplx s = 0.0;
        for (int k = 0; k < 3; k++) {
          const int bit = 3 * gi + k;
          if (bit >= n) continue;
          const int q = n - 1 - bit;
          s += T[q * 4 + ((rb >> k) & 1) * 2 + ((cb >> k) & 1)];
        }
        g[gi * 64 + rb * 8 + cb] = make_double2(s.real(), s.imag());
      }
  P->qterms.clear();
  P->qterms.insert(P->qterms.end(), L.begin(), L.end());
  P->qterms.insert(P->qterms.end(), R.begin(), R.end());
  P->qterms.insert(P->qterms.end(), J.begin(), J.end());
  P->qterms.insert(P->qterms.end(), Jx.begin(), Jx.end());
  QubitProg &Q = P->qdev;
  Q.n = n;
  Q.nL = (int)L.size();
  Q.nR = (int)R.size();
  Q.nJ = (int)J.size();
  Q.nJx = (int)Jx.size();
  Q.real = real ? 1 : 0;
  Q.ngroups = ng;
  Q.dr = P->dev.dr;
  Q.dc = P->dev.dc;
  double2 *gd = nullptr;
  QCUDA(cudaMalloc(&gd, g.size() * sizeof(double2)));
  QCUDA(cudaMemcpy(gd, g.data(), g.size() * sizeof(double2), cudaMemcpyHostToDevice));
  P->allocations.push_back(gd);
  Q.gtab = gd;
  P->has_qubit = true;
  return true;
}

}  // namespace quac
