// Term compiler: turns the recorded add_ham_term / add_lin_term products
// into the per-row tables the matrix-free L.x kernels read.
//
// Every QuaC basic operator has at most one nonzero per row and per column
// (kron.c:62-155, 294-538), so a product of them is a partial injection
// G: r -> (j(r), v(r)).  The superoperator pieces of construct_matrix
// (qsystem.c:593-676 via kron.c:702-729 and 995-1036) then become
//   Hamiltonian a*G : left  -i a G x      (rows),
//                     right +i a x G      (columns; the complex-coefficient
//                     fixtures pin +i a, not the conj(a) written at kron.c:723),
//   Lindblad   a*C : a C x C^dag - a/2 (C^dag C x + x C^dag C),
// with C^dag C diagonal, so it folds into the per-row / per-column diagonal.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "runtime.h"

namespace quac {

static void single_op(int64_t D, int64_t i, op_handle op, int64_t &j, cplx &v) {
  const int64_t L = op->my_levels;
  const int64_t na = D / (L * op->n_before);
  const int64_t isub = (i / na) % L;
  const int64_t base = i - isub * na;
  j = -1;
  v = 0.0;
  switch (op->my_op_type) {
    case LOWER:
      if (isub < L - 1) { j = base + (isub + 1) * na; v = std::sqrt((double)isub + 1.0); }
      break;
    case RAISE:
      if (isub >= 1) { j = base + (isub - 1) * na; v = std::sqrt((double)isub); }
      break;
    case SIGMA_X:
      if (isub == 0) { j = base + na; v = 1.0; }
      else if (isub == 1) { j = base; v = 1.0; }
      break;
    case SIGMA_Y:
      if (isub == 0) { j = base + na; v = cplx(0, -1); }
      else if (isub == 1) { j = base; v = cplx(0, 1); }
      break;
    case NUMBER:
      if (isub != 0) { j = i; v = (double)isub; }
      break;
    case IDENTITY:
      j = i; v = 1.0;
      break;
    case SIGMA_Z:
      if (isub == 0) { j = i; v = 1.0; }
      else if (isub == 1) { j = i; v = -1.0; }
      break;
    case OTHER:
      if (isub >= 2) { j = i; v = 1.0; }
      break;
    default:
      break;
  }
}

static void vec_pair(int64_t D, int64_t i, op_handle a, op_handle b, int64_t &j, cplx &v) {
  const int64_t L = a->my_levels;
  const int64_t na = D / (L * a->n_before);
  const int64_t isub = (i / na) % L;
  if (isub == a->position) { j = i - isub * na + b->position * na; v = 1.0; }
  else { j = -1; v = 0.0; }
}

void op_chain_map(int64_t D, const std::vector<op_handle> &ops, std::vector<int> &map,
                  std::vector<cplx> &val) {
  map.assign(D, -1);
  val.assign(D, 0.0);
  for (size_t k = 0; k < ops.size(); k++) {
    if (ops[k]->my_op_type == VEC) {
      if (k + 1 >= ops.size() || ops[k + 1]->my_op_type != VEC)
        fail(0, "ERROR! VEC operators must come in pairs\n");
      if (ops[k]->n_before != ops[k + 1]->n_before)
        fail(0, "ERROR! Vec Operators must be from the same Hilbert subspace\n");
      k++;
    }
  }
  for (int64_t r = 0; r < D; r++) {
    int64_t j = r;
    cplx v = 1.0;
    for (size_t k = 0; k < ops.size() && j >= 0; k++) {
      int64_t j2;
      cplx t;
      if (ops[k]->my_op_type == VEC) {
        vec_pair(D, j, ops[k], ops[k + 1], j2, t);
        k++;
      } else {
        single_op(D, j, ops[k], j2, t);
      }
      j = j2;
      v = t * v;
    }
    if (j >= 0) { map[r] = (int)j; val[r] = v; }
  }
}

void DeviceProgram::release() {
  for (void *p : allocations) cudaFree(p);
  allocations.clear();
  scratch = nullptr;
  errflag = nullptr;
  tile_done = nullptr;
  tile_claim = nullptr;
}

namespace {

struct MapKey {
  size_t h;
};

size_t hash_map(const std::vector<int> &m) {
  size_t h = 1469598103934665603ull;
  for (int x : m) { h ^= (size_t)(uint32_t)x; h *= 1099511628211ull; }
  return h;
}

// Adds a (map, values) table to a list, merging with an identical map.
void add_table(std::vector<std::vector<int>> &maps, std::vector<std::vector<cplx>> &vals,
               std::vector<size_t> &hashes, const std::vector<int> &m,
               const std::vector<cplx> &v) {
  size_t h = hash_map(m);
  for (size_t t = 0; t < maps.size(); t++) {
    if (hashes[t] == h && maps[t] == m) {
      for (size_t r = 0; r < v.size(); r++) vals[t][r] += v[r];
      return;
    }
  }
  maps.push_back(m);
  vals.push_back(v);
  hashes.push_back(h);
}

template <typename T>
const T *upload(DeviceProgram *P, const std::vector<T> &h) {
  if (h.empty()) return nullptr;
  void *d = nullptr;
  QCUDA(cudaMalloc(&d, h.size() * sizeof(T)));
  QCUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  P->allocations.push_back(d);
  return (const T *)d;
}

template <typename T>
std::vector<T> flatten(const std::vector<std::vector<T>> &v) {
  std::vector<T> out;
  for (auto &x : v) out.insert(out.end(), x.begin(), x.end());
  return out;
}

std::vector<double2> to_d2(const std::vector<cplx> &v) {
  std::vector<double2> o(v.size());
  for (size_t i = 0; i < v.size(); i++) o[i] = make_double2(v[i].real(), v[i].imag());
  return o;
}

}  // namespace

// Host half of the compiler: fills hp from the recorded terms (no GPU use).
bool compile_host(qsystem qs, int mode, HostProg &hp) {
  const int64_t D = qs->total_levels;
  if (D > (1LL << 30)) { fail(9, "ERROR! Hilbert dimension too large for the device tables\n"); return false; }
  hp = HostProg();
  hp.D = (int)D;
  hp.ncols = (mode == 0) ? (int)D : 1;
  hp.dr.assign(D, 0.0);
  hp.dc.assign(D, 0.0);
  std::vector<size_t> hL, hR;
  std::vector<int> map;
  std::vector<cplx> val;
  const cplx I(0, 1);
  for (auto &t : qs->impl->terms) {
    if (t.a == cplx(0.0, 0.0)) continue;
    op_chain_map(D, t.ops, map, val);
    bool any = false, diag = true;
    for (int64_t r = 0; r < D; r++) {
      if (map[r] >= 0) {
        any = true;
        if (map[r] != r) diag = false;
      }
    }
    if (!any) continue;
    if (t.kind == 1) {
      if (diag) {
        for (int64_t r = 0; r < D; r++) {
          if (map[r] < 0) continue;
          hp.dr[r] += -I * t.a * val[r];
          if (mode == 0) hp.dc[r] += I * t.a * val[r];
        }
      } else {
        std::vector<cplx> lv(D, 0.0);
        for (int64_t r = 0; r < D; r++)
          if (map[r] >= 0) lv[r] = -I * t.a * val[r];
        add_table(hp.Lmap, hp.Lval, hL, map, lv);
        if (mode == 0) {
          std::vector<int> rm(D, -1);
          std::vector<cplx> rv(D, 0.0);
          for (int64_t k = 0; k < D; k++) {
            if (map[k] < 0) continue;
            if (rm[map[k]] >= 0) fail(9, "ERROR! operator product is not a partial injection\n");
            rm[map[k]] = (int)k;
            rv[map[k]] = I * t.a * val[k];
          }
          add_table(hp.Rmap, hp.Rval, hR, rm, rv);
        }
      }
    } else {
      if (mode == 1) fail(0, "ERROR! Lindblad terms need the density-matrix equations\n");
      std::vector<double> gam(D, 0.0);
      for (int64_t r = 0; r < D; r++)
        if (map[r] >= 0) gam[map[r]] += std::norm(val[r]);
      if (mode == 2) {
        // MCWF effective Hamiltonian H - i/2 sum a C^dag C (kron.c:664-700),
        // applied as -i H_eff: C^dag C is diagonal (C has at most one
        // nonzero per row and column), so the term adds -a/2 |C|^2 to dr
        for (int64_t r = 0; r < D; r++) hp.dr[r] += -0.5 * t.a * gam[r];
        continue;
      }
      for (int64_t r = 0; r < D; r++) {
        hp.dr[r] += -0.5 * t.a * gam[r];
        hp.dc[r] += -0.5 * t.a * gam[r];
      }
      std::vector<cplx> row(D, 0.0), col(D, 0.0);
      for (int64_t r = 0; r < D; r++) {
        if (map[r] < 0) continue;
        row[r] = t.a * val[r];
        col[r] = std::conj(val[r]);
      }
      if (diag) {
        hp.Jdrow.push_back(row);
        hp.Jdcol.push_back(col);
      } else {
        hp.Jmap.push_back(map);
        hp.Jrow.push_back(row);
        hp.Jcol.push_back(col);
      }
    }
  }
  return !has_error();
}

// L(X^H) = (L X)^H for every X.  With the compiled form
//   (L X)[r,c] = d(r,c) X[r,c] + (M_L X)[r,c] + (X M_R)[r,c] + sum_t a_t[r] b_t[c] X[p_t(r), p_t(c)]
// this holds when M_L = M_R^H, every jump pair has b_t = lambda conj(a_t)
// with lambda real, the same for the diagonal products, and
// dr[k] - conj(dc[k]) is one real constant (so d(c,r) = conj(d(r,c))).
bool hermiticity_preserving(const HostProg &hp) {
  const int D = hp.D;
  double scale = 0.0;
  auto upd = [&](cplx v) { scale = std::max(scale, std::abs(v)); };
  std::unordered_map<uint64_t, cplx> ML, MR;  // key (row << 32) | col
  for (size_t t = 0; t < hp.Lmap.size(); t++)
    for (int r = 0; r < D; r++)
      if (hp.Lmap[t][r] >= 0) {
        ML[((uint64_t)r << 32) | (uint32_t)hp.Lmap[t][r]] += hp.Lval[t][r];
        upd(hp.Lval[t][r]);
      }
  for (size_t t = 0; t < hp.Rmap.size(); t++)
    for (int c = 0; c < D; c++)
      if (hp.Rmap[t][c] >= 0) {
        MR[((uint64_t)hp.Rmap[t][c] << 32) | (uint32_t)c] += hp.Rval[t][c];
        upd(hp.Rval[t][c]);
      }
  for (auto &v : hp.dr) upd(v);
  for (auto &v : hp.dc) upd(v);
  const double tol = 1e-13 * std::max(scale, 1e-300);
  auto transposed = [](uint64_t k) { return (k << 32) | (k >> 32); };
  for (auto &kv : ML) {
    auto it = MR.find(transposed(kv.first));
    const cplx other = it == MR.end() ? cplx(0.0) : std::conj(it->second);
    if (std::abs(kv.second - other) > tol) return false;
  }
  for (auto &kv : MR)
    if (ML.find(transposed(kv.first)) == ML.end() && std::abs(kv.second) > tol) return false;
  // products a[r] b[c]: b = lambda conj(a), lambda real
  auto pair_ok = [&](const std::vector<cplx> &a, const std::vector<cplx> &b) {
    cplx lam = 0.0;
    bool have = false;
    for (int k = 0; k < D; k++) {
      if (std::abs(a[k]) > tol) {
        const cplx l = b[k] / std::conj(a[k]);
        if (!have) { lam = l; have = true; }
        if (std::abs(l - lam) > 1e-12 * std::max(1.0, std::abs(lam))) return false;
      } else if (std::abs(b[k]) > tol) {
        return false;
      }
    }
    return std::abs(lam.imag()) <= 1e-12 * std::max(1.0, std::abs(lam));
  };
  for (size_t t = 0; t < hp.Jmap.size(); t++)
    if (!pair_ok(hp.Jrow[t], hp.Jcol[t])) return false;
  for (size_t t = 0; t < hp.Jdrow.size(); t++)
    if (!pair_ok(hp.Jdrow[t], hp.Jdcol[t])) return false;
  if (!hp.dr.empty()) {
    const cplx s0 = hp.dr[0] - std::conj(hp.dc[0]);
    if (std::abs(s0.imag()) > tol) return false;
    for (int k = 1; k < D; k++)
      if (std::abs(hp.dr[k] - std::conj(hp.dc[k]) - s0) > tol) return false;
  }
  return true;
}

DeviceProgram *compile_terms(qsystem qs, int mode) {
  DeviceProgram *P = new DeviceProgram();
  HostProg &hp = P->host;
  if (!compile_host(qs, mode, hp)) { delete P; return nullptr; }
  DevProg &d = P->dev;
  d.D = hp.D;
  d.ncols = hp.ncols;
  d.nL = (int)hp.Lmap.size();
  d.nR = (int)hp.Rmap.size();
  d.nJ = (int)hp.Jmap.size();
  d.nJd = (int)hp.Jdrow.size();
  d.Lmap = upload(P, flatten(hp.Lmap));
  d.Lval = upload(P, to_d2(flatten(hp.Lval)));
  d.Rmap = upload(P, flatten(hp.Rmap));
  d.Rval = upload(P, to_d2(flatten(hp.Rval)));
  d.Jmap = upload(P, flatten(hp.Jmap));
  d.Jrow = upload(P, to_d2(flatten(hp.Jrow)));
  d.Jcol = upload(P, to_d2(flatten(hp.Jcol)));
  d.Jdrow = upload(P, to_d2(flatten(hp.Jdrow)));
  d.Jdcol = upload(P, to_d2(flatten(hp.Jdcol)));
  d.dr = upload(P, to_d2(hp.dr));
  d.dc = upload(P, to_d2(hp.dc));
  d.qubit_path = 0;
  if (options().kernel_path != 1 && mode == 0) compile_qubit(qs, hp, P);
  if (P->has_qubit && options().kernel_path != 2) {
    // one 16-byte block: error word, tile-queue done counter, tile claim counter
    char *words = nullptr;
    QCUDA(cudaMalloc(&words, 16));
    QCUDA(cudaMemset(words, 0, 16));
    P->allocations.push_back(words);
    P->errflag = (int *)words;
    P->tile_done = (unsigned *)(words + 4);
    P->tile_claim = (unsigned long long *)(words + 8);
    if (!plan_qubit_passes(*P, P->passes)) P->passes.clear();
    if (!P->passes.empty()) P->herm_ok = hermiticity_preserving(hp);
  }
  d.qubit_path = P->has_qubit ? 1 : 0;
  return P;
}

}  // namespace quac

// Exports the compiled tables without touching the GPU (used to check the
// compiler on the CPU).  counts[6] = {D, ncols, nL, nR, nJ, nJd}.  With maps
// and vals non-null, maps receives Lmap|Rmap|Jmap and vals (complex pairs)
// receives Lval|Rval|Jrow|Jcol|Jdrow|Jdcol|dr|dc, each table D long.
extern "C" int quac_program_export(qsystem qs, int mode, int64_t *counts, int *maps, double *vals) {
  using namespace quac;
  HostProg hp;
  if (!compile_host(qs, mode, hp)) return 1;
  counts[0] = hp.D; counts[1] = hp.ncols;
  counts[2] = (int64_t)hp.Lmap.size(); counts[3] = (int64_t)hp.Rmap.size();
  counts[4] = (int64_t)hp.Jmap.size(); counts[5] = (int64_t)hp.Jdrow.size();
  if (!maps || !vals) return 0;
  size_t mi = 0, vi = 0;
  for (auto *tab : {&hp.Lmap, &hp.Rmap, &hp.Jmap})
    for (auto &m : *tab) for (int x : m) maps[mi++] = x;
  for (auto *tab : {&hp.Lval, &hp.Rval, &hp.Jrow, &hp.Jcol, &hp.Jdrow, &hp.Jdcol})
    for (auto &m : *tab) for (auto &z : m) { vals[vi++] = z.real(); vals[vi++] = z.imag(); }
  for (auto *v : {&hp.dr, &hp.dc})
    for (auto &z : *v) { vals[vi++] = z.real(); vals[vi++] = z.imag(); }
  return 0;
}

namespace {

// Entries (column, value) of row i of the compiled operator, merged by
// column in ascending order; the diagonal is always present.  Density
// matrices: i = c D + r (column stacking); wavefunctions: i = r.
void operator_row(const quac::HostProg &hp, int64_t i, std::vector<std::pair<int64_t, quac::cplx>> &row) {
  using quac::cplx;
  const int64_t D = hp.D;
  row.clear();
  if (hp.ncols == 1) {
    const int r = (int)i;
    row.emplace_back(i, hp.dr[r]);
    for (size_t t = 0; t < hp.Lmap.size(); t++)
      if (hp.Lmap[t][r] >= 0) row.emplace_back(hp.Lmap[t][r], hp.Lval[t][r]);
  } else {
    const int c = (int)(i / D), r = (int)(i - (int64_t)c * D);
    cplx d = hp.dr[r] + hp.dc[c];
    for (size_t t = 0; t < hp.Jdrow.size(); t++) d += hp.Jdrow[t][r] * hp.Jdcol[t][c];
    row.emplace_back(i, d);
    for (size_t t = 0; t < hp.Lmap.size(); t++)
      if (hp.Lmap[t][r] >= 0) row.emplace_back((int64_t)c * D + hp.Lmap[t][r], hp.Lval[t][r]);
    for (size_t t = 0; t < hp.Rmap.size(); t++)
      if (hp.Rmap[t][c] >= 0) row.emplace_back((int64_t)hp.Rmap[t][c] * D + r, hp.Rval[t][c]);
    for (size_t t = 0; t < hp.Jmap.size(); t++)
      if (hp.Jmap[t][r] >= 0 && hp.Jmap[t][c] >= 0)
        row.emplace_back((int64_t)hp.Jmap[t][c] * D + hp.Jmap[t][r], hp.Jrow[t][r] * hp.Jcol[t][c]);
  }
  std::sort(row.begin(), row.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  size_t k = 0;
  for (size_t j = 0; j < row.size(); j++) {
    if (k > 0 && row[k - 1].first == row[j].first) row[k - 1].second += row[j].second;
    else row[k++] = row[j];
  }
  row.resize(k);
}

bool put_be64(FILE *f, uint64_t v) {
  v = __builtin_bswap64(v);
  return fwrite(&v, 8, 1, f) == 1;
}

bool put_be_double(FILE *f, double x) {
  uint64_t v;
  std::memcpy(&v, &x, 8);
  return put_be64(f, v);
}

}  // namespace

// No counterpart in the reference, which only prints a summary of mat_A
// (solver.c:120-124); a QuaC user reaches the assembled operator with
// MatView on a binary viewer.  Here the operator is never assembled, so
// this writes it from the compiled term tables in PETSc's binary AIJ
// format with 64-bit indices (big endian: class id 1211216, M, N, nz, row
// lengths, column indices, complex128 values), the format of the
// reference's own test fixtures, without touching the GPU.  Density
// matrices give the D^2 x D^2 Liouvillian in the column-stacked ordering,
// wavefunctions the D x D Schroedinger operator -i H.
extern "C" int quac_write_superoperator_binary(qsystem qs, const char *filename) {
  using namespace quac;
  if (!filename) { fail(0, "ERROR! quac_write_superoperator_binary: no file name\n"); return 1; }
  HostProg hp;
  const int mode = qs->dm_equations ? 0 : 1;
  if (!compile_host(qs, mode, hp)) return 1;
  const int64_t n = hp.ncols == 1 ? (int64_t)hp.D : (int64_t)hp.D * hp.D;
  FILE *f = fopen(filename, "wb");
  if (!f) { fail(0, "ERROR! quac_write_superoperator_binary: cannot open %s\n", filename); return 1; }
  std::vector<std::pair<int64_t, cplx>> row;
  std::vector<int64_t> lens(n);
  int64_t nz = 0;
  for (int64_t i = 0; i < n; i++) {
    operator_row(hp, i, row);
    lens[i] = (int64_t)row.size();
    nz += lens[i];
  }
  bool ok = put_be64(f, 1211216) && put_be64(f, n) && put_be64(f, n) && put_be64(f, nz);
  for (int64_t i = 0; ok && i < n; i++) ok = put_be64(f, lens[i]);
  for (int64_t i = 0; ok && i < n; i++) {
    operator_row(hp, i, row);
    for (auto &e : row) ok = ok && put_be64(f, (uint64_t)e.first);
  }
  for (int64_t i = 0; ok && i < n; i++) {
    operator_row(hp, i, row);
    for (auto &e : row) ok = ok && put_be_double(f, e.second.real()) && put_be_double(f, e.second.imag());
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) { fail(0, "ERROR! quac_write_superoperator_binary: writing %s failed\n", filename); return 1; }
  return 0;
}
