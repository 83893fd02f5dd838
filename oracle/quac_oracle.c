/*
 * quac_oracle.c -- CPU ORACLE (test infrastructure only).
 *
 * This file restates, in plain C99, the arithmetic of QuaC's Lindblad path so
 * that the CUDA product can be checked against it.  It is NOT part of the
 * product: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.  Nothing under quac_b200/ links or calls it.
 *
 * What it restates (reference file:line):
 *   - per-operator row -> (column, value) maps            kron.c:294-538
 *   - |i><j| (VEC pair) maps                               kron.c:540-635
 *   - operator-product chains                              kron.c:161-207
 *   - Hamiltonian superoperator -i a (I x G) + i a (G^T x I) kron.c:702-729
 *     (the complex-coefficient fixtures pin "+i a" on the right-hand term;
 *      the shipped code writes conj(a) there -- compat flag below)
 *   - Lindblad superoperator                               kron.c:995-1036
 *   - Schroedinger-only and MCWF forms                     kron.c:638-700
 *   - construct_matrix (diag zeros, -i scale for WF/MCWF)  qsystem.c:593-676
 *   - expectation values on rho / psi                      qvec_utilities.c:1197-1350
 *   - gates on rho: superoperator engine                   quantum_circuits.c:435-481, 851-3036
 *                   in-place engine                        quantum_circuits.c:696-847, 1771-2147
 *   - steady state: (L + e0 vec(I)^T) x = e0 by GMRES(m)   solver.c:33-221
 *     with ILU(0) (what PCASM reduces to on one rank)
 *   - explicit RK (RK4 fixed, Bogacki-Shampine 3(2) with a basic step
 *     controller) standing in for PETSc TSRK                qsystem.c:895-1098
 *
 * Layout conventions pinned by the reference tests: vec(rho)[D*col+row] =
 * rho[row][col] (qvec_utilities.c:322-337); subsystem 0 is the most
 * significant Hilbert digit (n_after = D/(levels*n_before), kron.c:308).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex cplx;
typedef int64_t i64;

/* operator types, same numbering as operators_p.h:6-16 */
enum { O_RAISE = -1, O_NUMBER = 0, O_LOWER = 1, O_VEC = 2, O_SX = 3, O_SY = 4,
       O_SZ = 5, O_EYE = 6, O_OTHER = 7 };
/* tensor-control modes, kron_p.h:6-10 */
enum { T_IG = -1, T_GG = 0, T_GI = 1 };

typedef struct { int type; int sub; int pos; } oop;

typedef struct {
  int nsub;
  i64 levels[64];
  i64 n_before[64];
  i64 D;
} osys;

static void sys_init(osys *s, int nsub, const i64 *levels) {
  s->nsub = nsub;
  s->D = 1;
  for (int k = 0; k < nsub; k++) {
    s->levels[k] = levels[k];
    s->n_before[k] = s->D;
    s->D *= levels[k];
  }
}

/* Row i -> (j, val) of one basic operator embedded in the D- or D^2-space.
 * Follows kron.c:294-538.  j = -1 marks an empty row. */
static void val_j_single(const osys *s, i64 i, oop op, int tc, i64 *j, cplx *val) {
  i64 D = s->D;
  if (tc == T_GG) {
    i64 j1, j2; cplx v1, v2;
    val_j_single(s, i / D, op, T_IG, &j1, &v1);
    val_j_single(s, i % D, op, T_IG, &j2, &v2);
    if (j1 < 0 || j2 < 0) { *j = -1; *val = 0; return; }
    *j = D * j1 + j2;
    *val = conj(v1) * v2;
    return;
  }
  i64 L = s->levels[op.sub];
  i64 na = D / (L * s->n_before[op.sub]) * (tc == T_GI ? D : 1);
  i64 isub = (i / na) % L;
  i64 base = i - isub * na; /* i with this digit zeroed */
  *j = -1; *val = 0;
  switch (op.type) {
    case O_LOWER:
      if (isub < L - 1) { *j = base + (isub + 1) * na; *val = sqrt((double)isub + 1.0); }
      break;
    case O_RAISE:
      if (isub >= 1) { *j = base + (isub - 1) * na; *val = sqrt((double)isub); }
      break;
    case O_SX:
      if (isub == 0) { *j = base + na; *val = 1.0; }
      else if (isub == 1) { *j = base; *val = 1.0; }
      break;
    case O_SY:
      if (isub == 0) { *j = base + na; *val = -I; }
      else if (isub == 1) { *j = base; *val = I; }
      break;
    case O_NUMBER:
      if (isub != 0) { *j = i; *val = (double)isub; }
      break;
    case O_EYE:
      *j = i; *val = 1.0;
      break;
    case O_SZ:
      if (isub == 0) { *j = i; *val = 1.0; }
      else if (isub == 1) { *j = i; *val = -1.0; }
      break;
    case O_OTHER:
      if (isub >= 2) { *j = i; *val = 1.0; }
      break;
    default:
      break;
  }
  if (tc == T_GI) *val = conj(*val);
}

/* |pos1><pos2| on one subsystem, kron.c:540-635 */
static void val_j_vecvec(const osys *s, i64 i, oop a, oop b, int tc, i64 *j, cplx *val) {
  i64 D = s->D;
  if (tc == T_GG) {
    i64 j1, j2; cplx v1, v2;
    val_j_vecvec(s, i / D, a, b, T_IG, &j1, &v1);
    val_j_vecvec(s, i % D, a, b, T_IG, &j2, &v2);
    if (j1 < 0 || j2 < 0) { *j = -1; *val = 0; return; }
    *j = D * j1 + j2; *val = conj(v1) * v2; return;
  }
  i64 L = s->levels[a.sub];
  i64 na = D / (L * s->n_before[a.sub]) * (tc == T_GI ? D : 1);
  i64 isub = (i / na) % L;
  if (isub == a.pos) { *j = i - isub * na + (i64)b.pos * na; *val = 1.0; }
  else { *j = -1; *val = 0; }
  if (tc == T_GI) *val = conj(*val);
}

/* Product chain ops[0]*ops[1]*...: kron.c:161-207 */
static void val_j_ops(const osys *s, i64 *jio, cplx *val, int nops, const oop *ops, int tc) {
  i64 j = *jio; cplx v = 1.0;
  for (int k = 0; k < nops; k++) {
    i64 j2; cplx t;
    if (ops[k].type == O_VEC) {
      if (j != -1) { val_j_vecvec(s, j, ops[k], ops[k + 1], tc, &j2, &t); j = j2; v = t * v; }
      k++;
    } else if (j != -1) {
      val_j_single(s, j, ops[k], tc, &j2, &t); j = j2; v = t * v;
    }
  }
  *jio = j; *val = v;
}

/* ---------------------------------------------------------------- COO/CSR */
typedef struct { i64 n, cap; i64 *r, *c; cplx *v; } coo;

static void coo_push(coo *m, i64 r, i64 c, cplx v) {
  if (m->n == m->cap) {
    m->cap = m->cap ? 2 * m->cap : 1024;
    m->r = realloc(m->r, m->cap * sizeof(i64));
    m->c = realloc(m->c, m->cap * sizeof(i64));
    m->v = realloc(m->v, m->cap * sizeof(cplx));
  }
  m->r[m->n] = r; m->c[m->n] = c; m->v[m->n] = v; m->n++;
}

typedef struct { i64 nrows, ncols, row0; i64 *rowptr; i64 *col; cplx *val; } csr;

static csr *coo_to_csr(coo *m, i64 row0, i64 nrows, i64 ncols) {
  csr *A = calloc(1, sizeof(csr));
  A->nrows = nrows; A->ncols = ncols; A->row0 = row0;
  A->rowptr = calloc(nrows + 1, sizeof(i64));
  for (i64 k = 0; k < m->n; k++) A->rowptr[m->r[k] - row0 + 1]++;
  for (i64 r = 0; r < nrows; r++) A->rowptr[r + 1] += A->rowptr[r];
  i64 nnz = A->rowptr[nrows];
  i64 *pos = malloc(nrows * sizeof(i64));
  memcpy(pos, A->rowptr, nrows * sizeof(i64));
  i64 *col = malloc((nnz ? nnz : 1) * sizeof(i64));
  cplx *val = malloc((nnz ? nnz : 1) * sizeof(cplx));
  for (i64 k = 0; k < m->n; k++) {
    i64 r = m->r[k] - row0; i64 p = pos[r]++;
    col[p] = m->c[k]; val[p] = m->v[k];
  }
  free(pos);
  /* sort each row by column and merge duplicates (ADD_VALUES semantics) */
  i64 out = 0;
  i64 *newptr = calloc(nrows + 1, sizeof(i64));
  for (i64 r = 0; r < nrows; r++) {
    i64 a = A->rowptr[r], b = A->rowptr[r + 1];
    for (i64 x = a + 1; x < b; x++) { /* insertion sort: rows are short */
      i64 cc = col[x]; cplx vv = val[x]; i64 y = x - 1;
      while (y >= a && col[y] > cc) { col[y + 1] = col[y]; val[y + 1] = val[y]; y--; }
      col[y + 1] = cc; val[y + 1] = vv;
    }
    i64 start = out;
    for (i64 x = a; x < b; x++) {
      if (out > start && col[out - 1] == col[x]) val[out - 1] += val[x];
      else { col[out] = col[x]; val[out] = val[x]; out++; }
    }
    newptr[r + 1] = out;
  }
  free(A->rowptr);
  A->rowptr = newptr; A->col = col; A->val = val;
  return A;
}

void orc_csr_free(csr *A) {
  if (!A) return;
  free(A->rowptr); free(A->col); free(A->val); free(A);
}
i64 orc_csr_nnz(const csr *A) { return A->rowptr[A->nrows]; }
i64 orc_csr_nrows(const csr *A) { return A->nrows; }
void orc_csr_export(const csr *A, i64 *rowptr, i64 *col, double *val) {
  memcpy(rowptr, A->rowptr, (A->nrows + 1) * sizeof(i64));
  memcpy(col, A->col, orc_csr_nnz(A) * sizeof(i64));
  memcpy(val, A->val, orc_csr_nnz(A) * sizeof(cplx));
}

/* --------------------------------------------------------- term decoding */
/* Terms arrive flattened: kind[t] (1 = HAM, 2 = LINDBLAD), a[2t..2t+1],
 * nops[t], and ops as triples (type, sub, pos) consumed in order. */
typedef struct { int kind; cplx a; int nops; oop *ops; } oterm;

static oterm *decode_terms(int nterms, const int *kind, const double *a, const int *nops,
                           const int *optrip) {
  oterm *t = calloc(nterms, sizeof(oterm));
  int p = 0;
  for (int k = 0; k < nterms; k++) {
    t[k].kind = kind[k];
    t[k].a = a[2 * k] + I * a[2 * k + 1];
    t[k].nops = nops[k];
    t[k].ops = malloc(nops[k] * sizeof(oop));
    for (int q = 0; q < nops[k]; q++) {
      t[k].ops[q].type = optrip[3 * p]; t[k].ops[q].sub = optrip[3 * p + 1];
      t[k].ops[q].pos = optrip[3 * p + 2]; p++;
    }
  }
  return t;
}
static void free_terms(oterm *t, int n) { for (int k = 0; k < n; k++) free(t[k].ops); free(t); }

/* construct_matrix (qsystem.c:593-676) restricted to rows [row0,row1) of the
 * operator.  mode: 0 = density-matrix Liouvillian (D^2), 1 = Schroedinger
 * (-i H, D), 2 = MCWF effective -i(H - i/2 sum a C^dag C) (D).
 * conj_compat: 1 reproduces the shipped conj(a) in the right-hand H term. */
csr *orc_build(int nsub, const i64 *levels, int nterms, const int *kind, const double *a,
               const int *nops, const int *optrip, int mode, int conj_compat, i64 row0,
               i64 row1) {
  osys s; sys_init(&s, nsub, levels);
  oterm *T = decode_terms(nterms, kind, a, nops, optrip);
  i64 D = s.D;
  i64 dim = (mode == 0) ? D * D : D;
  if (row1 < 0 || row1 > dim) row1 = dim;
  coo m = {0};
  /* columns whose rows intersect [row0,row1) (density-matrix mode) */
  i64 cfirst = row0 / D, clast = (row1 + D - 1) / D;
  for (int t = 0; t < nterms; t++) {
    oterm *tm = &T[t];
    if (mode == 0) {
      /* the (G^T x I) parts only move the column digit: evaluate them once
       * per column (value independent of the row digit) and emit the rows
       * that land in the block */
      i64 *cmap = malloc(D * sizeof(i64));
      cplx *cval = malloc(D * sizeof(cplx));
      for (i64 c = 0; c < D; c++) {
        i64 j = c * D; cplx v;
        val_j_ops(&s, &j, &v, tm->nops, tm->ops, T_GI);
        cmap[c] = (j == -1) ? -1 : j / D;
        cval[c] = v;
      }
      if (tm->kind == 1) {
        for (i64 i = row0; i < row1; i++) {
          i64 jig = i; cplx vig;
          val_j_ops(&s, &jig, &vig, tm->nops, tm->ops, T_IG);
          if (jig != -1) coo_push(&m, i, jig, -tm->a * I * vig);
        }
        cplx aa = conj_compat ? conj(tm->a) : tm->a;
        for (i64 c = 0; c < D; c++) {
          if (cmap[c] < 0 || cmap[c] < cfirst || cmap[c] >= clast) continue;
          for (i64 r = 0; r < D; r++) {
            i64 tgt = cmap[c] * D + r;
            if (tgt >= row0 && tgt < row1) coo_push(&m, tgt, c * D + r, aa * I * conj(cval[c]));
          }
        }
      } else {
        for (i64 i = cfirst * D; i < clast * D && i < dim; i++) {
          i64 jig = i; cplx vig;
          val_j_ops(&s, &jig, &vig, tm->nops, tm->ops, T_IG);
          if (jig != -1 && jig >= row0 && jig < row1)
            coo_push(&m, jig, jig, -0.5 * tm->a * conj(vig) * vig);
        }
        for (i64 c = 0; c < D; c++) {
          if (cmap[c] < 0 || cmap[c] < cfirst || cmap[c] >= clast) continue;
          for (i64 r = 0; r < D; r++) {
            i64 tgt = cmap[c] * D + r;
            if (tgt >= row0 && tgt < row1)
              coo_push(&m, tgt, tgt, -0.5 * tm->a * conj(conj(cval[c]) * cval[c]));
          }
        }
        for (i64 i = row0; i < row1; i++) {
          i64 jgg = i; cplx vgg;
          val_j_ops(&s, &jgg, &vgg, tm->nops, tm->ops, T_GG);
          if (jgg != -1) coo_push(&m, i, jgg, tm->a * vgg);
        }
      }
      free(cmap); free(cval);
    } else {
      if (tm->kind == 1) {
        for (i64 i = row0; i < row1; i++) {
          i64 j = i; cplx v;
          val_j_ops(&s, &j, &v, tm->nops, tm->ops, T_IG);
          if (j != -1) coo_push(&m, i, j, tm->a * v);
        }
      } else if (mode == 2) {
        /* dagger list in reverse order, then the list: kron.c:664-700 */
        int n2 = 2 * tm->nops;
        oop *tmp = malloc(n2 * sizeof(oop));
        for (int q = 0; q < tm->nops; q++) {
          oop o = tm->ops[q], od = o;
          if (o.type == O_LOWER) od.type = O_RAISE;
          else if (o.type == O_RAISE) od.type = O_LOWER;
          tmp[tm->nops - q - 1] = (o.type == O_VEC) ? o : od;
          tmp[tm->nops + q] = o;
        }
        for (i64 i = row0; i < row1; i++) {
          i64 j = i; cplx v;
          val_j_ops(&s, &j, &v, n2, tmp, T_IG);
          if (j != -1) coo_push(&m, i, j, -I * tm->a / 2.0 * v);
        }
        free(tmp);
      }
    }
  }
  for (i64 i = row0; i < row1; i++) coo_push(&m, i, i, 0.0);
  csr *A = coo_to_csr(&m, row0, row1 - row0, dim);
  free(m.r); free(m.c); free(m.v);
  if (mode != 0) {
    i64 nnz = orc_csr_nnz(A);
    for (i64 k = 0; k < nnz; k++) A->val[k] *= -I;
  }
  free_terms(T, nterms);
  return A;
}

/* y[r] = sum_k A[r,k] x[k] for the rows the CSR holds (row0 offset). */
void orc_spmv(const csr *A, const double *xd, double *yd) {
  const cplx *x = (const cplx *)xd; cplx *y = (cplx *)yd;
#pragma omp parallel for schedule(static)
  for (i64 r = 0; r < A->nrows; r++) {
    cplx acc = 0;
    for (i64 p = A->rowptr[r]; p < A->rowptr[r + 1]; p++) acc += A->val[p] * x[A->col[p]];
    y[r] = acc;
  }
}

/* ------------------------------------------------------------ integrators */
/* Classic RK4, fixed step (PETSc "-ts_rk_type 4 -ts_adapt_type none"). */
void orc_rk4(const csr *A, double *yd, double dt, i64 nsteps) {
  i64 n = A->nrows;
  cplx *y = (cplx *)yd;
  cplx *k = malloc(n * sizeof(cplx)), *x = malloc(n * sizeof(cplx)), *acc = malloc(n * sizeof(cplx));
  for (i64 st = 0; st < nsteps; st++) {
    orc_spmv(A, (double *)y, (double *)k);
    for (i64 i = 0; i < n; i++) { acc[i] = y[i] + dt / 6.0 * k[i]; x[i] = y[i] + dt / 2.0 * k[i]; }
    orc_spmv(A, (double *)x, (double *)k);
    for (i64 i = 0; i < n; i++) { acc[i] += dt / 3.0 * k[i]; x[i] = y[i] + dt / 2.0 * k[i]; }
    orc_spmv(A, (double *)x, (double *)k);
    for (i64 i = 0; i < n; i++) { acc[i] += dt / 3.0 * k[i]; x[i] = y[i] + dt * k[i]; }
    orc_spmv(A, (double *)x, (double *)k);
    for (i64 i = 0; i < n; i++) y[i] = acc[i] + dt / 6.0 * k[i];
  }
  free(k); free(x); free(acc);
}

/* Bogacki-Shampine 3(2) with the basic controller the product uses:
 *   err = sqrt(mean_i (|e_i| / (atol + rtol*max(|y_i|,|ynew_i|)))^2)
 *   accept if err <= 1; h_new = h*clamp(0.9*err^(-1/3), 0.1, 10), then
 *   clamped to [hmin,hmax]; the last step is shortened to land on tmax.
 * Returns the number of accepted steps; *nrej gets the rejections. */
i64 orc_bs3(const csr *A, double *yd, double t0, double tmax, double dt0, double atol,
            double rtol, double hmin, double hmax, i64 max_steps, i64 *nrej) {
  i64 n = A->nrows;
  cplx *y = (cplx *)yd;
  cplx *k1 = malloc(n * sizeof(cplx)), *k2 = malloc(n * sizeof(cplx)),
       *k3 = malloc(n * sizeof(cplx)), *k4 = malloc(n * sizeof(cplx)),
       *x = malloc(n * sizeof(cplx)), *yn = malloc(n * sizeof(cplx));
  double t = t0, h = dt0;
  i64 acc = 0, rej = 0;
  while (t < tmax - 1e-12 * fabs(tmax) && acc < max_steps) {
    int last = 0;
    if (t + h >= tmax) { h = tmax - t; last = 1; }
    orc_spmv(A, (double *)y, (double *)k1);
    for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.5 * h * k1[i];
    orc_spmv(A, (double *)x, (double *)k2);
    for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.75 * h * k2[i];
    orc_spmv(A, (double *)x, (double *)k3);
    for (i64 i = 0; i < n; i++) yn[i] = y[i] + h * (2.0 / 9.0 * k1[i] + 1.0 / 3.0 * k2[i] + 4.0 / 9.0 * k3[i]);
    orc_spmv(A, (double *)yn, (double *)k4);
    double s = 0;
    for (i64 i = 0; i < n; i++) {
      cplx e = h * ((2.0 / 9.0 - 7.0 / 24.0) * k1[i] + (1.0 / 3.0 - 0.25) * k2[i] +
                    (4.0 / 9.0 - 1.0 / 3.0) * k3[i] - 0.125 * k4[i]);
      double m = fmax(cabs(y[i]), cabs(yn[i]));
      double q = cabs(e) / (atol + rtol * m);
      s += q * q;
    }
    double err = sqrt(s / (double)n);
    double fac = (err > 0) ? 0.9 * pow(err, -1.0 / 3.0) : 10.0;
    if (fac < 0.1) fac = 0.1;
    if (fac > 10.0) fac = 10.0;
    double hnew = h * fac;
    if (hnew < hmin) hnew = hmin;
    if (hnew > hmax) hnew = hmax;
    if (err <= 1.0 || h <= hmin * (1 + 1e-12)) {
      memcpy(y, yn, n * sizeof(cplx));
      t = last ? tmax : t + h;
      acc++;
    } else {
      rej++;
    }
    h = hnew;
  }
  if (nrej) *nrej = rej;
  free(k1); free(k2); free(k3); free(k4); free(x); free(yn);
  return acc;
}

/* Dormand-Prince 5(4) (the published 1980 tableau, FSAL) with the same
 * basic controller as orc_bs3 (exponent -1/5).  The error norm is the
 * weighted RMS of h*sum (b - bhat)_i k_i. */
static const double DP_C[7] = {0.0, 0.2, 0.3, 0.8, 8.0 / 9.0, 1.0, 1.0};
static const double DP_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.2, 0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
static const double DP_E[7] = {35.0 / 384.0 - 5179.0 / 57600.0, 0.0, 500.0 / 1113.0 - 7571.0 / 16695.0,
                               125.0 / 192.0 - 393.0 / 640.0, -2187.0 / 6784.0 + 92097.0 / 339200.0,
                               11.0 / 84.0 - 187.0 / 2100.0, -1.0 / 40.0};

i64 orc_dp5(const csr *A, double *yd, double t0, double tmax, double dt0, double atol,
            double rtol, double hmin, double hmax, i64 max_steps, i64 *nrej) {
  i64 n = A->nrows;
  cplx *y = (cplx *)yd;
  cplx *k[7];
  for (int s = 0; s < 7; s++) k[s] = malloc(n * sizeof(cplx));
  cplx *x = malloc(n * sizeof(cplx));
  double t = t0, h = dt0;
  i64 acc = 0, rej = 0;
  while (t < tmax - 1e-12 * fabs(tmax) && acc < max_steps) {
    int last = 0;
    if (t + h >= tmax) { h = tmax - t; last = 1; }
    orc_spmv(A, (double *)y, (double *)k[0]);
    for (int s = 1; s < 7; s++) {
      for (i64 i = 0; i < n; i++) {
        cplx v = y[i];
        for (int j = 0; j < s; j++) v += h * DP_A[s][j] * k[j][i];
        x[i] = v;
      }
      orc_spmv(A, (double *)x, (double *)k[s]);
    }
    /* x holds the 5th-order solution (stage 7 input) */
    double ssum = 0;
    for (i64 i = 0; i < n; i++) {
      cplx e = 0;
      for (int j = 0; j < 7; j++) e += h * DP_E[j] * k[j][i];
      double m = fmax(cabs(y[i]), cabs(x[i]));
      double q = cabs(e) / (atol + rtol * m);
      ssum += q * q;
    }
    double err = sqrt(ssum / (double)n);
    double fac = (err > 0) ? 0.9 * pow(err, -0.2) : 10.0;
    if (fac < 0.1) fac = 0.1;
    if (fac > 10.0) fac = 10.0;
    double hnew = h * fac;
    if (hnew < hmin) hnew = hmin;
    if (hnew > hmax) hnew = hmax;
    if (err <= 1.0 || h <= hmin * (1 + 1e-12)) {
      memcpy(y, x, n * sizeof(cplx));
      t = last ? tmax : t + h;
      acc++;
    } else {
      rej++;
    }
    h = hnew;
  }
  if (nrej) *nrej = rej;
  for (int s = 0; s < 7; s++) free(k[s]);
  free(x);
  return acc;
}

/* ------------------------------------------------------------ observables */
/* Tr(O rho) for O = ops[0]*ops[1]*...: qvec_utilities.c:1197-1283.
 * Sum over columns c of O[c, j(c)] * rho[j(c), c]. */
void orc_expect_dm(int nsub, const i64 *levels, int nops, const int *optrip, const double *rho_d,
                   double *out) {
  osys s; sys_init(&s, nsub, levels);
  oop *ops = malloc(nops * sizeof(oop));
  for (int q = 0; q < nops; q++) { ops[q].type = optrip[3 * q]; ops[q].sub = optrip[3 * q + 1]; ops[q].pos = optrip[3 * q + 2]; }
  const cplx *rho = (const cplx *)rho_d;
  cplx acc = 0;
  for (i64 c = 0; c < s.D; c++) {
    i64 j = c; cplx v;
    val_j_ops(&s, &j, &v, nops, ops, T_IG);
    if (j >= 0) acc += v * rho[s.D * c + j];
  }
  free(ops);
  out[0] = creal(acc); out[1] = cimag(acc);
}

/* <psi|O|psi>: qvec_utilities.c:1285-1350 */
void orc_expect_wf(int nsub, const i64 *levels, int nops, const int *optrip, const double *psi_d,
                   double *out) {
  osys s; sys_init(&s, nsub, levels);
  oop *ops = malloc(nops * sizeof(oop));
  for (int q = 0; q < nops; q++) { ops[q].type = optrip[3 * q]; ops[q].sub = optrip[3 * q + 1]; ops[q].pos = optrip[3 * q + 2]; }
  const cplx *psi = (const cplx *)psi_d;
  cplx acc = 0;
  for (i64 r = 0; r < s.D; r++) {
    i64 j = r; cplx v;
    val_j_ops(&s, &j, &v, nops, ops, T_IG);
    if (j >= 0) acc += conj(psi[r]) * v * psi[j];
  }
  free(ops);
  out[0] = creal(acc); out[1] = cimag(acc);
}

/* ------------------------------------------------------------------ gates */
/* Gate numbering as quantum_gates.h:11-33. */
enum { G_SQISWP = -8, G_CZARP = -7, G_CUSTOM2Q = -6, G_CZX = -5, G_CMZ = -4, G_CZ = -3,
       G_CXZ = -2, G_CNOT = -1, G_H = 1, G_X = 2, G_Y = 3, G_Z = 4, G_EYE = 5, G_RX = 6,
       G_RY = 7, G_RZ = 8, G_U1 = 9, G_U2 = 10, G_U3 = 11, G_CUSTOM1Q = 12 };

/* 2x2 matrices of the one-qubit gates (quantum_circuits.c:2160-2900) */
static void gate1_matrix(int g, double th, double ph, double la, const double *custom, cplx U[4]) {
  double c = cos(th / 2), sn = sin(th / 2);
  switch (g) {
    case G_H: U[0] = M_SQRT1_2; U[1] = M_SQRT1_2; U[2] = M_SQRT1_2; U[3] = -M_SQRT1_2; break;
    case G_X: U[0] = 0; U[1] = 1; U[2] = 1; U[3] = 0; break;
    case G_Y: U[0] = 0; U[1] = -I; U[2] = I; U[3] = 0; break;
    case G_Z: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = -1; break;
    case G_EYE: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = 1; break;
    case G_RX: U[0] = c; U[1] = -I * sn; U[2] = -I * sn; U[3] = c; break;
    case G_RY: U[0] = c; U[1] = -sn; U[2] = sn; U[3] = c; break;
    case G_RZ: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = cexp(I * th); break;
    case G_U1: case G_U2: case G_U3:
      U[0] = c; U[1] = -cexp(I * la) * sn; U[2] = cexp(I * ph) * sn; U[3] = cexp(I * (la + ph)) * c;
      break;
    case G_CUSTOM1Q:
      for (int k = 0; k < 4; k++) U[k] = custom[2 * k] + I * custom[2 * k + 1];
      break;
    default: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = 1; break;
  }
}

/* 4x4 matrices of the two-qubit gates in the basis index 2*d(q0)+d(q1)
 * (q0 = control).  The reference's basis permutation (quantum_circuits.c:
 * 2903-2953 with 851-916) makes CNOT/CXZ/CZX/CmZ/CZ/CZ_ARP act with
 * qubit_numbers[0] as the control whatever the subsystem order. */
static void gate2_matrix(int g, const double *custom, cplx U[16]) {
  for (int k = 0; k < 16; k++) U[k] = 0;
  switch (g) {
    case G_CNOT: U[0] = 1; U[5] = 1; U[11] = 1; U[14] = 1; break;
    case G_CXZ: U[0] = 1; U[5] = 1; U[2 * 4 + 3] = -1; U[3 * 4 + 2] = 1; break;
    case G_CZX: U[0] = 1; U[5] = 1; U[2 * 4 + 3] = 1; U[3 * 4 + 2] = -1; break;
    case G_CMZ: U[0] = 1; U[5] = 1; U[10] = -1; U[15] = 1; break;
    case G_CZ: U[0] = 1; U[5] = 1; U[10] = 1; U[15] = -1; break;
    case G_CZARP: U[0] = 1; U[5] = -1; U[10] = -1; U[15] = -1; break;
    case G_SQISWP:
      U[0] = 1; U[5] = M_SQRT1_2; U[6] = I * M_SQRT1_2; U[9] = I * M_SQRT1_2; U[10] = M_SQRT1_2; U[15] = 1;
      break;
    case G_CUSTOM2Q:
      for (int k = 0; k < 16; k++) U[k] = custom[2 * k] + I * custom[2 * k + 1];
      break;
    default: U[0] = U[5] = U[10] = U[15] = 1; break;
  }
}

/* Superoperator engine (_apply_gate_sys, quantum_circuits.c:435-481):
 * rho <- U rho U^dag with qubit q = subsystem q (digit stride n_after).
 * CUSTOM2Q is applied in the significance-ordered basis (the reference
 * evaluates the user function on the permuted i_sub directly). */
void orc_gate_superop(int nsub, const i64 *levels, int g, int nq, const int *qubits, double th,
                      double ph, double la, const double *custom, double *rho_d, int is_dm) {
  osys s; sys_init(&s, nsub, levels);
  i64 D = s.D;
  cplx *rho = (cplx *)rho_d;
  i64 ncols = is_dm ? D : 1;
  cplx *tmp = malloc(D * sizeof(cplx));
  if (nq == 1) {
    cplx U[4]; gate1_matrix(g, th, ph, la, custom, U);
    i64 st = D / (2 * s.n_before[qubits[0]]);
    /* rows: U acting on the row digit */
    for (i64 c = 0; c < ncols; c++) {
      cplx *col = rho + c * D;
      for (i64 r = 0; r < D; r++) {
        i64 d = (r / st) % 2, b = r - d * st;
        tmp[r] = U[d * 2 + 0] * col[b] + U[d * 2 + 1] * col[b + st];
      }
      memcpy(col, tmp, D * sizeof(cplx));
    }
    if (is_dm) { /* columns: conj(U) acting on the column digit */
      cplx *row = malloc(D * sizeof(cplx));
      for (i64 r = 0; r < D; r++) {
        for (i64 c = 0; c < D; c++) {
          i64 d = (c / st) % 2, b = c - d * st;
          row[c] = conj(U[d * 2 + 0]) * rho[b * D + r] + conj(U[d * 2 + 1]) * rho[(b + st) * D + r];
        }
        for (i64 c = 0; c < D; c++) rho[c * D + r] = row[c];
      }
      free(row);
    }
  } else {
    cplx U[16]; gate2_matrix(g, custom, U);
    int q0 = qubits[0], q1 = qubits[1];
    i64 s0 = D / (2 * s.n_before[q0]), s1 = D / (2 * s.n_before[q1]);
    int swap = (g == G_CUSTOM2Q && s.n_before[q1] < s.n_before[q0]);
    for (i64 c = 0; c < ncols; c++) {
      cplx *col = rho + c * D;
      for (i64 r = 0; r < D; r++) {
        i64 d0 = (r / s0) % 2, d1 = (r / s1) % 2, b = r - d0 * s0 - d1 * s1;
        i64 ri = swap ? 2 * d1 + d0 : 2 * d0 + d1;
        cplx acc = 0;
        for (int e0 = 0; e0 < 2; e0++)
          for (int e1 = 0; e1 < 2; e1++) {
            i64 ci = swap ? 2 * e1 + e0 : 2 * e0 + e1;
            acc += U[ri * 4 + ci] * col[b + e0 * s0 + e1 * s1];
          }
        tmp[r] = acc;
      }
      memcpy(col, tmp, D * sizeof(cplx));
    }
    if (is_dm) {
      cplx *row = malloc(D * sizeof(cplx));
      for (i64 r = 0; r < D; r++) {
        for (i64 c = 0; c < D; c++) {
          i64 d0 = (c / s0) % 2, d1 = (c / s1) % 2, b = c - d0 * s0 - d1 * s1;
          i64 ri = swap ? 2 * d1 + d0 : 2 * d0 + d1;
          cplx acc = 0;
          for (int e0 = 0; e0 < 2; e0++)
            for (int e1 = 0; e1 < 2; e1++) {
              i64 ci = swap ? 2 * e1 + e0 : 2 * e0 + e1;
              acc += conj(U[ri * 4 + ci]) * rho[(b + e0 * s0 + e1 * s1) * D + r];
            }
          row[c] = acc;
        }
        for (i64 c = 0; c < D; c++) rho[c * D + r] = row[c];
      }
      free(row);
    }
  }
  free(tmp);
}

/* In-place engine (_apply_gate2 + *_gate_func_wf, quantum_circuits.c:696-
 * 847, 1771-2147).  dims = qvec hspace_dims (for a DM: [L..., L...]);
 * qubit q acts with stride prod(dims[0..q-1]).  For a DM the gate is
 * applied to the row half, then (conjugated, except RZ which the reference
 * never conjugates) to the column half with q shifted by ndims/2.
 * Two-qubit gates use bit positions q (insertTwoZeroBits) except CNOT which
 * uses the products of dims. */
static void wf_gate_pass(i64 n, const i64 *dims, int g, const int *q, double th, double ph,
                         double la, const double *custom, int conj_gate, cplx *a) {
  if (g == G_CNOT) {
    i64 nb = 1, nb2 = 1;
    for (int k = 0; k < q[1]; k++) nb *= dims[k];
    for (int k = 0; k < q[0]; k++) nb2 *= dims[k];
    for (i64 i = 0; i < n / 2; i++) {
      i64 i1 = (i / nb) * 2 * nb + i % nb, i0 = i1 + nb;
      if ((i1 / nb2) % 2 == 1) { cplx t = a[i1]; a[i1] = a[i0]; a[i0] = t; }
    }
    return;
  }
  if (g == G_CZARP || g == G_SQISWP || g == G_CUSTOM2Q) {
    cplx U[16]; gate2_matrix(g, custom, U);
    if (g == G_SQISWP && conj_gate) for (int k = 0; k < 16; k++) U[k] = conj(U[k]);
    /* basis index k: bit0 <-> q[0], bit1 <-> q[1] */
    cplx V[16];
    /* the reference's 4x4 for these is written as array[ind01] = row 1 with
       ind01 = q0 flipped, ind10 = q1 flipped: i.e. index = b(q0) + 2 b(q1) */
    for (int k = 0; k < 16; k++) V[k] = U[k];
    int lo = q[0] < q[1] ? q[0] : q[1], hi = q[0] < q[1] ? q[1] : q[0];
    for (i64 i = 0; i < n / 4; i++) {
      i64 x = i;
      x = ((x >> lo) << (lo + 1)) | (x & ((1LL << lo) - 1));
      x = ((x >> hi) << (hi + 1)) | (x & ((1LL << hi) - 1));
      i64 idx[4] = {x, x ^ (1LL << q[0]), x ^ (1LL << q[1]), x ^ (1LL << q[0]) ^ (1LL << q[1])};
      cplx v[4] = {a[idx[0]], a[idx[1]], a[idx[2]], a[idx[3]]};
      for (int r = 0; r < 4; r++) {
        cplx acc = 0;
        for (int cc = 0; cc < 4; cc++) acc += V[r * 4 + cc] * v[cc];
        a[idx[r]] = acc;
      }
    }
    return;
  }
  i64 nb = 1;
  for (int k = 0; k < q[0]; k++) nb *= dims[k];
  cplx U[4];
  if (g == G_RZ) { U[0] = 1; U[1] = 0; U[2] = 0; U[3] = cexp(I * th); }
  else {
    gate1_matrix(g, th, ph, la, custom, U);
    if (conj_gate && (g == G_U1 || g == G_U2 || g == G_U3)) for (int k = 0; k < 4; k++) U[k] = conj(U[k]);
  }
  for (i64 i = 0; i < n / 2; i++) {
    i64 i0 = (i / nb) * 2 * nb + i % nb, i1 = i0 + nb;
    cplx t0 = a[i0], t1 = a[i1];
    a[i0] = U[0] * t0 + U[1] * t1;
    a[i1] = U[2] * t0 + U[3] * t1;
  }
}

void orc_gate_inplace(int ndims, const i64 *dims, int g, int nq, const int *qubits, double th,
                      double ph, double la, const double *custom, double *state_d, int is_dm) {
  i64 n = 1;
  for (int k = 0; k < ndims; k++) n *= dims[k];
  cplx *a = (cplx *)state_d;
  int q[2] = {qubits[0], nq > 1 ? qubits[1] : 0};
  wf_gate_pass(n, dims, g, q, th, ph, la, custom, 0, a);
  if (is_dm) {
    int qs[2] = {q[0] + ndims / 2, q[1] + ndims / 2};
    double cc[32];
    const double *cu = custom;
    if (g == G_CUSTOM1Q || g == G_CUSTOM2Q) {
      int m = (g == G_CUSTOM1Q) ? 4 : 16;
      for (int k = 0; k < m; k++) { cc[2 * k] = custom[2 * k]; cc[2 * k + 1] = -custom[2 * k + 1]; }
      cu = cc;
    }
    wf_gate_pass(n, dims, g, qs, th, ph, la, cu, 1, a);
  }
}

/* ---------------------------------------------------------- steady state */
/* ILU(0) on a square CSR (in place on a copy of the values). */
typedef struct { i64 n; i64 *rowptr, *col, *diag; cplx *lu; } ilu0;

static ilu0 *ilu0_factor(const csr *A) {
  ilu0 *F = calloc(1, sizeof(ilu0));
  i64 n = A->nrows, nnz = orc_csr_nnz(A);
  F->n = n; F->rowptr = A->rowptr; F->col = A->col;
  F->lu = malloc(nnz * sizeof(cplx));
  memcpy(F->lu, A->val, nnz * sizeof(cplx));
  F->diag = malloc(n * sizeof(i64));
  i64 *pos = malloc(n * sizeof(i64));
  for (i64 k = 0; k < n; k++) pos[k] = -1;
  for (i64 i = 0; i < n; i++) {
    F->diag[i] = -1;
    for (i64 p = A->rowptr[i]; p < A->rowptr[i + 1]; p++) { pos[A->col[p]] = p; if (A->col[p] == i) F->diag[i] = p; }
    for (i64 p = A->rowptr[i]; p < A->rowptr[i + 1] && A->col[p] < i; p++) {
      i64 k = A->col[p];
      if (F->diag[k] < 0 || F->lu[F->diag[k]] == 0) continue;
      cplx m = F->lu[p] / F->lu[F->diag[k]];
      F->lu[p] = m;
      for (i64 q = F->diag[k] + 1; q < A->rowptr[k + 1]; q++) {
        i64 jj = A->col[q];
        if (pos[jj] >= 0) F->lu[pos[jj]] -= m * F->lu[q];
      }
    }
    for (i64 p = A->rowptr[i]; p < A->rowptr[i + 1]; p++) pos[A->col[p]] = -1;
  }
  free(pos);
  return F;
}

static void ilu0_solve(const ilu0 *F, const cplx *b, cplx *x) {
  i64 n = F->n;
  for (i64 i = 0; i < n; i++) {
    cplx s = b[i];
    for (i64 p = F->rowptr[i]; p < F->rowptr[i + 1] && F->col[p] < i; p++) s -= F->lu[p] * x[F->col[p]];
    x[i] = s;
  }
  for (i64 i = n - 1; i >= 0; i--) {
    cplx s = x[i];
    for (i64 p = F->diag[i] + 1; p < F->rowptr[i + 1]; p++) s -= F->lu[p] * x[F->col[p]];
    x[i] = (F->diag[i] >= 0 && F->lu[F->diag[i]] != 0) ? s / F->lu[F->diag[i]] : s;
  }
}

static double nrm2(i64 n, const cplx *x) {
  double s = 0;
  for (i64 i = 0; i < n; i++) s += creal(x[i]) * creal(x[i]) + cimag(x[i]) * cimag(x[i]);
  return sqrt(s);
}

/* Adds the trace row of solver.c:60-75 (row 0 += 1 at columns i*(D+1)) to a
 * full Liouvillian CSR (rows 0..D^2-1) and returns the new matrix. */
csr *orc_add_trace_row(const csr *A, i64 D) {
  coo m = {0};
  for (i64 r = 0; r < A->nrows; r++)
    for (i64 p = A->rowptr[r]; p < A->rowptr[r + 1]; p++) coo_push(&m, r, A->col[p], A->val[p]);
  for (i64 i = 0; i < D; i++) coo_push(&m, 0, i * (D + 1), 1.0);
  csr *B = coo_to_csr(&m, 0, A->nrows, A->ncols);
  free(m.r); free(m.c); free(m.v);
  return B;
}

/* GMRES(m) with right ILU(0) preconditioning (A M^-1 y = b, x = M^-1 y),
 * classical Gram-Schmidt, on the stabilised operator with b = x0 = e0
 * (solver.c:143-198).  Right preconditioning keeps the Arnoldi residual
 * equal to the true residual ||b - A x||, which is the quantity the
 * steady-state comparison is judged on (PETSc's default is left
 * preconditioning; the fixed point is the same).  Returns iterations. */
i64 orc_gmres_ilu(const csr *B, double *xd, double rtol, int restart, i64 maxit, int use_ilu) {
  i64 n = B->nrows;
  cplx *x = (cplx *)xd;
  ilu0 *F = use_ilu ? ilu0_factor(B) : NULL;
  int m = restart;
  cplx *V = malloc((size_t)(m + 1) * n * sizeof(cplx));
  cplx *H = calloc((size_t)(m + 1) * m, sizeof(cplx));
  cplx *cs = malloc(m * sizeof(cplx)), *sn = malloc(m * sizeof(cplx)), *g = malloc((m + 1) * sizeof(cplx));
  cplx *w = malloc(n * sizeof(cplx)), *t = malloc(n * sizeof(cplx)), *b = calloc(n, sizeof(cplx));
  b[0] = 1.0;
  double bnorm = 1.0;
  i64 it = 0;
  while (it < maxit) {
    orc_spmv(B, (double *)x, (double *)w);
    for (i64 i = 0; i < n; i++) w[i] = b[i] - w[i];
    double beta = nrm2(n, w);
    if (beta <= rtol * bnorm) break;
    for (i64 i = 0; i < n; i++) V[i] = w[i] / beta;
    for (int k = 0; k <= m; k++) g[k] = 0;
    g[0] = beta;
    int j;
    for (j = 0; j < m && it < maxit; j++, it++) {
      const cplx *vj = V + (size_t)j * n;
      if (F) ilu0_solve(F, vj, t); else memcpy(t, vj, n * sizeof(cplx));
      orc_spmv(B, (double *)t, (double *)w);
      for (int k = 0; k <= j; k++) {
        cplx h = 0; const cplx *vk = V + (size_t)k * n;
        for (i64 i = 0; i < n; i++) h += conj(vk[i]) * w[i];
        H[k * m + j] = h;
        for (i64 i = 0; i < n; i++) w[i] -= h * vk[i];
      }
      double hn = nrm2(n, w);
      H[(j + 1) * m + j] = hn;
      if (hn > 0) for (i64 i = 0; i < n; i++) V[(size_t)(j + 1) * n + i] = w[i] / hn;
      for (int k = 0; k < j; k++) {
        cplx a = H[k * m + j], bb = H[(k + 1) * m + j];
        H[k * m + j] = conj(cs[k]) * a + conj(sn[k]) * bb;
        H[(k + 1) * m + j] = -sn[k] * a + cs[k] * bb;
      }
      cplx a = H[j * m + j], bb = H[(j + 1) * m + j];
      double r = sqrt(creal(a * conj(a)) + creal(bb * conj(bb)));
      if (r == 0) { cs[j] = 1; sn[j] = 0; }
      else { cs[j] = a / r; sn[j] = bb / r; }
      H[j * m + j] = r; H[(j + 1) * m + j] = 0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = conj(cs[j]) * g[j];
      if (cabs(g[j + 1]) <= rtol * bnorm) { j++; it++; break; }
    }
    cplx *yv = calloc(j > 0 ? j : 1, sizeof(cplx));
    for (int k = j - 1; k >= 0; k--) {
      cplx s = g[k];
      for (int q = k + 1; q < j; q++) s -= H[k * m + q] * yv[q];
      yv[k] = s / H[k * m + k];
    }
    /* x += M^-1 (V y) */
    for (i64 i = 0; i < n; i++) w[i] = 0;
    for (int k = 0; k < j; k++) {
      const cplx *vk = V + (size_t)k * n;
      for (i64 i = 0; i < n; i++) w[i] += yv[k] * vk[i];
    }
    if (F) ilu0_solve(F, w, t); else memcpy(t, w, n * sizeof(cplx));
    for (i64 i = 0; i < n; i++) x[i] += t[i];
    free(yv);
  }
  free(V); free(H); free(cs); free(sn); free(g); free(w); free(t); free(b);
  if (F) { free(F->lu); free(F->diag); free(F); }
  return it;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ MCWF
 * Quantum-jump trajectories (use_mcwf_solver / _sys_MCWF_PostEventFunction,
 * qsystem.c:358-403, 1139-1235) with the jump-time location and the random
 * stream the CUDA engine defines for them: norm threshold r ~ U[0,1), the
 * crossing of |psi|^2 = r located by bisection on the step length to
 * 1e-9, jump k with probability Re(a_k) |C_k psi|^2 / total, then
 * psi <- sqrt(a_k) C_k psi / sqrt(Re(a_k) |C_k psi|^2), new threshold.
 * Draw k of trajectory i: SplitMix64 (Steele, Lea and Flood, 2014) of
 * seed ^ SplitMix64((i << 32) ^ k), top 53 bits.  Heff is the mode-2
 * operator of orc_build, C[k] the jump operators as CSR (one term each),
 * scheme 0 adaptive BS3 (the orc_bs3 controller), 1 fixed BS3, 2 fixed
 * classical RK4.  psi (ntraj x D), thr and cnt are advanced in place;
 * returns 0, or 1 / 2 on a step limit / unlocated jump.                   */
static uint64_t sm64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double orc_mcwf_draw(uint64_t seed, i64 i, uint64_t k) {
  uint64_t h = sm64(seed ^ sm64(((uint64_t)i << 32) ^ k));
  return (double)(h >> 11) * 0x1.0p-53;
}

static double mc_norm2(const cplx *x, i64 n) {
  double s = 0;
  for (i64 i = 0; i < n; i++) s += creal(x[i]) * creal(x[i]) + cimag(x[i]) * cimag(x[i]);
  return s;
}

static double mc_step(const csr *A, int scheme, double atol, double rtol, double h, const cplx *y, cplx *yn,
                      cplx *k1, cplx *k2, cplx *k3, cplx *k4, cplx *x) {
  i64 n = A->nrows;
  orc_spmv(A, (const double *)y, (double *)k1);
  if (scheme == 2) {
    for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.5 * h * k1[i];
    orc_spmv(A, (const double *)x, (double *)k2);
    for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.5 * h * k2[i];
    orc_spmv(A, (const double *)x, (double *)k3);
    for (i64 i = 0; i < n; i++) x[i] = y[i] + h * k3[i];
    orc_spmv(A, (const double *)x, (double *)k4);
    for (i64 i = 0; i < n; i++) yn[i] = y[i] + h / 6.0 * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
    return 0.0;
  }
  for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.5 * h * k1[i];
  orc_spmv(A, (const double *)x, (double *)k2);
  for (i64 i = 0; i < n; i++) x[i] = y[i] + 0.75 * h * k2[i];
  orc_spmv(A, (const double *)x, (double *)k3);
  for (i64 i = 0; i < n; i++) yn[i] = y[i] + h * (2.0 / 9.0 * k1[i] + 1.0 / 3.0 * k2[i] + 4.0 / 9.0 * k3[i]);
  if (scheme != 0) return 0.0;
  orc_spmv(A, (const double *)yn, (double *)k4);
  double s = 0;
  for (i64 i = 0; i < n; i++) {
    cplx e = h * ((2.0 / 9.0 - 7.0 / 24.0) * k1[i] + (1.0 / 3.0 - 0.25) * k2[i] +
                  (4.0 / 9.0 - 1.0 / 3.0) * k3[i] - 0.125 * k4[i]);
    double m = fmax(cabs(y[i]), cabs(yn[i]));
    double q = cabs(e) / (atol + rtol * m);
    s += q * q;
  }
  return sqrt(s / (double)n);
}

int orc_mcwf(const csr *Heff, int nJ, const csr *const *C, const double *a, double *psid, int ntraj,
             double *thr, uint64_t *cnt, uint64_t seed, double t0, double tmax, double dt, double atol,
             double rtol, double hmin, double hmax, int scheme, i64 max_steps, i64 *stats) {
  i64 D = Heff->nrows;
  cplx *y = malloc(D * sizeof(cplx)), *yn = malloc(D * sizeof(cplx)), *k1 = malloc(D * sizeof(cplx)),
       *k2 = malloc(D * sizeof(cplx)), *k3 = malloc(D * sizeof(cplx)), *k4 = malloc(D * sizeof(cplx)),
       *x = malloc(D * sizeof(cplx)), *cy = malloc(D * sizeof(cplx));
  double *pj = malloc((nJ > 0 ? nJ : 1) * sizeof(double));
  int status = 0;
  for (int i = 0; i < ntraj && !status; i++) {
    cplx *psi = (cplx *)psid + (i64)i * D;
    memcpy(y, psi, D * sizeof(cplx));
    double r = thr[i];
    uint64_t c = cnt[i];
    double t = t0, h = dt;
    i64 steps = 0, jumps = 0;
    double tend_tol = 1e-12 * fmax(1.0, fabs(tmax));
    while (t < tmax - tend_tol) {
      if (steps >= max_steps) { status = 1; break; }
      double h_try = h;
      int last = 0;
      if (t + h_try >= tmax - tend_tol) { h_try = tmax - t; last = 1; }
      double err = mc_step(Heff, scheme, atol, rtol, h_try, y, yn, k1, k2, k3, k4, x);
      double h_next = h;
      if (scheme == 0) {
        double fac = err > 0 ? 0.9 * pow(err, -1.0 / 3.0) : 10.0;
        fac = fmin(10.0, fmax(0.1, fac));
        h_next = fmin(hmax, fmax(hmin, h_try * fac));
        if (!(err <= 1.0 || h_try <= hmin * (1 + 1e-12))) { h = h_next; continue; }
      }
      if (mc_norm2(yn, D) < r) {
        double lo = 0.0, hi = h_try, mid = h_try;
        int found = 0;
        for (int it = 0; it < 200; it++) {
          mid = 0.5 * (lo + hi);
          mc_step(Heff, scheme, atol, rtol, mid, y, yn, k1, k2, k3, k4, x);
          double nm = mc_norm2(yn, D);
          if (fabs(nm - r) <= 1e-9) { found = 1; break; }
          if (nm < r) hi = mid; else lo = mid;
          if (hi - lo <= 1e-15 * fmax(1.0, fabs(t))) { found = 1; break; }
        }
        if (!found) { status = 2; break; }
        t += mid;
        double ptot = 0;
        for (int k = 0; k < nJ; k++) {
          orc_spmv(C[k], (const double *)yn, (double *)cy);
          pj[k] = a[2 * k] * mc_norm2(cy, D);
          ptot += pj[k];
        }
        double u = orc_mcwf_draw(seed, i, c++);
        int kj = -1;
        double pk = 0, cum = 0;
        for (int k = 0; k < nJ; k++) {
          cum += pj[k] / ptot;
          if (cum >= u) { kj = k; pk = pj[k]; break; }
        }
        if (kj >= 0 && pk > 0) {
          cplx sa = csqrt(a[2 * kj] + I * a[2 * kj + 1]);
          cplx sc = sa / sqrt(pk);
          orc_spmv(C[kj], (const double *)yn, (double *)cy);
          for (i64 q = 0; q < D; q++) y[q] = sc * cy[q];
          jumps++;
        } else {
          double nn = 1.0 / sqrt(mc_norm2(yn, D));
          for (i64 q = 0; q < D; q++) y[q] = yn[q] * nn;
        }
        r = orc_mcwf_draw(seed, i, c++);
        continue;
      }
      memcpy(y, yn, D * sizeof(cplx));
      steps++;
      t = last ? tmax : t + h_try;
      if (scheme == 0) h = h_next;
    }
    memcpy(psi, y, D * sizeof(cplx));
    thr[i] = r;
    cnt[i] = c;
    if (stats) { stats[2 * i] += steps; stats[2 * i + 1] += jumps; }
  }
  free(y); free(yn); free(k1); free(k2); free(k3); free(k4); free(x); free(cy); free(pj);
  return status;
}
