// extern "C" QuaC API: system building, qvecs, observables, gates and the
// legacy global-state entry points.  Time stepping lives in integrate.cpp,
// the steady-state solver in steady.cu.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <random>

#include "runtime.h"

namespace quac {

// ------------------------------------------------------------------ errors
static int g_error_mode = QUAC_ERRORS_EXIT;
static std::string g_last_error;
static bool g_has_error = false;
static std::atomic<int64_t> g_launches{0};

void fail(int exit_code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  g_has_error = true;
  if (g_error_mode == QUAC_ERRORS_EXIT) {
    fputs(buf, stdout);
    fflush(stdout);
    exit(exit_code);
  }
}

bool has_error() { return g_has_error; }

void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e != cudaSuccess) fail(9, "ERROR! CUDA call %s failed at %s:%d: %s\n", what, file, line,
                             cudaGetErrorString(e));
}

void count_launch(int n) { g_launches += n; }

Options &options() {
  static Options o;
  return o;
}

// -------------------------------------------------------------------- Vecs
Vec vec_new(int64_t n) {
  Vec v = new _p_Vec();
  v->n = n;
  QCUDA(cudaMalloc(&v->d, (size_t)n * sizeof(double2)));
  QCUDA(cudaMemset(v->d, 0, (size_t)n * sizeof(double2)));
  return v;
}

void vec_free(Vec v) {
  if (!v) return;
  if (v->d) cudaFree(v->d);
  delete v;
}

int64_t vec_len(Vec v) { return v ? v->n : 0; }

void vec_sync_to_device(Vec v) {
  if (v && v->host_pending) {
    QCUDA(cudaMemcpy(v->d, v->h.data(), (size_t)v->n * sizeof(double2), cudaMemcpyHostToDevice));
    v->host_pending = false;
  }
}

static void vec_pull_host(Vec v) {
  if (!v->host_pending) {
    v->h.resize(v->n);
    QCUDA(cudaMemcpy(v->h.data(), v->d, (size_t)v->n * sizeof(double2), cudaMemcpyDeviceToHost));
  }
}

void Workspace::ensure(int64_t d, int nb) {
  if (dim != d) release();
  dim = d;
  while ((int)bufs.size() < nb) {
    double2 *p = nullptr;
    QCUDA(cudaMalloc(&p, (size_t)d * sizeof(double2)));
    bufs.push_back(p);
  }
  if (!dsum) {
    QCUDA(cudaMalloc(&dsum, 64 * sizeof(double)));
    QCUDA(cudaMallocHost(&hsum, 64 * sizeof(double)));
  }
}

void Workspace::release() {
  for (auto p : bufs) cudaFree(p);
  bufs.clear();
  dim = 0;
}

cudaStream_t stream_of(qsystem qs) {
  if (qs->impl->user_stream) return qs->impl->user_stream;
  if (!qs->impl->stream) QCUDA(cudaStreamCreateWithFlags(&qs->impl->stream, cudaStreamNonBlocking));
  return qs->impl->stream;
}

void ensure_program(qsystem qs) {
  // 0: density matrix, 1: Schroedinger, 2: MCWF effective Hamiltonian
  const int mode = qs->mcwf_solver ? 2 : (qs->dm_equations ? 0 : 1);
  if (qs->impl->prog && qs->impl->prog_mode == mode) return;
  if (qs->impl->prog) {
    qs->impl->prog->release();
    delete qs->impl->prog;
  }
  qs->impl->prog = compile_terms(qs, mode);
  qs->impl->prog_mode = mode;
}

// Cache of operator-product maps uploaded for expectation values.
struct ObsEntry {
  int *map = nullptr;
  double2 *val = nullptr;
};
static std::mutex g_obs_mu;
static std::map<std::pair<int64_t, std::vector<op_handle>>, ObsEntry> g_obs;

static ObsEntry obs_tables(int64_t D, const std::vector<op_handle> &ops) {
  std::lock_guard<std::mutex> lk(g_obs_mu);
  auto key = std::make_pair(D, ops);
  auto it = g_obs.find(key);
  if (it != g_obs.end()) return it->second;
  std::vector<int> map;
  std::vector<cplx> val;
  op_chain_map(D, ops, map, val);
  ObsEntry e;
  QCUDA(cudaMalloc(&e.map, D * sizeof(int)));
  QCUDA(cudaMalloc(&e.val, D * sizeof(double2)));
  QCUDA(cudaMemcpy(e.map, map.data(), D * sizeof(int), cudaMemcpyHostToDevice));
  QCUDA(cudaMemcpy(e.val, val.data(), D * sizeof(double2), cudaMemcpyHostToDevice));
  g_obs[key] = e;
  return e;
}

void ObsMonitor::release() {
  if (dmap) cudaFree(dmap);
  if (dval) cudaFree(dval);
  if (dvalues) cudaFree(dvalues);
  dmap = nullptr;
  dval = nullptr;
  dvalues = nullptr;
  D = 0;
}

static void drop_obs_cache_for(op_handle op) {
  std::lock_guard<std::mutex> lk(g_obs_mu);
  for (auto it = g_obs.begin(); it != g_obs.end();) {
    bool hit = false;
    for (auto p : it->first.second) hit |= (p == op);
    if (hit) {
      cudaFree(it->second.map);
      cudaFree(it->second.val);
      it = g_obs.erase(it);
    } else {
      ++it;
    }
  }
}

static cudaStream_t g_default_stream() {
  static cudaStream_t s = nullptr;
  if (!s) QCUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

}  // namespace quac

using namespace quac;

// gate kernels (gates.cu)
namespace quac {
void launch_gate1(double2 *a, int64_t n, int64_t sr, int64_t sc, const cplx *U, const cplx *W,
                  cudaStream_t s);
void launch_gate2(double2 *a, int64_t n, const int64_t strides[4], const cplx *U, const cplx *W,
                  cudaStream_t s);
}  // namespace quac

extern "C" {

// ------------------------------------------------------------- runtime
static bool g_initialized = false;

void QuaC_initialize(int argc, char **args) {
  g_initialized = true;
  Options &o = options();
  for (int i = 1; i + 1 < argc + 1 && i < argc; i++) {
    const char *a = args[i];
    const char *v = (i + 1 < argc) ? args[i + 1] : "";
    if (!strcmp(a, "-ts_rk_type")) { o.rk_type = v; i++; }
    else if (!strcmp(a, "-quac_rk4_classic")) { o.rk4_classic = true; }
    else if (!strcmp(a, "-ts_adapt_type")) { o.adapt_type = v; i++; }
    else if (!strcmp(a, "-ts_rtol")) { o.rtol = atof(v); o.rtol_set = true; i++; }
    else if (!strcmp(a, "-ts_atol")) { o.atol = atof(v); o.atol_set = true; i++; }
    else if (!strcmp(a, "-ts_max_steps")) { o.max_steps = atoll(v); i++; }
    else if (!strcmp(a, "-ksp_gmres_restart")) { o.gmres_restart = atoi(v); i++; }
    else if (!strcmp(a, "-ksp_rtol")) { o.gmres_rtol = atof(v); i++; }
  }
}

void QuaC_finalize(void) { g_initialized = false; }
static void legacy_clear();
// quac.c:60-80: forgets the legacy global system (its terms and operator
// matrix) so that a program can build a new one; the operators created
// with create_op stay the caller's to destroy, as in the reference
void QuaC_clear(void) { legacy_clear(); }

int PetscPrintf(int comm, const char *fmt, ...) {
  (void)comm;
  va_list ap;
  va_start(ap, fmt);
  int r = vprintf(fmt, ap);
  va_end(ap);
  return r;
}

void quac_set_error_mode(int mode) { g_error_mode = mode; }
const char *quac_last_error(void) { return g_last_error.c_str(); }
void quac_clear_error(void) { g_last_error.clear(); g_has_error = false; }
int64_t quac_kernel_launch_count(void) { return g_launches.load(); }

int quac_set_ts_options(const char *rk_type, const char *adapt_type, double rtol, double atol,
                        PetscInt max_steps) {
  Options &o = options();
  if (rk_type && *rk_type) {
    std::string s(rk_type);
    if (s != "3bs" && s != "4" && s != "5dp" && s != "4classic") { fail(9, "ERROR! unknown rk type %s\n", rk_type); return 1; }
    o.rk4_classic = (s == "4classic");
    o.rk_type = (s == "4classic") ? "4" : s;
  }
  if (adapt_type && *adapt_type) {
    std::string s(adapt_type);
    if (s != "basic" && s != "none") { fail(9, "ERROR! unknown adapt type %s\n", adapt_type); return 1; }
    o.adapt_type = s;
  }
  if (rtol > 0) { o.rtol = rtol; o.rtol_set = true; }
  if (atol > 0) { o.atol = atol; o.atol_set = true; }
  o.max_steps = max_steps;
  return 0;
}

// ------------------------------------------------------- system building
void initialize_system(qsystem *qsys) {
  if (!g_initialized) {
    fail(0, "ERROR! You need to call QuaC_initialize before creating\n       any systems!\n");
    return;
  }
  qsystem q = new qsystem_s();
  memset(q, 0, sizeof(*q));
  q->total_levels = 1;
  q->dim = 1;
  q->np = 1;
  q->nid = 0;
  q->num_circuits = -1;
  q->impl = new qsystem_impl();
  *qsys = q;
}

void clear_mat_terms_sys(qsystem qs) {
  qs->impl->terms.clear();
  release_td_programs(qs);
  qs->impl->td.clear();
  if (qs->impl->prog) {
    qs->impl->prog->release();
    delete qs->impl->prog;
    qs->impl->prog = nullptr;
  }
  qs->impl->prog_mode = -1;
  qs->num_time_indep = 0;
  qs->num_time_dep = 0;
  qs->mat_allocated = 0;
}

void destroy_system(qsystem *qsys) {
  qsystem q = *qsys;
  if (!q) return;
  q->impl->obsmon.release();
  clear_mat_terms_sys(q);
  mcwf_release_system(q);
  precond_release_system(q);
  q->impl->ws.release();
  if (q->impl->host_vec) vec_free(q->impl->host_vec);
  if (q->impl->ws.dsum) cudaFree(q->impl->ws.dsum);
  if (q->impl->ws.hsum) cudaFreeHost(q->impl->ws.hsum);
  if (q->impl->stream) cudaStreamDestroy(q->impl->stream);
  free(q->subsystem_list);
  if (q->circuit_list) free(q->circuit_list);
  delete q->impl;
  delete q;
  *qsys = nullptr;
}

static op_handle new_single_op(PetscInt n_before, PetscInt levels, op_type t) {
  op_handle o = (op_handle)calloc(1, sizeof(*o));
  o->n_before = n_before;
  o->my_levels = levels;
  o->my_op_type = t;
  o->position = -1;
  const double s = 1.0 / std::sqrt(2.0);
  // eigen-data of the Pauli operators (qsystem.c:93-151)
  if (t == SIGMA_Z) {
    o->evals[0] = 1; o->evals[1] = -1;
    o->evecs[0][0] = -1; o->evecs[0][1] = 0; o->evecs[1][0] = 0; o->evecs[1][1] = -1;
  } else if (t == SIGMA_Y) {
    o->evals[0] = -1; o->evals[1] = 1;
    o->evecs[0][0] = -s; o->evecs[0][1] = PetscScalar(0, s);
    o->evecs[1][0] = -s; o->evecs[1][1] = PetscScalar(0, -s);
  } else if (t == SIGMA_X) {
    o->evals[0] = -1; o->evals[1] = 1;
    o->evecs[0][0] = -s; o->evecs[0][1] = s; o->evecs[1][0] = s; o->evecs[1][1] = s;
  }
  return o;
}

static void push_subsystem(qsystem qs, op_handle op, PetscInt levels) {
  qs->subsystem_list =
      (op_handle *)realloc(qs->subsystem_list, (qs->num_subsystems + 1) * sizeof(op_handle));
  op->pos_in_sys_hspace = qs->num_subsystems;
  qs->subsystem_list[qs->num_subsystems++] = op;
  qs->total_levels *= levels;
}

static void make_family(PetscInt n_before, PetscInt levels, op_handle base) {
  op_handle a = base;
  a->dag = new_single_op(n_before, levels, RAISE);
  a->dag->dag = a;
  a->n = new_single_op(n_before, levels, NUMBER);
  a->n->dag = a->n;
  a->eye = new_single_op(n_before, levels, IDENTITY);
  a->eye->dag = a->eye;
  a->sig_x = new_single_op(n_before, levels, SIGMA_X);
  a->sig_x->dag = a->sig_x;
  a->sig_z = new_single_op(n_before, levels, SIGMA_Z);
  a->sig_z->dag = a->sig_z;
  a->sig_y = new_single_op(n_before, levels, SIGMA_Y);
  a->sig_y->dag = a->sig_y;
  a->other = new_single_op(n_before, levels, OTHER);
  a->other->dag = a->other;
}

void create_op_sys(qsystem qs, PetscInt levels, op_handle *new_op) {
  if (qs->hspace_frozen) {
    fail(0, "ERROR! You cannot add more operators after\n       the creating a dm or constructing the matrix!\n");
    return;
  }
  op_handle a = new_single_op(qs->total_levels, levels, LOWER);
  make_family(qs->total_levels, levels, a);
  push_subsystem(qs, a, levels);
  *new_op = a;
}

void destroy_op_sys(op_handle *op) {
  op_handle a = *op;
  if (!a) return;
  op_handle fam[] = {a->dag, a->n, a->eye, a->sig_x, a->sig_z, a->sig_y, a->other, a};
  for (op_handle f : fam) { drop_obs_cache_for(f); free(f); }
  *op = nullptr;
}

void create_vec_op_sys(qsystem qs, PetscInt levels, vec_op *new_vec) {
  if (qs->hspace_frozen) {
    fail(0, "ERROR! You cannot add more vec_ops after\n       the creating a dm or constructing the matrix!\n");
    return;
  }
  vec_op v = (vec_op)calloc(levels, sizeof(op_handle));
  for (PetscInt i = 0; i < levels; i++) {
    op_handle o = new_single_op(qs->total_levels, levels, VEC);
    o->position = i;
    o->eye = new_single_op(qs->total_levels, levels, IDENTITY);
    o->sig_x = new_single_op(qs->total_levels, levels, SIGMA_X);
    o->sig_z = new_single_op(qs->total_levels, levels, SIGMA_Z);
    o->sig_y = new_single_op(qs->total_levels, levels, SIGMA_Y);
    o->other = new_single_op(qs->total_levels, levels, OTHER);
    v[i] = o;
  }
  v[0]->vec_op_list = v;
  push_subsystem(qs, v[0], levels);
  *new_vec = v;
}

void destroy_vec_op_sys(vec_op *vop) {
  vec_op v = *vop;
  if (!v) return;
  PetscInt L = v[0]->my_levels;
  for (PetscInt i = 0; i < L; i++) {
    op_handle fam[] = {v[i]->eye, v[i]->sig_x, v[i]->sig_z, v[i]->sig_y, v[i]->other, v[i]};
    for (op_handle f : fam) { drop_obs_cache_for(f); free(f); }
  }
  free(v);
  *vop = nullptr;
}

void set_init_excited_op(op_handle op, PetscInt initial_exc) {
  if (initial_exc >= op->my_levels && op->my_op_type != VEC) {
    fail(0, "ERROR! The initial excitation level must be less than the number of levels and can't be used for VEC_OP!\n");
    return;
  }
  op->initial_exc = initial_exc;
}

static void record_term(qsystem qs, int kind, PetscScalar a, PetscInt num_ops, op_handle *ops) {
  Term t;
  t.kind = kind;
  t.a = cplx(a.real(), a.imag());
  for (PetscInt i = 0; i < num_ops; i++) {
    if (!ops[i]) { fail(9, "ERROR! NULL operator passed to a term\n"); return; }
    t.ops.push_back(ops[i]);
  }
  if (kind == 2) qs->dm_equations = PETSC_TRUE;
  qs->impl->terms.push_back(t);
  qs->num_time_indep = (PetscInt)qs->impl->terms.size();
  if (qs->impl->prog) {  // terms changed after construct_matrix: rebuild lazily
    qs->impl->prog->release();
    delete qs->impl->prog;
    qs->impl->prog = nullptr;
  }
}

void add_ham_term(qsystem qs, PetscScalar a, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops);
  va_list ap;
  va_start(ap, num_ops);
  for (PetscInt i = 0; i < num_ops; i++) ops[i] = va_arg(ap, op_handle);
  va_end(ap);
  record_term(qs, 1, a, num_ops, ops.data());
}

void add_lin_term(qsystem qs, PetscScalar a, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops);
  va_list ap;
  va_start(ap, num_ops);
  for (PetscInt i = 0; i < num_ops; i++) ops[i] = va_arg(ap, op_handle);
  va_end(ap);
  record_term(qs, 2, a, num_ops, ops.data());
}

void add_lin_term_list(qsystem qs, PetscScalar a, PetscInt num_ops, op_handle *ops) {
  record_term(qs, 2, a, num_ops, ops);
}

void add_ham_term_list(qsystem qs, PetscScalar a, PetscInt num_ops, op_handle *ops) {
  record_term(qs, 1, a, num_ops, ops);
}

static void record_td_term(qsystem qs, int kind, PetscScalar a, void *ctx, quac_time_dep_func f,
                           quac_time_dep_func_parts g, PetscInt num_ops, op_handle *ops) {
  if (!f && !g) { fail(9, "ERROR! NULL time-dependence function passed to a time-dependent term\n"); return; }
  TdTerm td;
  td.term.kind = kind;
  td.term.a = cplx(PetscRealPart(a), PetscImaginaryPart(a));
  for (PetscInt i = 0; i < num_ops; i++) {
    if (!ops[i]) { fail(9, "ERROR! NULL operator passed to a term\n"); return; }
    td.term.ops.push_back(ops[i]);
  }
  td.f = f;
  td.g = g;
  td.ctx = ctx;
  if (kind == 2) qs->dm_equations = PETSC_TRUE;  // qsystem.c:531
  qs->impl->td.push_back(td);
  qs->num_time_dep = (PetscInt)qs->impl->td.size();
}

void add_ham_term_time_dep(qsystem qs, PetscScalar a, void *ctx, quac_time_dep_func f, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops);
  va_list ap;
  va_start(ap, num_ops);
  for (PetscInt i = 0; i < num_ops; i++) ops[i] = va_arg(ap, op_handle);
  va_end(ap);
  record_td_term(qs, 1, a, ctx, f, nullptr, num_ops, ops.data());
}

void add_lin_term_time_dep(qsystem qs, PetscScalar a, void *ctx, quac_time_dep_func f, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops);
  va_list ap;
  va_start(ap, num_ops);
  for (PetscInt i = 0; i < num_ops; i++) ops[i] = va_arg(ap, op_handle);
  va_end(ap);
  record_td_term(qs, 2, a, ctx, f, nullptr, num_ops, ops.data());
}

int quac_add_term_time_dep_list(qsystem qs, int kind, PetscScalar a, void *ctx, quac_time_dep_func_parts g,
                                PetscInt num_ops, op_handle *ops) {
  if (kind != 1 && kind != 2) { fail(0, "ERROR! term kind must be 1 (Hamiltonian) or 2 (Lindblad)\n"); return 1; }
  record_td_term(qs, kind, a, ctx, nullptr, g, num_ops, ops);
  return has_error() ? 1 : 0;
}

void use_mcwf_solver(qsystem qs, PetscInt num_tot_trajs, PetscInt seed) {
  if (qs->hspace_frozen) {
    fail(9, "ERROR! use_mcwf_solver must be called before construct_matrix or create_qvec_sys!\n");
    return;
  }
  if (!qs->dm_equations) {
    fail(9, "ERROR! use_mcwf_solver must be used with a Lindblad term!\n");
    return;
  }
  if (num_tot_trajs < 2) {
    fail(9, "ERROR! use_mcwf_solver must be called with more than 2 num_tot_trajs!\n");
    return;
  }
  if (num_tot_trajs > (1 << 30)) { fail(9, "ERROR! num_tot_trajs too large\n"); return; }
  uint64_t sd = (uint64_t)seed;
  if (seed == 0) {  // the reference draws a seed (make_sprng_seed) when given NULL
    std::random_device rd;
    sd = ((uint64_t)rd() << 32) ^ rd();
  }
  qs->hspace_frozen = PETSC_TRUE;
  qs->mcwf_solver = PETSC_TRUE;
  qs->impl->mcwf_seed = sd;
  qs->impl->mcwf_ntraj = num_tot_trajs;
  if (qs->impl->prog) {
    qs->impl->prog->release();
    delete qs->impl->prog;
    qs->impl->prog = nullptr;
  }
}

void construct_matrix(qsystem qs) {
  qs->hspace_frozen = 1;
  if (qs->num_subsystems == 0) {
    fail(0, "ERROR! You need to create operators before you construct\n       a matrix!\n");
    return;
  }
  if (qs->impl->terms.empty() && qs->impl->td.empty()) {
    fail(0, "ERROR! You need to add some terms before you construct\n       a matrix!\n");
    return;
  }
  // the MCWF solver works in the wavefunction space (qsystem.c:613-619)
  qs->dim = (qs->dm_equations && !qs->mcwf_solver) ? qs->total_levels * qs->total_levels : qs->total_levels;
  ensure_program(qs);
  qs->mat_allocated = 1;
}

// ---------------------------------------------------------------- qvecs
static qvec new_qvec(qvec_type t, PetscInt n, PetscInt total_levels, PetscInt ndims,
                     const PetscInt *dims) {
  qvec q = (qvec)calloc(1, sizeof(*q));
  q->my_type = t;
  q->n = n;
  q->Istart = 0;
  q->Iend = n;
  q->total_levels = total_levels;
  q->ndims_hspace = ndims;
  q->n_ops = ndims;
  q->hspace_dims = (PetscInt *)malloc(ndims * sizeof(PetscInt));
  for (PetscInt i = 0; i < ndims; i++) q->hspace_dims[i] = dims[i];
  q->n_ensemble = -1;
  q->ens_i = -1;
  q->data = vec_new(n);
  return q;
}

void create_dm_sys(qsystem qs, qvec *out) {
  if (qs->num_subsystems == 0) {
    fail(0, "ERROR! You need to create operators before you construct\n       a density matrix!\n");
    return;
  }
  qs->dm_equations = 1;
  qs->dim = qs->total_levels * qs->total_levels;
  qs->hspace_frozen = 1;
  std::vector<PetscInt> dims(2 * qs->num_subsystems);
  for (PetscInt i = 0; i < qs->num_subsystems; i++)
    dims[i] = dims[i + qs->num_subsystems] = qs->subsystem_list[i]->my_levels;
  *out = new_qvec(DENSITY_MATRIX, qs->dim, qs->total_levels, 2 * qs->num_subsystems, dims.data());
  (*out)->n_ops = qs->num_subsystems;
}

void create_wf_sys(qsystem qs, qvec *out) {
  if (qs->num_subsystems == 0) {
    fail(0, "ERROR! You need to crveate operators before you construct\n       a wavefunction!\n");
    return;
  }
  if (qs->dm_equations) {
    fail(0, "ERROR!\nMust use density matrices if Lindblad terms are used without using mcwf_solver.\n");
    return;
  }
  qs->dim = qs->total_levels;
  qs->hspace_frozen = 1;
  std::vector<PetscInt> dims(qs->num_subsystems);
  for (PetscInt i = 0; i < qs->num_subsystems; i++) dims[i] = qs->subsystem_list[i]->my_levels;
  *out = new_qvec(WAVEFUNCTION, qs->dim, qs->total_levels, qs->num_subsystems, dims.data());
}

// WF_ENSEMBLE of the MCWF solver (qvec_utilities.c:790-830): data is the
// initial wavefunction; the trajectories are spawned from it by the first
// time_step_sys
static void create_wf_ens_sys(qsystem qs, qvec *out) {
  qs->dim = qs->total_levels;
  qs->hspace_frozen = 1;
  std::vector<PetscInt> dims(qs->num_subsystems);
  for (PetscInt i = 0; i < qs->num_subsystems; i++) dims[i] = qs->subsystem_list[i]->my_levels;
  *out = new_qvec(WF_ENSEMBLE, qs->total_levels, qs->total_levels, qs->num_subsystems, dims.data());
  (*out)->n_ensemble = qs->impl->mcwf_ntraj;
  (*out)->ens_spawned = PETSC_FALSE;
}

void create_qvec_sys(qsystem qs, qvec *out) {
  if (qs->mcwf_solver) create_wf_ens_sys(qs, out);
  else if (qs->dm_equations) create_dm_sys(qs, out);
  else create_wf_sys(qs, out);
}

void create_arb_qvec(qvec *out, PetscInt nstates, qvec_type t) {
  if (t == WAVEFUNCTION) {
    *out = new_qvec(t, nstates, nstates, 1, &nstates);
  } else if (t == DENSITY_MATRIX) {
    PetscInt L = (PetscInt)std::llround(std::sqrt((double)nstates));
    if (L * L != nstates) { fail(9, "ERROR! n for DENSITY_MATRIX must be perfect square!\n"); return; }
    PetscInt dims[2] = {L, L};
    *out = new_qvec(t, nstates, L, 2, dims);
    (*out)->ndims_hspace = 1;
    (*out)->n_ops = 1;
  } else {
    fail(9, "ERROR! Type not understood in create_arb_qvec.\n");
  }
}

void destroy_qvec(qvec *q) {
  if (!*q) return;
  mcwf_release(*q);
  free((*q)->hspace_dims);
  vec_free((*q)->data);
  free(*q);
  *q = nullptr;
}

void add_to_qvec_loc(qvec q, PetscScalar alpha, PetscInt loc) {
  if (loc > q->n || loc < 0) { fail(0, "ERROR! Adding to a qvec location that is out of range!\n"); return; }
  if (loc == q->n) return;  // passes the reference's range check but no rank owns it: nothing is added
  Vec v = q->data;
  if (!v->host_pending) { vec_pull_host(v); v->host_pending = true; }
  v->h[loc] += cplx(alpha.real(), alpha.imag());
}

void add_to_qvec(qvec q, PetscScalar alpha, ...) {
  va_list ap;
  va_start(ap, alpha);
  PetscInt loc = va_arg(ap, PetscInt);
  if (q->my_type == DENSITY_MATRIX) {
    PetscInt loc2 = va_arg(ap, PetscInt);
    loc = (PetscInt)std::llround(std::sqrt((double)q->n)) * loc + loc2;  // D*col + row
  }
  va_end(ap);
  add_to_qvec_loc(q, alpha, loc);
}

// qvec_utilities.c:996-1033: the vector index of the basis state with op
// i in Fock state fock_states[i] and every other subsystem in 0, as the
// reference computes it: sum_i fock_i * n_before_i (its strides are the
// levels BEFORE each subsystem, which is the position of that digit only
// when subsystem 0 is the least significant, a quirk kept for parity), and
// the diagonal element (loc, loc) of a density matrix.
void get_qvec_loc_fock_op_list(qvec q, PetscInt *loc, PetscInt num_ops, op_handle *ops, PetscInt *fock_states) {
  *loc = 0;
  for (PetscInt i = 0; i < num_ops; i++) {
    if (fock_states[i] >= ops[i]->my_levels || fock_states[i] < 0) {
      fail(0, "ERROR! The Fock State must be less than the number of levels and greater than 0!\n");
      return;
    }
    *loc += fock_states[i] * ops[i]->n_before;
  }
  if (q->my_type == DENSITY_MATRIX) {
    *loc = (PetscInt)std::llround(std::sqrt((double)q->n)) * *loc + *loc;
  } else if (q->my_type != WAVEFUNCTION && q->my_type != WF_ENSEMBLE) {
    fail(0, "ERROR! qvec type not understood.");
  }
}

// qvec_utilities.c:973-994: (op, fock state) pairs as variadic arguments
void get_qvec_loc_fock_op(qvec q, PetscInt *loc, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops > 0 ? num_ops : 0);
  std::vector<PetscInt> fock(ops.size());
  va_list ap;
  va_start(ap, num_ops);
  for (size_t i = 0; i < ops.size(); i++) {
    ops[i] = va_arg(ap, op_handle);
    fock[i] = (PetscInt)(int32_t)va_arg(ap, PetscInt);  // an int or a PetscInt argument
  }
  va_end(ap);
  get_qvec_loc_fock_op_list(q, loc, num_ops, ops.data(), fock.data());
}

// qvec_utilities.c:832-872: alpha added at that basis state
void add_to_qvec_fock_op_list(PetscScalar alpha, qvec q, PetscInt num_ops, op_handle *ops, PetscInt *fock_states) {
  PetscInt loc = 0;
  get_qvec_loc_fock_op_list(q, &loc, num_ops, ops, fock_states);
  if (!has_error()) add_to_qvec_loc(q, alpha, loc);
}

void add_to_qvec_fock_op(PetscScalar alpha, qvec q, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops > 0 ? num_ops : 0);
  std::vector<PetscInt> fock(ops.size());
  va_list ap;
  va_start(ap, num_ops);
  for (size_t i = 0; i < ops.size(); i++) {
    ops[i] = va_arg(ap, op_handle);
    fock[i] = (PetscInt)(int32_t)va_arg(ap, PetscInt);  // an int or a PetscInt argument
  }
  va_end(ap);
  add_to_qvec_fock_op_list(alpha, q, num_ops, ops.data(), fock.data());
}

void assemble_qvec(qvec q) { vec_sync_to_device(q->data); }

void set_qvec_from_init_excited_op(qsystem qs, qvec q) {
  PetscInt row = 0;
  for (PetscInt i = 0; i < qs->num_subsystems; i++) {
    op_handle s = qs->subsystem_list[i];
    PetscInt n_after = qs->total_levels / (s->my_levels * s->n_before);
    row += s->initial_exc * n_after;
  }
  if (qs->dm_equations) row = qs->total_levels * row + row;
  add_to_qvec_loc(q, PetscScalar(1.0, 0.0), row);
}

static PetscScalar read_element(qvec q, PetscInt loc) {
  Vec v = q->data;
  if (v->host_pending) return PetscScalar(v->h[loc].real(), v->h[loc].imag());
  double2 x;
  QCUDA(cudaMemcpy(&x, v->d + loc, sizeof(double2), cudaMemcpyDeviceToHost));
  return PetscScalar(x.x, x.y);
}

void get_dm_element_qvec(qvec q, PetscInt row, PetscInt col, PetscScalar *val) {
  PetscInt D = (PetscInt)std::llround(std::sqrt((double)q->n));
  *val = read_element(q, D * col + row);
}

void get_wf_element_qvec(qvec q, PetscInt loc, PetscScalar *val) { *val = read_element(q, loc); }

void get_trace_qvec(qvec q, PetscScalar *val) {
  if (q->my_type != DENSITY_MATRIX) { fail(0, "ERROR! Can only take the trace of density matrices!\n"); return; }
  vec_sync_to_device(q->data);
  PetscInt D = (PetscInt)std::llround(std::sqrt((double)q->n));
  cplx t = dm_trace(q->data->d, D, g_default_stream());
  *val = PetscScalar(t.real(), t.imag());
}

void get_expectation_value_qvec_list(qvec q, PetscScalar *val, PetscInt num_ops, op_handle *ops) {
  vec_sync_to_device(q->data);
  std::vector<op_handle> v(ops, ops + num_ops);
  if (q->my_type == DENSITY_MATRIX) {
    PetscInt D = (PetscInt)std::llround(std::sqrt((double)q->n));
    ObsEntry e = obs_tables(D, v);
    cplx r = dm_expectation(q->data->d, D, e.map, e.val, g_default_stream());
    *val = PetscScalar(r.real(), r.imag());
  } else if (q->my_type == WAVEFUNCTION || (q->my_type == WF_ENSEMBLE && !mcwf_spawned(q))) {
    ObsEntry e = obs_tables(q->n, v);
    cplx r = wf_expectation(q->data->d, q->n, e.map, e.val, g_default_stream());
    *val = PetscScalar(r.real(), r.imag());
  } else if (q->my_type == WF_ENSEMBLE) {
    ObsEntry e = obs_tables(q->n, v);
    cplx r = mcwf_expectation(q, e.map, e.val);
    *val = PetscScalar(r.real(), r.imag());
  } else {
    fail(0, "ERROR! qvec type not understood.");
  }
}

void get_expectation_value_qvec(qvec q, PetscScalar *val, PetscInt num_ops, ...) {
  std::vector<op_handle> ops(num_ops);
  va_list ap;
  va_start(ap, num_ops);
  for (PetscInt i = 0; i < num_ops; i++) ops[i] = va_arg(ap, op_handle);
  va_end(ap);
  get_expectation_value_qvec_list(q, val, num_ops, ops.data());
}

void get_fidelity_qvec(qvec q1, qvec q2, PetscReal *fidelity, PetscReal *var) {
  *var = 0;
  vec_sync_to_device(q1->data);
  vec_sync_to_device(q2->data);
  cudaStream_t s = g_default_stream();
  if (q1->my_type == WAVEFUNCTION && q2->my_type == WAVEFUNCTION) {
    cplx d = vdot(q1->data->d, q2->data->d, q1->n, s);
    *fidelity = std::norm(d);
  } else if (q1->my_type == DENSITY_MATRIX && q2->my_type == WAVEFUNCTION) {
    if (q1->n != q2->n * q2->n) { fail(0, "ERROR! The input density matrix and wavefunction are not compatible!\n"); return; }
    *fidelity = dm_wf_fidelity(q1->data->d, q2->data->d, q2->n, s);
  } else if (q2->my_type == DENSITY_MATRIX && q1->my_type == WAVEFUNCTION) {
    if (q2->n != q1->n * q1->n) { fail(0, "ERROR! The input density matrix and wavefunction are not compatible!\n"); return; }
    *fidelity = dm_wf_fidelity(q2->data->d, q1->data->d, q1->n, s);
  } else {
    fail(9, "Types not understand in get_fidelity_qvec!\n");
  }
}

void get_bitstring_probs(qvec q, PetscInt *nloc, PetscReal **probs, PetscReal **vars) {
  vec_sync_to_device(q->data);
  PetscInt D = q->my_type == DENSITY_MATRIX ? (PetscInt)std::llround(std::sqrt((double)q->n)) : q->n;
  std::vector<cplx> h(q->n);
  QCUDA(cudaMemcpy(h.data(), q->data->d, q->n * sizeof(double2), cudaMemcpyDeviceToHost));
  *nloc = D;
  *probs = (PetscReal *)malloc(D * sizeof(PetscReal));
  *vars = (PetscReal *)calloc(D, sizeof(PetscReal));
  for (PetscInt i = 0; i < D; i++)
    (*probs)[i] = q->my_type == DENSITY_MATRIX ? h[i * D + i].real() : std::norm(h[i]);
}

void copy_qvec(qvec src, qvec dst) {
  if (src->n != dst->n) { fail(0, "ERROR! qvecs are not the same size in copy_qvec\n"); return; }
  vec_sync_to_device(src->data);
  QCUDA(cudaMemcpy(dst->data->d, src->data->d, src->n * sizeof(double2), cudaMemcpyDeviceToDevice));
  dst->data->host_pending = false;
}

void print_qvec(qvec q) {
  vec_sync_to_device(q->data);
  std::vector<cplx> h(q->n);
  QCUDA(cudaMemcpy(h.data(), q->data->d, q->n * sizeof(double2), cudaMemcpyDeviceToHost));
  if (q->my_type == DENSITY_MATRIX) {
    PetscInt D = (PetscInt)std::llround(std::sqrt((double)q->n));
    for (PetscInt r = 0; r < D; r++) {
      for (PetscInt c = 0; c < D; c++) printf("%4.3e + %4.3ei ", h[c * D + r].real(), h[c * D + r].imag());
      printf("\n");
    }
  } else {
    for (PetscInt i = 0; i < q->n; i++) printf("%e + %ei\n", h[i].real(), h[i].imag());
  }
}

// PETSc binary Vec I/O (qvec_utilities.c:97-167): big-endian int64 class
// id 1211214, int64 n, then n complex128.
static uint64_t bswap64(uint64_t x) { return __builtin_bswap64(x); }

static bool read_petsc_vec(const char *fn, std::vector<cplx> &out) {
  FILE *f = fopen(fn, "rb");
  if (!f) return false;
  uint64_t hdr[2];
  if (fread(hdr, 8, 2, f) != 2) { fclose(f); return false; }
  if ((int64_t)bswap64(hdr[0]) != 1211214) { fclose(f); return false; }
  int64_t n = (int64_t)bswap64(hdr[1]);
  std::vector<uint64_t> raw(2 * n);
  bool ok = fread(raw.data(), 8, 2 * n, f) == (size_t)(2 * n);
  fclose(f);
  if (!ok) return false;
  out.resize(n);
  for (int64_t i = 0; i < n; i++) {
    uint64_t re = bswap64(raw[2 * i]), im = bswap64(raw[2 * i + 1]);
    double dr, di;
    memcpy(&dr, &re, 8);
    memcpy(&di, &im, 8);
    out[i] = cplx(dr, di);
  }
  return true;
}

static void load_into(qvec q, const std::vector<cplx> &h) {
  QCUDA(cudaMemcpy(q->data->d, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice));
}

void read_qvec_dm_binary(qvec *q, const char filename[]) {
  std::vector<cplx> h;
  if (!read_petsc_vec(filename, h)) { fail(9, "ERROR! could not read PETSc binary vector %s\n", filename); return; }
  create_arb_qvec(q, (PetscInt)h.size(), DENSITY_MATRIX);
  if (*q) load_into(*q, h);
}

void read_qvec_wf_binary(qvec *q, const char filename[]) {
  std::vector<cplx> h;
  if (!read_petsc_vec(filename, h)) { fail(9, "ERROR! could not read PETSc binary vector %s\n", filename); return; }
  create_arb_qvec(q, (PetscInt)h.size(), WAVEFUNCTION);
  if (*q) load_into(*q, h);
}

void print_qvec_file(qvec q, char filename[]) {
  vec_sync_to_device(q->data);
  std::vector<cplx> h(q->n);
  QCUDA(cudaMemcpy(h.data(), q->data->d, q->n * sizeof(double2), cudaMemcpyDeviceToHost));
  FILE *f = fopen(filename, "wb");
  if (!f) { fail(9, "ERROR! could not open %s\n", filename); return; }
  uint64_t hdr[2] = {bswap64(1211214), bswap64((uint64_t)q->n)};
  fwrite(hdr, 8, 2, f);
  for (auto &z : h) {
    double d[2] = {z.real(), z.imag()};
    uint64_t u[2];
    memcpy(u, d, 16);
    u[0] = bswap64(u[0]);
    u[1] = bswap64(u[1]);
    fwrite(u, 8, 2, f);
  }
  fclose(f);
}

void *quac_qvec_device_ptr(qvec q) {
  vec_sync_to_device(q->data);
  return q->data->d;
}

// ------------------------------------------------------------ PETSc shims
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) {
  if (!v->host_pending) vec_pull_host(v);
  v->host_pending = true;
  v->host_mapped = true;
  *a = reinterpret_cast<PetscScalar *>(v->h.data());
  return 0;
}

PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) {
  v->host_mapped = false;
  vec_sync_to_device(v);
  if (a) *a = nullptr;
  return 0;
}

PetscErrorCode VecGetSize(Vec v, PetscInt *n) { *n = v->n; return 0; }

PetscErrorCode VecCreateSeq(int comm, PetscInt n, Vec *v) { (void)comm; *v = vec_new(n); return 0; }

PetscErrorCode VecDuplicate(Vec v, Vec *out) { *out = vec_new(v->n); return 0; }

PetscErrorCode VecCopy(Vec src, Vec dst) {
  vec_sync_to_device(src);
  QCUDA(cudaMemcpy(dst->d, src->d, src->n * sizeof(double2), cudaMemcpyDeviceToDevice));
  dst->host_pending = false;
  return 0;
}

PetscErrorCode VecDestroy(Vec *v) { vec_free(*v); *v = nullptr; return 0; }

PetscErrorCode TSGetTime(TS ts, PetscReal *t) { *t = ts->t; return 0; }
PetscErrorCode TSGetTimeStep(TS ts, PetscReal *dt) { *dt = ts->dt; return 0; }

// ------------------------------------------------------------ circuits
void create_circuit(circuit *circ, PetscInt num_gates) {
  circ->start_time = 0.0;
  circ->num_gates = 0;
  circ->gate_list_size = num_gates;
  circ->current_gate = 0;
  circ->num_layers = 0;
  circ->current_layer = 0;
  circ->gate_list = (struct quantum_gate_struct *)calloc(num_gates > 0 ? num_gates : 1,
                                                         sizeof(struct quantum_gate_struct));
  circ->layer_list = (struct gate_layer_struct *)calloc(num_gates > 0 ? num_gates : 1,
                                                         sizeof(struct gate_layer_struct));
}

void destroy_circuit(circuit *circ) {
  for (PetscInt i = 0; i < circ->num_gates; i++) free(circ->gate_list[i].qubit_numbers);
  for (PetscInt i = 0; i < circ->num_layers; i++) free(circ->layer_list[i].gate_list);
  free(circ->gate_list);
  free(circ->layer_list);
  circ->gate_list = nullptr;
  circ->layer_list = nullptr;
  circ->num_gates = 0;
}

static int gate_nqubits(gate_type g) {
  switch (g) {
    case HADAMARD: case SIGMAX: case SIGMAY: case SIGMAZ: case EYE: case RZ: case RX: case RY:
    case U1: case U2: case U3: case CUSTOM1QGATE:
      return 1;
    case CZ_ARP: case CNOT: case CXZ: case CZ: case CmZ: case CZX: case CUSTOM2QGATE: case SQiSWP:
      return 2;
    default:
      return 0;
  }
}

// Reads qubits (int) then the parameters the gate takes (quantum_circuits.c:203-250).
static bool read_gate_args(struct quantum_gate_struct &g, gate_type t, va_list ap) {
  int nq = gate_nqubits(t);
  if (!nq) { fail(0, "ERROR! Gate type not recognized\n"); return false; }
  g.my_gate_type = t;
  g.num_qubits = nq;
  g.qubit_numbers = (PetscInt *)malloc(nq * sizeof(PetscInt));
  for (int i = 0; i < nq; i++) g.qubit_numbers[i] = va_arg(ap, int);
  g.theta = g.phi = g.lambda = 0;
  g.gate_ctx = nullptr;
  g.custom_func = nullptr;
  if (t == RX || t == RY || t == RZ) {
    g.theta = va_arg(ap, PetscReal);
  } else if (t == U3 || t == U2 || t == U1) {
    g.theta = va_arg(ap, PetscReal);
    g.phi = va_arg(ap, PetscReal);
    g.lambda = va_arg(ap, PetscReal);
  } else if (t == CUSTOM1QGATE || t == CUSTOM2QGATE) {
    g.gate_ctx = va_arg(ap, void *);
    g.custom_func = va_arg(ap, custom_gate_func_type);
  }
  return true;
}

void add_gate_to_circuit_sys(circuit *circ, PetscReal time, gate_type t, ...) {
  if (circ->num_gates == circ->gate_list_size) { fail(1, "ERROR! Gate list not large enough!\n"); return; }
  struct quantum_gate_struct &g = circ->gate_list[circ->num_gates];
  va_list ap;
  va_start(ap, t);
  bool ok = read_gate_args(g, t, ap);
  va_end(ap);
  if (!ok) return;
  g.time = time;
  g.run_time = -1;
  circ->num_gates++;
}

}  // extern "C"

// ------------------------------------------------------- gate application
namespace quac {

static void gate1_matrix(const struct quantum_gate_struct &g, cplx U[4]) {
  const double th = g.theta, ph = g.phi, la = g.lambda;
  const double c = std::cos(th / 2), s = std::sin(th / 2);
  const cplx I(0, 1);
  const double r = 1.0 / std::sqrt(2.0);
  switch (g.my_gate_type) {
    case HADAMARD: U[0] = r; U[1] = r; U[2] = r; U[3] = -r; break;
    case SIGMAX: U[0] = 0; U[1] = 1; U[2] = 1; U[3] = 0; break;
    case SIGMAY: U[0] = 0; U[1] = -I; U[2] = I; U[3] = 0; break;
    case SIGMAZ: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = -1; break;
    case EYE: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = 1; break;
    case RX: U[0] = c; U[1] = -I * s; U[2] = -I * s; U[3] = c; break;
    case RY: U[0] = c; U[1] = -s; U[2] = s; U[3] = c; break;
    case RZ: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = std::exp(I * th); break;
    case U1: case U2: case U3:
      U[0] = c; U[1] = -std::exp(I * la) * s; U[2] = std::exp(I * ph) * s;
      U[3] = std::exp(I * (la + ph)) * c;
      break;
    case CUSTOM1QGATE: {
      custom_gate_data *d = (custom_gate_data *)g.gate_ctx;
      if (!d) { fail(0, "ERROR! CUSTOM1QGATE needs its gate data\n"); return; }
      for (int k = 0; k < 4; k++) U[k] = cplx(d->gate_data[k / 2][k % 2].real(), d->gate_data[k / 2][k % 2].imag());
      break;
    }
    default: U[0] = 1; U[1] = 0; U[2] = 0; U[3] = 1; break;
  }
}

// 4x4 in the basis 2*d(q0) + d(q1) with q0 = qubit_numbers[0] (control).
static void gate2_matrix(const struct quantum_gate_struct &g, cplx U[16]) {
  for (int k = 0; k < 16; k++) U[k] = 0;
  const double r = 1.0 / std::sqrt(2.0);
  const cplx I(0, 1);
  switch (g.my_gate_type) {
    case CNOT: U[0] = 1; U[5] = 1; U[11] = 1; U[14] = 1; break;
    case CXZ: U[0] = 1; U[5] = 1; U[11] = -1; U[14] = 1; break;
    case CZX: U[0] = 1; U[5] = 1; U[11] = 1; U[14] = -1; break;
    case CmZ: U[0] = 1; U[5] = 1; U[10] = -1; U[15] = 1; break;
    case CZ: U[0] = 1; U[5] = 1; U[10] = 1; U[15] = -1; break;
    case CZ_ARP: U[0] = 1; U[5] = -1; U[10] = -1; U[15] = -1; break;
    case SQiSWP: U[0] = 1; U[5] = r; U[6] = I * r; U[9] = I * r; U[10] = r; U[15] = 1; break;
    default: U[0] = U[5] = U[10] = U[15] = 1; break;
  }
}

// Superoperator engine: qubit q = subsystem q, digit stride n_after.
void apply_gate_superop(qsystem qs, const struct quantum_gate_struct &g, Vec v, bool is_dm,
                        cudaStream_t s) {
  const int64_t D = qs->total_levels;
  const int64_t n = v->n;
  auto stride = [&](PetscInt q) -> int64_t {
    if (q < 0 || q >= qs->num_subsystems) { fail(0, "ERROR! qubit index out of range\n"); return 0; }
    op_handle o = qs->subsystem_list[q];
    if (o->my_levels != 2) { fail(0, "ERROR! Single qubit gates can only affect 2-level systems\n"); return 0; }
    return D / (o->my_levels * o->n_before);
  };
  if (g.num_qubits == 1) {
    if (g.my_gate_type == CUSTOM1QGATE) { fail(0, "ERROR! CUSTOM1QGATE has no superoperator form\n"); return; }
    cplx U[4], W[4];
    gate1_matrix(g, U);
    for (int k = 0; k < 4; k++) W[k] = std::conj(U[k]);
    int64_t st = stride(g.qubit_numbers[0]);
    if (has_error()) return;
    launch_gate1(v->d, n, st, is_dm ? st * D : 0, U, is_dm ? W : nullptr, s);
  } else {
    int64_t s0 = stride(g.qubit_numbers[0]), s1 = stride(g.qubit_numbers[1]);
    if (has_error()) return;
    if (s0 == s1) { fail(0, "ERROR! two-qubit gate on a single qubit\n"); return; }
    if (g.my_gate_type == CUSTOM2QGATE && !g.custom_func) { fail(0, "ERROR! CUSTOM2QGATE needs its function\n"); return; }
    cplx U[16], W[16];
    if (g.my_gate_type == CUSTOM2QGATE) {
      // the user function is evaluated in the significance-ordered basis
      // (quantum_circuits.c:1700-1760 with 2903-2953)
      const bool swap = qs->subsystem_list[g.qubit_numbers[1]]->n_before <
                        qs->subsystem_list[g.qubit_numbers[0]]->n_before;
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          PetscScalar val;
          g.custom_func(&val, i, j, g.gate_ctx);
          // kernel basis is 2*d(q0)+d(q1); significance basis swaps when q1 is more significant
          int ki = swap ? ((i & 1) << 1 | (i >> 1)) : i;
          int kj = swap ? ((j & 1) << 1 | (j >> 1)) : j;
          U[ki * 4 + kj] = cplx(val.real(), val.imag());
        }
    } else {
      gate2_matrix(g, U);
    }
    for (int k = 0; k < 16; k++) W[k] = std::conj(U[k]);
    int64_t st[4] = {s0, s1, is_dm ? s0 * D : 0, is_dm ? s1 * D : 0};
    launch_gate2(v->d, n, st, U, is_dm ? W : nullptr, s);
  }
}

// In-place engine (_apply_gate2): strides from the qvec's hspace_dims.
void apply_gate_inplace(qvec q, const struct quantum_gate_struct &g, cudaStream_t s) {
  Vec v = q->data;
  const int64_t n = v->n;
  const bool dm = q->my_type == DENSITY_MATRIX;
  const PetscInt half = q->ndims_hspace / 2;
  auto nbef = [&](PetscInt qq) -> int64_t {
    int64_t p = 1;
    for (PetscInt i = 0; i < qq && i < q->ndims_hspace; i++) p *= q->hspace_dims[i];
    return p;
  };
  const gate_type t = g.my_gate_type;
  const PetscInt nq_max = dm ? half : q->ndims_hspace;
  for (PetscInt k = 0; k < g.num_qubits; k++) {
    if (g.qubit_numbers[k] < 0 || g.qubit_numbers[k] >= nq_max) {
      fail(0, "ERROR! qubit %ld out of range for this state\n", (long)g.qubit_numbers[k]);
      return;
    }
  }
  if (g.num_qubits == 2 && g.qubit_numbers[0] == g.qubit_numbers[1]) {
    fail(0, "ERROR! two-qubit gate on a single qubit\n");
    return;
  }
  if (g.num_qubits == 1) {
    cplx U[4], W[4];
    if (t == RZ) {
      U[0] = 1; U[1] = 0; U[2] = 0; U[3] = std::exp(cplx(0, g.theta));
      for (int k = 0; k < 4; k++) W[k] = U[k];  // the column pass is not conjugated
    } else if (t == HADAMARD || t == SIGMAX || t == U1 || t == U2 || t == U3 || t == CUSTOM1QGATE) {
      gate1_matrix(g, U);
      if (has_error()) return;
      for (int k = 0; k < 4; k++) W[k] = std::conj(U[k]);
    } else {
      fail(0, "ERROR! Gate not recognized in get_gate_func_wf!\n");
      return;
    }
    const PetscInt q0 = g.qubit_numbers[0];
    const int64_t sr = nbef(q0);
    const int64_t sc = dm ? nbef(q0 + half) : 0;
    launch_gate1(v->d, n, sr, sc, U, dm ? W : nullptr, s);
    return;
  }
  const PetscInt q0 = g.qubit_numbers[0], q1 = g.qubit_numbers[1];
  cplx U[16], W[16];
  int64_t st[4];
  if (t == CNOT) {
    gate2_matrix(g, U);  // control digit A = q0 (stride from dims), target B = q1
    for (int k = 0; k < 16; k++) W[k] = U[k];
    st[0] = nbef(q0); st[1] = nbef(q1);
    st[2] = dm ? nbef(q0 + half) : 0; st[3] = dm ? nbef(q1 + half) : 0;
  } else if (t == CZ_ARP || t == SQiSWP || t == CUSTOM2QGATE) {
    // basis index d(q0) + 2 d(q1) on bit positions q (quantum_circuits.c:1771-1990)
    cplx M[16];
    if (t == CUSTOM2QGATE) {
      custom_gate_data *d = (custom_gate_data *)g.gate_ctx;
      if (!d) { fail(0, "ERROR! CUSTOM2QGATE needs its gate data\n"); return; }
      for (int k = 0; k < 16; k++) M[k] = cplx(d->gate_data[k / 4][k % 4].real(), d->gate_data[k / 4][k % 4].imag());
    } else {
      gate2_matrix(g, M);
    }
    // kernel basis: 2*d(A) + d(B) with A = q1, B = q0 equals the reference index
    for (int k = 0; k < 16; k++) U[k] = M[k];
    for (int k = 0; k < 16; k++) W[k] = (t == CZ_ARP) ? M[k] : std::conj(M[k]);
    st[0] = (int64_t)1 << q1; st[1] = (int64_t)1 << q0;
    st[2] = dm ? (int64_t)1 << (q1 + half) : 0; st[3] = dm ? (int64_t)1 << (q0 + half) : 0;
  } else {
    fail(0, "ERROR! Gate not recognized in get_gate_func_wf!\n");
    return;
  }
  launch_gate2(v->d, n, st, U, dm ? W : nullptr, s);
}

}  // namespace quac

extern "C" {

void apply_gate2(qvec q, gate_type t, ...) {
  struct quantum_gate_struct g;
  memset(&g, 0, sizeof(g));
  va_list ap;
  va_start(ap, t);
  bool ok = read_gate_args(g, t, ap);
  va_end(ap);
  if (!ok) return;
  vec_sync_to_device(q->data);
  apply_gate_inplace(q, g, g_default_stream());
  QCUDA(cudaStreamSynchronize(g_default_stream()));
  free(g.qubit_numbers);
}

void apply_circuit_to_qvec(qsystem qs, circuit circ, qvec q) {
  vec_sync_to_device(q->data);
  cudaStream_t s = stream_of(qs);
  for (PetscInt i = 0; i < circ.num_gates && !has_error(); i++)
    apply_gate_superop(qs, circ.gate_list[i], q->data, q->my_type == DENSITY_MATRIX, s);
  QCUDA(cudaStreamSynchronize(s));
}

void schedule_circuit_layers(qsystem qs, circuit *circ) {
  std::vector<PetscInt> cur(qs->num_subsystems, 0);
  for (PetscInt i = 0; i < circ->num_gates; i++) {
    circ->layer_list[i].gate_list =
        (struct quantum_gate_struct *)calloc(qs->num_subsystems, sizeof(struct quantum_gate_struct));
    circ->layer_list[i].num_gates = 0;
  }
  for (PetscInt i = 0; i < circ->num_gates; i++) {
    struct quantum_gate_struct &g = circ->gate_list[i];
    PetscInt ml = 0;
    for (PetscInt j = 0; j < g.num_qubits; j++) ml = std::max(ml, cur[g.qubit_numbers[j]]);
    struct gate_layer_struct &L = circ->layer_list[ml];
    L.gate_list[L.num_gates++] = g;
    for (PetscInt j = 0; j < g.num_qubits; j++) cur[g.qubit_numbers[j]] = ml + 1;
  }
  PetscInt ml = 0;
  for (auto c : cur) ml = std::max(ml, c);
  // release the unused layer lists
  for (PetscInt i = ml; i < circ->num_gates; i++) {
    free(circ->layer_list[i].gate_list);
    circ->layer_list[i].gate_list = nullptr;
  }
  circ->num_layers = ml;
  if (ml > 0 && circ->layer_list[0].num_gates > 0 && circ->layer_list[0].gate_list[0].run_time > 0) {
    double t = 1.0;
    for (PetscInt i = 0; i < ml; i++) {
      circ->layer_list[i].time = t;
      double mx = -2;
      for (PetscInt j = 0; j < circ->layer_list[i].num_gates; j++) mx = std::max(mx, circ->layer_list[i].gate_list[j].run_time);
      if (mx < 0) mx = 1.0;
      t += mx;
    }
  } else {
    for (PetscInt i = 0; i < ml; i++) circ->layer_list[i].time = i + 1;
  }
}

void apply_circuit_to_sys(qsystem qs, circuit *circ, PetscReal time) {
  circ->start_time = time;
  if (qs->num_circuits == -1) {
    qs->circuit_list_size = 10;
    qs->circuit_list = (circuit *)malloc(qs->circuit_list_size * sizeof(circuit));
    qs->num_circuits = 0;
    qs->current_circuit = 0;
  }
  if (qs->num_circuits == qs->circuit_list_size) {
    qs->circuit_list_size *= 2;
    qs->circuit_list = (circuit *)realloc(qs->circuit_list, qs->circuit_list_size * sizeof(circuit));
  }
  qs->circuit_list[qs->num_circuits++] = *circ;
}

// ------------------------------------------------ legacy global-state API
static qsystem g_legacy = nullptr;

static qsystem legacy() {
  if (!g_legacy) {
    bool saved = g_initialized;
    g_initialized = true;
    initialize_system(&g_legacy);
    g_initialized = saved;
  }
  return g_legacy;
}

void create_op(int levels, op_handle *op) { create_op_sys(legacy(), levels, op); }
void create_vec(int levels, vec_op *vop) { create_vec_op_sys(legacy(), levels, vop); }
void destroy_op(op_handle *op) { destroy_op_sys(op); }
void destroy_vec(vec_op *vop) { destroy_vec_op_sys(vop); }
void add_to_ham(PetscScalar a, op_handle op) { add_ham_term(legacy(), a, 1, op); }
void add_to_ham_mult2(PetscScalar a, op_handle o1, op_handle o2) { add_ham_term(legacy(), a, 2, o1, o2); }
void add_to_ham_mult3(PetscScalar a, op_handle o1, op_handle o2, op_handle o3) {
  add_ham_term(legacy(), a, 3, o1, o2, o3);
}
void add_lin(PetscScalar a, op_handle op) { add_lin_term(legacy(), a, 1, op); }
void add_lin_mult2(PetscScalar a, op_handle o1, op_handle o2) { add_lin_term(legacy(), a, 2, o1, o2); }

static quac_ts_monitor g_legacy_monitor = nullptr;
static void *g_legacy_ctx = nullptr;
void set_ts_monitor(quac_ts_monitor monitor) {
  g_legacy_monitor = monitor;
  g_legacy_ctx = nullptr;
}
void set_ts_monitor_ctx(quac_ts_monitor monitor, void *ctx) {
  g_legacy_monitor = monitor;
  g_legacy_ctx = ctx;
}

static void legacy_clear() {
  if (g_legacy) destroy_system(&g_legacy);
  g_legacy = nullptr;
  g_legacy_monitor = nullptr;
  g_legacy_ctx = nullptr;
}

// solver.c:236-510: the legacy global system integrated from init_time to
// time_max on the caller's Vec (density matrix or wavefunction, as the
// legacy terms define), with the monitor of set_ts_monitor(_ctx).  The
// reference runs PETSc TS with TSRK3BS here; this runs the same
// integrator as time_step_sys (its controller settings and -ts_* options,
// last step matched to time_max).
void time_step(Vec x, PetscReal init_time, PetscReal time_max, PetscReal dt, PetscInt steps_max) {
  qsystem qs = legacy();
  if (!qs->mat_allocated) construct_matrix(qs);
  if (has_error()) return;
  set_ts_monitor_sys(qs, g_legacy_monitor, g_legacy_ctx);
  qvec tmp = (qvec)calloc(1, sizeof(*tmp));
  tmp->my_type = qs->dm_equations ? DENSITY_MATRIX : WAVEFUNCTION;
  tmp->n = x->n;
  tmp->data = x;
  time_step_sys(qs, tmp, init_time, time_max, dt, steps_max);
  free(tmp);
}

void steady_state(Vec x) {
  qsystem qs = legacy();
  if (!qs->dm_equations) {
    fail(0, "Warning! Steady state not supported for Schrodinger.\n         Defaulting to (less efficient) Lindblad Solver\n");
    return;
  }
  construct_matrix(qs);
  qvec tmp = (qvec)calloc(1, sizeof(*tmp));
  tmp->my_type = DENSITY_MATRIX;
  tmp->n = x->n;
  tmp->data = x;
  PetscInt its = steady_state_sys(qs, tmp);
  free(tmp);
  if (its >= 0) printf("Iterations %ld\n", (long)its);
}

int quac_set_observable_monitor(qsystem qs, PetscInt nobs, const PetscInt *nops, op_handle *ops,
                                quac_observable_monitor cb, void *ctx, PetscInt batch) {
  ObsMonitor &M = qs->impl->obsmon;
  M.release();
  M.obs.clear();
  M.cb = cb;
  M.ctx = ctx;
  if (!cb) return 0;
  if (nobs < 1 || nobs > 64 || batch < 1 || batch > (1 << 20)) {
    fail(0, "ERROR! observable monitor: 1..64 observables and a batch of 1..2^20 steps\n");
    M.cb = nullptr;
    return 1;
  }
  PetscInt k = 0;
  for (PetscInt o = 0; o < nobs; o++) {
    if (nops[o] < 1) { fail(0, "ERROR! observable %ld has no operators\n", (long)o); M.cb = nullptr; return 1; }
    std::vector<op_handle> v(ops + k, ops + k + nops[o]);
    for (op_handle h : v)
      if (!h) { fail(9, "ERROR! NULL operator in an observable\n"); M.cb = nullptr; return 1; }
    M.obs.push_back(v);
    k += nops[o];
  }
  M.batch = batch;
  return 0;
}

}  // extern "C"

namespace quac {
// Device tables of the monitor's observables for dimension D
void observable_monitor_tables(qsystem qs, int64_t D) {
  ObsMonitor &M = qs->impl->obsmon;
  if (M.D == D && M.dmap) return;
  M.release();
  const int nobs = (int)M.obs.size();
  std::vector<int> maps;
  std::vector<double2> vals;
  std::vector<int> map;
  std::vector<cplx> val;
  for (auto &ops : M.obs) {
    op_chain_map(D, ops, map, val);
    for (int64_t r = 0; r < D; r++) {
      maps.push_back(map[r]);
      vals.push_back(make_double2(val[r].real(), val[r].imag()));
    }
  }
  QCUDA(cudaMalloc(&M.dmap, maps.size() * sizeof(int)));
  QCUDA(cudaMalloc(&M.dval, vals.size() * sizeof(double2)));
  QCUDA(cudaMalloc(&M.dvalues, (size_t)M.batch * nobs * sizeof(double2)));
  QCUDA(cudaMemcpy(M.dmap, maps.data(), maps.size() * sizeof(int), cudaMemcpyHostToDevice));
  QCUDA(cudaMemcpy(M.dval, vals.data(), vals.size() * sizeof(double2), cudaMemcpyHostToDevice));
  M.D = D;
}
}  // namespace quac

extern "C" {

// legacy density-matrix helpers (dm_utilities.c): the Vec holds the
// column-stacked density matrix of the legacy system
void create_full_dm(Vec *dm) {
  qsystem qs = legacy();
  const int64_t D = qs->total_levels;
  *dm = vec_new(qs->dm_equations ? D * D : D);
}

void create_dm(Vec *dm, PetscInt size) { *dm = vec_new((int64_t)size * size); }

void destroy_dm(Vec dm) { vec_free(dm); }

static int64_t dm_side(Vec v) { return (int64_t)std::llround(std::sqrt((double)v->n)); }

void add_value_to_dm(Vec dm, PetscInt row, PetscInt col, PetscScalar val) {
  // like the reference on one rank: a location outside the vector is not stored
  const int64_t loc = dm_side(dm) * col + row;
  if (loc < 0 || loc >= dm->n) return;
  if (!dm->host_pending) vec_pull_host(dm);
  dm->host_pending = true;
  dm->h[loc] += cplx(PetscRealPart(val), PetscImaginaryPart(val));
}

void assemble_dm(Vec dm) { vec_sync_to_device(dm); }

void get_dm_element(Vec dm, PetscInt row, PetscInt col, PetscScalar *val) {
  const int64_t loc = dm_side(dm) * col + row;
  if (loc < 0 || loc >= dm->n) { *val = PetscScalar(0.0, 0.0); return; }
  if (dm->host_pending) { *val = PetscScalar(dm->h[loc].real(), dm->h[loc].imag()); return; }
  double2 x;
  QCUDA(cudaMemcpy(&x, dm->d + loc, sizeof(double2), cudaMemcpyDeviceToHost));
  *val = PetscScalar(x.x, x.y);
}

int get_num_populations(void) {
  qsystem qs = legacy();
  int np = 0;
  for (PetscInt i = 0; i < qs->num_subsystems; i++)
    np += qs->subsystem_list[i]->my_op_type == VEC ? (int)qs->subsystem_list[i]->my_levels : 1;
  return np;
}

void get_populations(Vec x, double **populations) {
  qsystem qs = legacy();
  vec_sync_to_device(x);
  const int64_t D = qs->total_levels;
  const bool dm = qs->dm_equations != 0;
  if (x->n != (dm ? D * D : D)) { fail(0, "ERROR! get_populations: the vector does not hold the full legacy system\n"); return; }
  // diagonal of rho (stride D + 1) or the wavefunction, one strided copy
  std::vector<cplx> dg(D);
  QCUDA(cudaMemcpy2D(dg.data(), sizeof(double2), x->d, dm ? (D + 1) * sizeof(double2) : sizeof(double2),
                     sizeof(double2), D, cudaMemcpyDeviceToHost));
  double *pop = *populations;
  int np = 0;
  std::vector<int> first(qs->num_subsystems);
  for (PetscInt j = 0; j < qs->num_subsystems; j++) {
    first[j] = np;
    np += qs->subsystem_list[j]->my_op_type == VEC ? (int)qs->subsystem_list[j]->my_levels : 1;
  }
  for (int k = 0; k < np; k++) pop[k] = 0.0;
  for (int64_t i = 0; i < D; i++) {
    const double w = dm ? dg[i].real() : std::norm(dg[i]);  // Schroedinger form: |psi_i|^2
    for (PetscInt j = 0; j < qs->num_subsystems; j++) {
      op_handle s = qs->subsystem_list[j];
      const int64_t n_after = D / (s->my_levels * s->n_before);
      const int64_t cur = (i / n_after) % s->my_levels;
      if (s->my_op_type == VEC) pop[first[j] + cur] += w;
      else pop[first[j]] += w * (double)cur;
    }
  }
}

}  // extern "C"

// ------------------------------------------- non-variadic gate entry points
extern "C" {

static bool fill_gate(struct quantum_gate_struct &g, int t, int nq, const int *qubits, double th,
                      double ph, double la, void *ctx, void *func) {
  memset(&g, 0, sizeof(g));
  int need = gate_nqubits((gate_type)t);
  if (!need || need != nq) { fail(0, "ERROR! Gate type not recognized\n"); return false; }
  g.my_gate_type = (gate_type)t;
  g.num_qubits = nq;
  g.qubit_numbers = (PetscInt *)malloc(nq * sizeof(PetscInt));
  for (int i = 0; i < nq; i++) g.qubit_numbers[i] = qubits[i];
  g.theta = th;
  g.phi = ph;
  g.lambda = la;
  g.gate_ctx = ctx;
  g.custom_func = (custom_gate_func_type)func;
  g.run_time = -1;
  return true;
}

int quac_add_gate(circuit *circ, double time, int t, int nq, const int *qubits, double th, double ph,
                  double la, void *ctx, void *func) {
  if (circ->num_gates == circ->gate_list_size) { fail(1, "ERROR! Gate list not large enough!\n"); return 1; }
  struct quantum_gate_struct &g = circ->gate_list[circ->num_gates];
  if (!fill_gate(g, t, nq, qubits, th, ph, la, ctx, func)) return 1;
  g.time = time;
  circ->num_gates++;
  return 0;
}

int quac_apply_gate(qvec q, int t, int nq, const int *qubits, double th, double ph, double la,
                    void *ctx) {
  struct quantum_gate_struct g;
  if (!fill_gate(g, t, nq, qubits, th, ph, la, ctx, nullptr)) return 1;
  vec_sync_to_device(q->data);
  apply_gate_inplace(q, g, g_default_stream());
  QCUDA(cudaStreamSynchronize(g_default_stream()));
  free(g.qubit_numbers);
  return has_error() ? 1 : 0;
}

}  // extern "C"

extern "C" void quac_set_stream(qsystem qs, void *stream) {
  qs->impl->user_stream = (cudaStream_t)stream;
}

extern "C" void quac_set_kernel_path(int path) {
  options().kernel_path = path;
}

extern "C" int quac_set_gmres_restart(int m) {
  if (m < 1 || m > 1024) { fail(0, "ERROR! GMRES restart must be in [1, 1024]\n"); return 1; }
  options().gmres_restart = m;
  return 0;
}

extern "C" int quac_set_gmres_precision(int precision) {
  if (precision != 0 && precision != 1) { fail(0, "ERROR! GMRES precision must be 0 (FP64) or 1 (FP32 inner)\n"); return 1; }
  options().gmres_f32 = precision;
  return 0;
}

extern "C" int quac_set_deflation_refresh(int mode) {
  if (mode != 0 && mode != 1) { fail(0, "ERROR! deflation refresh must be 0 (off) or 1 (every restart)\n"); return 1; }
  options().defl_refresh = mode;
  return 0;
}

extern "C" int quac_set_gmres_tolerance(double rtol) {
  if (!(rtol > 0.0 && rtol < 1.0)) { fail(0, "ERROR! GMRES tolerance must lie in (0, 1)\n"); return 1; }
  options().gmres_rtol = rtol;
  return 0;
}

extern "C" int quac_set_gmres_preconditioner(int mode) {
  if (mode < 0 || mode > 2) {
    fail(0, "ERROR! GMRES preconditioner must be 0 (none), 1 (no-jump inverse) or 2 (its Hermitian-part form)\n");
    return 1;
  }
  options().gmres_precond = mode;
  return 0;
}

extern "C" int quac_set_hermitian_mode(int mode) {
  if (mode < 0 || mode > 2) {
    fail(0, "ERROR! Hermitian mode must be 0 (off), 1 (automatic in time_step_sys) or 2 (also single L.x)\n");
    return 1;
  }
  options().herm_mode = mode;
  return 0;
}

extern "C" int quac_set_lrho_precision(int precision) {
  if (precision != 0 && precision != 1) { fail(0, "ERROR! L.rho precision must be 0 (FP64) or 1 (FP32 contraction)\n"); return 1; }
  options().lrho_f32 = precision;
  return 0;
}
