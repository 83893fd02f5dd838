// Host-side runtime objects behind the opaque handles of quac_b200.h.
#pragma once
#include <map>
#include <string>
#include <vector>

#include "common.h"

// Vec: one complex128 vector in device memory with an on-demand host copy
// (the VecGetArray stand-in maps it to host memory).
struct _p_Vec {
  int64_t n = 0;
  double2 *d = nullptr;               // device data
  std::vector<quac::cplx> h;          // host staging copy
  bool host_pending = false;          // h holds additions not yet on the device
  bool host_mapped = false;           // VecGetArray outstanding
};

struct _p_TS {
  double t = 0, dt = 0;
  int64_t step = 0;
};

namespace quac {

struct Term {
  int kind;  // 1 = Hamiltonian, 2 = Lindblad
  cplx a;
  std::vector<op_handle> ops;
};

struct DeviceProgram;
// Observables recorded on the device every step (quac_set_observable_monitor)
struct ObsMonitor {
  std::vector<std::vector<op_handle>> obs;
  quac_observable_monitor cb = nullptr;
  void *ctx = nullptr;
  int64_t batch = 1000;
  int *dmap = nullptr;        // nobs x D observable row maps (device)
  double2 *dval = nullptr;    // nobs x D values
  double2 *dvalues = nullptr; // batch x nobs recorded values
  int64_t D = 0;
  void release();
};
// A time-dependent term: its superoperator with coefficient 1, scaled by
// a f(t) at every stage (qsystem.c:1300-1330)
struct TdTerm {
  Term term;                                // term.a = the caller's coefficient
  quac_time_dep_func f = nullptr;           // one of the two callback forms
  quac_time_dep_func_parts g = nullptr;
  void *ctx = nullptr;
  DeviceProgram *prog = nullptr;
  int prog_mode = -1;
  cplx scale(double t) const;
};

struct Options {
  std::string rk_type = "3bs";
  std::string adapt_type = "basic";
  double rtol = 5e-7, atol = 5e-7;  // qsystem.c:902
  int64_t max_steps = -1;           // -1: use the caller's steps_max
  bool rtol_set = false, atol_set = false;
  int kernel_path = 0;              // see quac_set_kernel_path
  int lrho_f32 = 0;                 // see quac_set_lrho_precision
  int herm_mode = 1;                // see quac_set_hermitian_mode
  int gmres_f32 = 0;                // see quac_set_gmres_precision
  int defl_refresh = 1;             // see quac_set_deflation_refresh
  double gmres_rtol = 1e-11;        // -ksp_rtol (solver.c:14, 179: 1e-11 on ||b|| = 1)
  int gmres_restart = 100;          // -ksp_gmres_restart (solver.c uses PETSc's default 100 via KSPGMRESSetRestart)
  int gmres_precond = 2;            // see quac_set_gmres_preconditioner
  bool rk4_classic = false;         // rk_type "4classic": four-stage form instead of Horner
};
Options &options();

// Workspace of one integrator (device buffers of dim complex128 each).
struct Workspace {
  int64_t dim = 0;
  std::vector<double2 *> bufs;
  double *dsum = nullptr;   // device scalars
  double *hsum = nullptr;   // pinned host mirror
  void ensure(int64_t dim, int nbufs);
  void release();
};

}  // namespace quac

struct qsystem_impl {
  std::vector<quac::Term> terms;
  quac::DeviceProgram *prog = nullptr;
  int prog_mode = -1;
  cudaStream_t stream = nullptr;       // owned
  cudaStream_t user_stream = nullptr;  // set by quac_set_stream (not owned)
  quac::Workspace ws;
  std::vector<op_handle> owned_ops;  // every operator struct created for this system
  Vec host_vec = nullptr;            // device state of quac_time_step_host, kept between calls
  std::vector<quac::TdTerm> td;      // time-dependent terms
  quac::ObsMonitor obsmon;           // quac_set_observable_monitor
  uint64_t mcwf_seed = 0;            // use_mcwf_solver
  int64_t mcwf_ntraj = 0;
  double2 *td_acc = nullptr;         // L(t) x and one term's contribution (2 x dim, lazily allocated)
  int64_t td_acc_n = 0;
};

namespace quac {
cudaStream_t stream_of(qsystem qs);
void ensure_program(qsystem qs);
// y-side of one RK stage at time t: the fused L.x launch for a
// time-independent system; with time-dependent terms, L(t) x is summed
// term group by term group and the epilogue runs as its own pass
void apply_L(qsystem qs, double t, const double2 *x, const Epi &e, cudaStream_t s);
void release_td_programs(qsystem qs);
// MCWF trajectories (mcwf.cu)
int mcwf_integrate(qsystem qs, qvec x, double t0, double tmax, double dt, int64_t steps_max);
bool mcwf_spawned(qvec q);
void mcwf_release(qvec q);
void mcwf_release_system(qsystem qs);
cplx mcwf_expectation(qvec q, const int *map, const double2 *val);
// steady-state preconditioner cache (precond.cu)
void precond_release_system(qsystem qs);
// device tables of the observable monitor's observables (capi.cpp)
void observable_monitor_tables(qsystem qs, int64_t D);
// small_run.cu
bool small_rk4_eligible(const DeviceProgram &P);
void launch_small_rk4(const DeviceProgram &P, double2 *state, int nsteps, double h, int nobs, const int *omap,
                      const double2 *oval, double2 *values, cudaStream_t s);
int64_t vec_len(Vec v);
void vec_sync_to_device(Vec v);       // flush pending host additions
Vec vec_new(int64_t n);
void vec_free(Vec v);
// Observable kernels (observe.cu)
cplx dm_expectation(const double2 *rho, int64_t D, const int *colmap, const double2 *colval,
                    cudaStream_t s);
cplx wf_expectation(const double2 *psi, int64_t D, const int *map, const double2 *val,
                    cudaStream_t s);
cplx dm_trace(const double2 *rho, int64_t D, cudaStream_t s);
double dm_wf_fidelity(const double2 *rho, const double2 *psi, int64_t D, cudaStream_t s);
cplx vdot(const double2 *a, const double2 *b, int64_t n, cudaStream_t s);
// Operator-product row map on the Hilbert space (terms.cpp)
void op_chain_map(int64_t D, const std::vector<op_handle> &ops, std::vector<int> &map,
                  std::vector<cplx> &val);
}  // namespace quac
