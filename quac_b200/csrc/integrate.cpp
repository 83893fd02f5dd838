// time_step_sys: explicit Runge-Kutta integration of d(rho)/dt = L rho with
// every stage fused into one matrix-free L.x launch (lrho.cu).
//
// Replaces the PETSc TS set-up of qsystem.c:895-1098: TS_LINEAR with the
// assembled Liouvillian as constant Jacobian, TSRK3BS by default,
// atol = rtol = 5e-7, step limits [0.01, 1], final step matched to tmax,
// the user monitor after every step, and circuit gates applied at their
// event times (quantum_circuits.c:17-120).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "runtime.h"

namespace quac {

const double kDP_C[7] = {0.0, 0.2, 0.3, 0.8, 8.0 / 9.0, 1.0, 1.0};
const double kDP_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {0.2, 0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
    {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
const double kDP_E[7] = {35.0 / 384.0 - 5179.0 / 57600.0, 0.0, 500.0 / 1113.0 - 7571.0 / 16695.0,
                         125.0 / 192.0 - 393.0 / 640.0, -2187.0 / 6784.0 + 92097.0 / 339200.0,
                         11.0 / 84.0 - 187.0 / 2100.0, -1.0 / 40.0};

void apply_gate_superop(qsystem qs, const struct quantum_gate_struct &g, Vec v, bool is_dm,
                        cudaStream_t s);
void apply_gate_inplace(qvec q, const struct quantum_gate_struct &g, cudaStream_t s);

cplx TdTerm::scale(double t) const {
  cplx v;
  if (f) {
    const PetscScalar r = f(t, ctx);
    v = cplx(PetscRealPart(r), PetscImaginaryPart(r));
  } else {
    double re = 0.0, im = 0.0;
    g(t, ctx, &re, &im);
    v = cplx(re, im);
  }
  return term.a * v;
}

void release_td_programs(qsystem qs) {
  for (TdTerm &td : qs->impl->td) {
    if (td.prog) {
      td.prog->release();
      delete td.prog;
      td.prog = nullptr;
    }
    td.prog_mode = -1;
  }
  if (qs->impl->td_acc) cudaFree(qs->impl->td_acc);
  qs->impl->td_acc = nullptr;
  qs->impl->td_acc_n = 0;
}

namespace {

// Each time-dependent term compiled on its own with coefficient 1
// (construct_matrix, qsystem.c:642-651), in the system's current mode
void ensure_td_programs(qsystem qs) {
  const int mode = qs->dm_equations ? 0 : 1;
  for (TdTerm &td : qs->impl->td) {
    if (td.prog && td.prog_mode == mode) continue;
    if (td.prog) {
      td.prog->release();
      delete td.prog;
      td.prog = nullptr;
    }
    std::vector<Term> saved;
    saved.swap(qs->impl->terms);
    Term one = td.term;
    one.a = cplx(1.0, 0.0);
    qs->impl->terms.push_back(one);
    td.prog = compile_terms(qs, mode);
    qs->impl->terms.swap(saved);
    td.prog_mode = mode;
    if (!td.prog) return;
  }
}

}  // namespace

void apply_L(qsystem qs, double t, const double2 *x, const Epi &e, cudaStream_t s) {
  qsystem_impl &I = *qs->impl;
  if (I.td.empty()) {
    launch_lrho_any(*I.prog, x, e, s);
    return;
  }
  // Y = A X + sum_k a_k f_k(t) A_k X (qsystem.c:1300-1330), then the
  // stage epilogue on Y
  ensure_td_programs(qs);
  if (has_error()) return;
  const DeviceProgram &P = *I.prog;
  const int64_t n = (int64_t)P.dev.D * P.dev.ncols;
  if (I.td_acc_n != n) {
    if (I.td_acc) QCUDA(cudaFree(I.td_acc));
    I.td_acc = nullptr;
    QCUDA(cudaMalloc(&I.td_acc, 2 * (size_t)n * sizeof(double2)));
    I.td_acc_n = n;
  }
  double2 *K = I.td_acc, *T = I.td_acc + n;
  Epi e0;
  zero_epi(e0);
  e0.kout = K;
  launch_lrho_any(P, x, e0, s);
  for (const TdTerm &td : I.td) {
    const cplx sc = td.scale(t);
    if (std::abs(sc) <= 1e-10) continue;  // min_time_dep, qsystem.c:34, 1320
    Epi ek;
    zero_epi(ek);
    ek.kout = T;
    launch_lrho_any(*td.prog, x, ek, s);
    launch_caxpy(K, T, sc, n, s);
  }
  launch_epilogue(K, e, n, s);
}

namespace {

struct Event {
  double t;
  int circ;
  int idx;   // layer (scheduled) or gate (unscheduled) index
  bool layer;
};

std::vector<Event> collect_events(qsystem qs, double t0, double tmax) {
  std::vector<Event> ev;
  for (PetscInt c = 0; c < qs->num_circuits; c++) {
    circuit &C = qs->circuit_list[c];
    if (C.num_layers > 0) {
      for (PetscInt l = 0; l < C.num_layers; l++)
        ev.push_back({C.layer_list[l].time + C.start_time, (int)c, (int)l, true});
    } else {
      for (PetscInt g = 0; g < C.num_gates; g++)
        ev.push_back({C.gate_list[g].time + C.start_time, (int)c, (int)g, false});
    }
  }
  std::stable_sort(ev.begin(), ev.end(), [](const Event &a, const Event &b) { return a.t < b.t; });
  std::vector<Event> out;
  for (auto &e : ev)
    if (e.t > t0 && e.t <= tmax * (1 + 1e-14) + 1e-14) out.push_back(e);
  return out;
}

// Stage helpers -------------------------------------------------------
struct Stepper {
  qsystem qs;
  const DeviceProgram *P;
  cudaStream_t s;
  int64_t n;
  double atol, rtol;
  int herm;  // Hermitian mode of the multi-pass kernel (see Epi::herm)

  void stage(double ts, const double2 *X,
             std::initializer_list<std::tuple<double2 *, const double2 *, double>> upd,
             double *nsum = nullptr, int err_upd = 0, const double2 *ny = nullptr,
             const double2 *nyn = nullptr) {
    Epi e;
    zero_epi(e);
    int u = 0;
    for (auto &t : upd) {
      e.out[u] = std::get<0>(t);
      e.base[u] = std::get<1>(t);
      e.coef[u] = std::get<2>(t);
      u++;
    }
    e.nupd = u;
    e.nsum = nsum;
    e.err_upd = err_upd;
    e.ny = ny;
    e.nyn = nyn;
    e.atol = atol;
    e.rtol = rtol;
    e.herm = herm;
    apply_L(qs, ts, X, e, s);
  }
};

}  // namespace

// Runs the integration on vector v (device-resident, length qs->dim).  The
// qvec (if any) receives circuit gates and is handed to the monitor.
int integrate(qsystem qs, qvec x, Vec v, double t0, double tmax, double dt, int64_t steps_max) {
  if (qs->mcwf_solver) return mcwf_integrate(qs, x, t0, tmax, dt, steps_max);
  ensure_program(qs);
  if (has_error() || !qs->impl->prog) return 1;
  const DeviceProgram &PP = *qs->impl->prog;
  const DevProg &P = PP.dev;
  const int64_t n = v->n;
  if (n != (int64_t)P.D * P.ncols) {
    fail(0, "ERROR! qvec size %ld does not match the system dimension %ld\n", (long)n,
         (long)((int64_t)P.D * P.ncols));
    return 1;
  }
  Options &o = options();
  if (o.max_steps > 0) steps_max = o.max_steps;
  const bool fixed = (o.rk_type == "4") || (o.adapt_type == "none");
  const bool rk4 = (o.rk_type == "4");
  const bool dp5 = (o.rk_type == "5dp");
  cudaStream_t s = stream_of(qs);
  Workspace &W = qs->impl->ws;
  W.ensure(n, dp5 ? 8 : 4);
  vec_sync_to_device(v);  // blocking copy of pending host values; everything else is ordered on s

  std::vector<Event> events = x ? collect_events(qs, t0, tmax) : std::vector<Event>();
  // Hermitian mode: L preserves Hermiticity (checked on the compiled
  // tables), the multi-pass kernel runs, no gate lands inside this run, and
  // the initial state is Hermitian to rounding; every stage then keeps the
  // state exactly Hermitian (conjugate-transposed blocks are written, not
  // computed)
  const bool td = !qs->impl->td.empty();
  int herm = 0;
  if (o.herm_mode && !td && PP.herm_ok && PP.has_qubit && !PP.passes.empty() && P.ncols == P.D && events.empty())
    herm = hermitian_asymmetry(v->d, P.D, s) <= 1e-13 ? 1 : 0;
  Stepper st{qs, &PP, s, n, o.atol, o.rtol, herm};
  ObsMonitor &OM = qs->impl->obsmon;
  const int nobs = OM.cb ? (int)OM.obs.size() : 0;
  if (nobs) observable_monitor_tables(qs, P.D);
  if (has_error()) return 1;
  // monitored small system, fixed RK4, nothing else per step: many steps
  // per launch with the state in shared memory (small_run.cu)
  if (nobs && !qs->ts_monitor && fixed && rk4 && !o.rk4_classic && !td && events.empty() && P.ncols == P.D &&
      small_rk4_eligible(PP)) {
    const double tol = 1e-12 * std::max(1.0, std::fabs(tmax));
    std::vector<double> hs, ts;
    double tt = t0;
    while ((int64_t)hs.size() < steps_max && tt < tmax - tol) {
      double h_try = dt;
      bool last = false;
      if (tt + h_try >= tmax - tol) { h_try = tmax - tt; last = true; }
      hs.push_back(h_try);
      tt = last ? tmax : tt + h_try;
      ts.push_back(tt);
    }
    std::vector<PetscScalar> vals;
    std::vector<PetscInt> stepno;
    for (size_t i = 0; i < hs.size() && !has_error();) {
      size_t j = i;
      while (j < hs.size() && (int64_t)(j - i) < OM.batch && hs[j] == hs[i]) j++;
      const int cnt = (int)(j - i);
      launch_small_rk4(PP, v->d, cnt, hs[i], nobs, OM.dmap, OM.dval, OM.dvalues, s);
      vals.resize((size_t)cnt * nobs);
      QCUDA(cudaMemcpyAsync(vals.data(), OM.dvalues, vals.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
      QCUDA(cudaStreamSynchronize(s));
      stepno.resize(cnt);
      for (int k = 0; k < cnt; k++) stepno[k] = (PetscInt)(i + k + 1);
      OM.cb(cnt, stepno.data(), ts.data() + i, vals.data(), OM.ctx);
      i = j;
    }
    qs->current_time = hs.empty() ? t0 : ts.back();
    return has_error() ? 1 : 0;
  }
  std::vector<PetscInt> ob_steps;
  std::vector<PetscReal> ob_times;
  std::vector<PetscScalar> ob_vals;
  auto flush_obs = [&]() {
    if (!ob_steps.empty()) OM.cb((PetscInt)ob_steps.size(), ob_steps.data(), ob_times.data(), ob_vals.data(), OM.ctx);
    ob_steps.clear();
    ob_times.clear();
    ob_vals.clear();
  };
  size_t next_ev = 0;
  _p_TS ts;
  ts.t = t0;
  ts.dt = dt;
  ts.step = 0;
  if (qs->ts_monitor) qs->ts_monitor(&ts, 0, t0, v, qs->ts_ctx);

  double t = t0, h = dt;
  const double hmin = 0.01, hmax = 1.0;
  int64_t steps = 0;
  const double tend_tol = 1e-12 * std::max(1.0, std::fabs(tmax));
  while (steps < steps_max && t < tmax - tend_tol && !has_error()) {
    double h_try = h;
    bool last = false;
    if (t + h_try >= tmax - tend_tol) { h_try = tmax - t; last = true; }
    bool at_event = false;
    if (next_ev < events.size() && t + h_try >= events[next_ev].t - tend_tol) {
      h_try = events[next_ev].t - t;
      at_event = true;
      last = false;
      if (std::fabs(events[next_ev].t - tmax) <= tend_tol) last = true;
    }
    double2 *y = v->d;
    bool accepted = true;
    double h_next = h;
    if (dp5) {
      // Dormand-Prince 5(4): K_s = L x_s (one launch each), stage inputs and
      // the error norm by fused linear combinations of the stored K's
      double2 *K[7] = {W.bufs[0], W.bufs[1], W.bufs[2], W.bufs[3], W.bufs[4], W.bufs[5], W.bufs[6]};
      double2 *xs = W.bufs[7];
      for (int st_i = 0; st_i < 7; st_i++) {
        const double2 *X = y;
        if (st_i > 0) {
          double c[6];
          for (int j = 0; j < st_i; j++) c[j] = h_try * kDP_A[st_i][j];
          launch_lincomb(xs, y, st_i, (const double2 *const *)K, c, n, s);
          X = xs;
        }
        Epi e;
        zero_epi(e);
        e.kout = K[st_i];
        e.herm = herm;
        apply_L(qs, t + kDP_C[st_i] * h_try, X, e, s);
      }
      // xs now holds the fifth-order solution (input of stage 7)
      double c[7];
      for (int j = 0; j < 7; j++) c[j] = h_try * kDP_E[j];
      if (fixed) {
        std::swap(v->d, W.bufs[7]);
      } else {
        QCUDA(cudaMemsetAsync(W.dsum, 0, sizeof(double), s));
        launch_lincomb_norm(y, xs, 7, (const double2 *const *)K, c, n, o.atol, o.rtol, W.dsum, s);
        QCUDA(cudaMemcpyAsync(W.hsum, W.dsum, sizeof(double), cudaMemcpyDeviceToHost, s));
        QCUDA(cudaStreamSynchronize(s));
        const double err = std::sqrt(W.hsum[0] / (double)n);
        double fac = err > 0 ? 0.9 * std::pow(err, -0.2) : 10.0;
        fac = std::min(10.0, std::max(0.1, fac));
        h_next = std::min(hmax, std::max(hmin, h_try * fac));
        accepted = (err <= 1.0) || (h_try <= hmin * (1 + 1e-12));
        if (accepted) std::swap(v->d, W.bufs[7]);
        if (!accepted) { h = h_next; continue; }
      }
    } else if (fixed && rk4 && !o.rk4_classic && !td) {
      // For a time-independent linear right-hand side the classical RK4 step
      // equals the degree-4 Taylor polynomial of exp(hL); evaluated by
      // Horner's rule each stage reads one vector besides its input:
      //   v <- y + (h/4) L y;  v <- y + (h/3) L v;  v <- y + (h/2) L v;  y <- y + h L v
      double2 *va = W.bufs[0], *vb = W.bufs[1];
      st.stage(t, y, {{va, y, h_try / 4.0}});
      st.stage(t, va, {{vb, y, h_try / 3.0}});
      st.stage(t, vb, {{va, y, h_try / 2.0}});
      st.stage(t, va, {{y, y, h_try}});
    } else if (fixed && rk4) {
      double2 *acc = W.bufs[0], *xa = W.bufs[1], *xb = W.bufs[2];
      st.stage(t, y, {{acc, y, h_try / 6.0}, {xa, y, h_try / 2.0}});
      st.stage(t + 0.5 * h_try, xa, {{acc, acc, h_try / 3.0}, {xb, y, h_try / 2.0}});
      st.stage(t + 0.5 * h_try, xb, {{acc, acc, h_try / 3.0}, {xa, y, h_try}});
      st.stage(t + h_try, xa, {{y, acc, h_try / 6.0}});
    } else {
      // Bogacki-Shampine 3(2): c = (0, 1/2, 3/4, 1), b = (2/9, 1/3, 4/9, 0),
      // bhat = (7/24, 1/4, 1/3, 1/8); error = h * sum (b - bhat)_i k_i.
      double2 *x1 = W.bufs[0], *x2 = W.bufs[1], *yn = W.bufs[2], *er = W.bufs[3];
      st.stage(t, y, {{x1, y, 0.5 * h_try}, {yn, y, 2.0 / 9.0 * h_try}, {er, nullptr, (2.0 / 9.0 - 7.0 / 24.0) * h_try}});
      st.stage(t + 0.5 * h_try, x1, {{x2, y, 0.75 * h_try}, {yn, yn, h_try / 3.0}, {er, er, (1.0 / 3.0 - 0.25) * h_try}});
      st.stage(t + 0.75 * h_try, x2, {{yn, yn, 4.0 / 9.0 * h_try}, {er, er, (4.0 / 9.0 - 1.0 / 3.0) * h_try}});
      if (fixed) {
        std::swap(v->d, W.bufs[2]);
      } else {
        QCUDA(cudaMemsetAsync(W.dsum, 0, sizeof(double), s));
        st.stage(t + h_try, yn, {{er, er, -0.125 * h_try}}, W.dsum, 0, y, yn);
        QCUDA(cudaMemcpyAsync(W.hsum, W.dsum, sizeof(double), cudaMemcpyDeviceToHost, s));
        QCUDA(cudaStreamSynchronize(s));
        const double err = std::sqrt(W.hsum[0] / (double)n);
        double fac = err > 0 ? 0.9 * std::pow(err, -1.0 / 3.0) : 10.0;
        fac = std::min(10.0, std::max(0.1, fac));
        h_next = std::min(hmax, std::max(hmin, h_try * fac));
        accepted = (err <= 1.0) || (h_try <= hmin * (1 + 1e-12));
        if (accepted) std::swap(v->d, W.bufs[2]);
        if (!accepted) { h = h_next; continue; }
      }
    }
    steps++;
    t = last ? tmax : t + h_try;
    if (!fixed) h = h_next;
    if (at_event && x) {
      const double te = events[next_ev].t;
      while (next_ev < events.size() && std::fabs(events[next_ev].t - te) <= tend_tol) {
        const Event &e = events[next_ev];
        circuit &C = qs->circuit_list[e.circ];
        if (e.layer) {
          gate_layer_struct &L = C.layer_list[e.idx];
          for (PetscInt g = 0; g < L.num_gates; g++)
            apply_gate_superop(qs, L.gate_list[g], v, x->my_type == DENSITY_MATRIX, s);
          C.current_layer = e.idx + 1;
        } else {
          apply_gate_inplace(x, C.gate_list[e.idx], s);
          C.current_gate = e.idx + 1;
        }
        next_ev++;
      }
    }
    if (qs->ts_monitor) {
      QCUDA(cudaStreamSynchronize(s));
      ts.t = t;
      ts.dt = h_try;
      ts.step = steps;
      qs->ts_monitor(&ts, steps, t, v, qs->ts_ctx);
    }
    if (nobs) {
      for (int ob = 0; ob < nobs; ob++) {
        const int *m = OM.dmap + (size_t)ob * P.D;
        const double2 *w = OM.dval + (size_t)ob * P.D;
        const cplx e = P.ncols == P.D ? dm_expectation(v->d, P.D, m, w, s) : wf_expectation(v->d, P.D, m, w, s);
        ob_vals.push_back(PetscScalar(e.real(), e.imag()));
      }
      ob_steps.push_back(steps);
      ob_times.push_back(t);
      if ((int64_t)ob_steps.size() >= OM.batch) flush_obs();
    }
  }
  if (nobs) flush_obs();
  // one wait at the end: the error-flag read-back is queued behind the last
  // stage (check_program_error synchronises), or a plain stream sync
  if (qs->impl->prog->errflag) check_program_error(*qs->impl->prog, s);
  else QCUDA(cudaStreamSynchronize(s));
  qs->current_time = t;
  if (std::fabs(t - tmax) > 1e-8 && !has_error()) printf("ERROR! Did not reach final time! Reason: %d\n", -1);
  return has_error() ? 1 : 0;
}

// Hermitian mode 2 for a single L.x: the program supports it and x is
// Hermitian to 1e-13 (relative Frobenius asymmetry)
int apply_herm(qsystem qs, const double2 *x, cudaStream_t s) {
  const DeviceProgram &PP = *qs->impl->prog;
  if (options().herm_mode != 2 || !qs->impl->td.empty() || !PP.herm_ok || !PP.has_qubit || PP.passes.empty() || PP.dev.ncols != PP.dev.D)
    return 0;
  return hermitian_asymmetry(x, PP.dev.D, s) <= 1e-13 ? 1 : 0;
}

}  // namespace quac

using namespace quac;

extern "C" {

void set_ts_monitor_sys(qsystem qs, quac_ts_monitor monitor, void *ctx) {
  qs->ts_monitor = monitor;
  qs->ts_ctx = ctx;
}

void time_step_sys(qsystem qs, qvec x, PetscReal t0, PetscReal tmax, PetscReal dt,
                   PetscInt steps_max) {
  qs->time_step_called = PETSC_TRUE;
  qs->solution_qvec = x;
  if (qs->mat_allocated != 1) {
    fail(0, "ERROR! Matrix does not seem to be constructed! You need to\n       call construct_matrix!\n");
    return;
  }
  integrate(qs, x, x->data, t0, tmax, dt, steps_max);
}

int quac_lrho_apply_device(qsystem qs, const void *x_dev, void *y_dev) {
  if (qs->mat_allocated != 1) { fail(0, "ERROR! call construct_matrix first\n"); return 1; }
  ensure_program(qs);
  if (has_error()) return 1;
  Epi e;
  zero_epi(e);
  e.kout = (double2 *)y_dev;
  cudaStream_t s = stream_of(qs);
  e.herm = apply_herm(qs, (const double2 *)x_dev, s);
  apply_L(qs, qs->current_time, (const double2 *)x_dev, e, s);
  QCUDA(cudaStreamSynchronize(s));
  check_program_error(*qs->impl->prog, s);
  return has_error() ? 1 : 0;
}

int quac_lrho_apply_host(qsystem qs, const PetscScalar *x_host, PetscScalar *y_host) {
  if (qs->mat_allocated != 1) { fail(0, "ERROR! call construct_matrix first\n"); return 1; }
  Workspace &W = qs->impl->ws;
  const int64_t n = qs->dim;
  W.ensure(n, 4);
  cudaStream_t s = stream_of(qs);
  QCUDA(cudaMemcpyAsync(W.bufs[0], x_host, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  ensure_program(qs);
  if (has_error()) return 1;
  Epi e;
  zero_epi(e);
  e.kout = W.bufs[1];
  e.herm = apply_herm(qs, W.bufs[0], s);
  apply_L(qs, qs->current_time, W.bufs[0], e, s);
  QCUDA(cudaMemcpyAsync(y_host, W.bufs[1], n * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  check_program_error(*qs->impl->prog, s);
  return has_error() ? 1 : 0;
}

int quac_time_step_host(qsystem qs, PetscScalar *x_host, PetscReal t0, PetscReal tmax,
                        PetscReal dt, PetscInt steps_max) {
  if (qs->mat_allocated != 1) { fail(0, "ERROR! call construct_matrix first\n"); return 1; }
  const int64_t n = qs->dim;
  Vec &v = qs->impl->host_vec;  // device copy kept for the next call
  if (v && vec_len(v) != n) {
    vec_free(v);
    v = nullptr;
  }
  if (!v) v = vec_new(n);
  if (has_error()) return 1;
  cudaStream_t s = stream_of(qs);
  QCUDA(cudaMemcpyAsync(v->d, x_host, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  QCUDA(cudaStreamSynchronize(s));
  int rc = integrate(qs, nullptr, v, t0, tmax, dt, steps_max);
  QCUDA(cudaMemcpyAsync(x_host, v->d, n * sizeof(double2), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  return rc;
}

}  // extern "C"
