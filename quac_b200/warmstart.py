"""Learned warm start for steady states of parameter sweeps.

Pipeline (driven Tavis-Cummings sweep: Omega ~ U[0, 0.5], Delta ~ U[-1, 1],
kappa ~ U[0.01, 0.2], gamma ~ U[1e-3, 1e-2], g = 0.1):

1. training states come from the solver itself: points are visited along a
   greedy nearest-neighbour chain; the first is solved from e0, every later
   one starts from the rank-16 factors of the nearest point solved so far;
2. the network (quac_wsnet_*) learns parameters -> rank-r factors F with
   F F^H ~ rho_ss;
3. a new point is solved from the proposal F F^H / tr.

With the steady-state preconditioner on (quac_set_gmres_preconditioner:
the inverse of the no-jump Liouvillian, exact or from the Hermitian part of
H_eff) every solve is a preconditioned GMRES(100) started from the better
of the proposal and e0; the eigen-decomposition behind the preconditioner
is a large part of such a solve at D = 512 and the proposal cannot shorten
it.  With the preconditioner off, the proposal also supplies a deflation
space
{ u_i u_j^H } from the kd leading left singular vectors of F
(quac_steady_state_guided: Galerkin projection refreshed at every restart
from the iterate), which is what makes unpreconditioned GMRES converge on
these slow Liouvillians.  The residual ||(L + e0 vec(I)^T) rho - e0|| <=
1e-11 decides every solve.
"""
import argparse
import sys
import time

import numpy as np

from . import systems as Sy

RANGES = np.array([[0.0, 0.5], [-1.0, 1.0], [0.01, 0.2], [1e-3, 1e-2]])


def sweep_params(count, seed=5, fixed=None):
    """(count, 4) array of (omega, delta, kappa, gamma); `fixed` maps a
    column index to a constant value."""
    rng = np.random.default_rng(seed)
    lo, hi = RANGES[:, 0], RANGES[:, 1]
    th = lo + (hi - lo) * rng.uniform(size=(count, 4))
    for k, v in (fixed or {}).items():
        th[:, k] = v
    return th


def normalize(theta):
    lo, hi = RANGES[:, 0], RANGES[:, 1]
    return 2.0 * (np.asarray(theta, dtype=np.float64) - lo) / (hi - lo) - 1.0


def build_tc(q, theta, ne, nc, g=0.1):
    B = Sy.Builder(q)
    om, de, ka, ga = theta
    Sy.tavis_cummings(B, ne=ne, nc=nc, omega=om, delta=de, kappa=ka, gamma=ga, g=g)
    q.construct_matrix(B.qs)
    return B


def factors_from_rho(x, D, r):
    """Leading rank-r factors F (D x r) of the Hermitian part of rho."""
    rho = x.reshape(D, D, order="F")
    w, V = np.linalg.eigh((rho + rho.conj().T) / 2)
    idx = np.argsort(-w)[:r]
    return V[:, idx] * np.sqrt(np.maximum(w[idx], 0.0))


def proposal_from_factors(F, kd):
    """Initial state F F^H / tr and the kd leading left singular vectors of F."""
    rho = F @ F.conj().T
    tr = np.trace(rho).real
    x0 = (rho / tr if tr > 0 else np.eye(F.shape[0]) / F.shape[0]).reshape(-1, order="F")
    U, _, _ = np.linalg.svd(F, full_matrices=False)
    return x0, np.ascontiguousarray(U[:, :kd])


def nn_chain(thetas):
    """Greedy nearest-neighbour visiting order in normalised parameter space."""
    z = normalize(thetas)
    n = len(z)
    order, left = [0], set(range(1, n))
    while left:
        last = z[order[-1]]
        nxt = min(left, key=lambda i: float(np.sum((z[i] - last) ** 2)))
        order.append(nxt)
        left.remove(nxt)
    return order


def solve_cold(q, theta, ne, nc):
    B = build_tc(q, theta, ne, nc)
    v = q.create_qvec_sys(B.qs)
    t = time.perf_counter()
    its = q.steady_state_sys(B.qs, v)
    dt = time.perf_counter() - t
    x = v.to_numpy()
    v.destroy()
    B.qs.destroy()
    return x, its, dt


def solve_guided(q, theta, ne, nc, x0, U, maxit_guided=3000):
    """Steady state of one point from x0 (deflation space U, or none when U
    has no columns)."""
    B = build_tc(q, theta, ne, nc)
    v = q.create_qvec_sys(B.qs)
    v.from_numpy(x0)
    t = time.perf_counter()
    its, res = q.steady_state_guided(B.qs, v, U, maxit_guided)
    dt = time.perf_counter() - t
    return B, v, its, res, dt


def generate(q, net, thetas, ne, nc, kd=8, rank=16, maxit_guided=3000, log=None, precond=False):
    """Solves every point and adds it to the network's samples; returns the
    iteration counts in visiting order."""
    D = 2 ** ne * nc
    z = normalize(thetas)
    solved = []  # (normalised parameters, factors)
    its_all = []
    for k, i in enumerate(nn_chain(thetas)):
        if not solved:
            x, its, dt = solve_cold(q, thetas[i], ne, nc)
            B = build_tc(q, thetas[i], ne, nc)
            v = q.create_qvec_sys(B.qs)
            v.from_numpy(x)
        else:
            near = min(solved, key=lambda s: float(np.sum((s[0] - z[i]) ** 2)))
            x0, U = proposal_from_factors(near[1], 0 if precond else kd)
            B, v, its, res, dt = solve_guided(q, thetas[i], ne, nc, x0, U, maxit_guided)
            x = v.to_numpy()
        net.add_sample(z[i], v)
        solved.append((z[i], factors_from_rho(x, D, rank)))
        its_all.append(its)
        if log:
            log(f"sample {k}: point {i} {its} iterations {dt * 1e3:.0f} ms")
        v.destroy()
        B.qs.destroy()
    return its_all


def solve_learned(q, net, theta, ne, nc, kd=8, maxit_guided=3000):
    F = net.predict(normalize(theta)[None, :])[0]
    x0, U = proposal_from_factors(F, kd)
    B, v, its, res, dt = solve_guided(q, theta, ne, nc, x0, U, maxit_guided)
    x = v.to_numpy()
    v.destroy()
    B.qs.destroy()
    return x, its, res, dt


def sweep_settings(**kw):
    """Settings of measure_sweep: ne emitters, nc cavity levels, train / held
    parameter points, 2-D sweep (kappa and gamma fixed), network training
    steps and learning rate, guided-solver basis precision (fp32), deflation
    rank kd, restart length and refresh, preconditioner, cold sample size
    and GMRES tolerance; kw overrides the defaults."""
    a = argparse.Namespace(ne=3, nc=4, train=48, held=12, sweep2d=False, steps=8000, lr=2e-3, fp32=1, kd=8,
                           seed=5, restart=100, refresh=1, precond=0, cold_sample=None, rtol=1e-11)
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def measure_sweep(q, a):
    """Steady states of a driven Tavis-Cummings sweep, learned warm start
    against cold GMRES on held-out parameter points (`a` from
    sweep_settings).  Training states are generated by the solver itself
    (generate), the network is trained on the GPU, then every held-out point
    is solved by each arm, each to ||(L + e0 vec(I)^T) x - e0|| <= 1e-11:

    cold     unpreconditioned complex128 GMRES(100) from e0 (on the first
             a.cold_sample points when set), the plain path;
    method   the learned run's solver without the network: with a.precond,
             GMRES(100) preconditioned by the point's own decomposition, in
             the a.fp32 basis precision; otherwise the guided solver with the
             first kd unit vectors as deflation space; both from e0;
    learned  the network's proposal as start (the better of it and e0 by
             residual), with a.precond preconditioned GMRES(100) in the
             a.fp32 basis precision, otherwise with the proposal's deflation
             space; its time includes inference and the proposal.

    Every arm builds its own system (and with a.precond its own
    decomposition, inside the timed solve).  Returns solves/s and
    iterations of each arm, the ratios, and the largest population
    difference and residual."""
    WS = sys.modules[__name__]
    D = 2 ** a.ne * a.nc
    kd = 0 if a.precond else a.kd
    fixed = {2: 0.1, 3: 5e-3} if a.sweep2d else None
    thetas = WS.sweep_params(a.train + a.held, seed=a.seed, fixed=fixed)
    train, held = thetas[:a.train], thetas[a.train:]
    ncold = len(held) if a.cold_sample is None else min(len(held), a.cold_sample)
    net = q.WarmStartNet(D, rank=16, hidden=256, batch=min(128, a.train), max_samples=a.train, seed=2)

    def learned_settings():
        q.set_gmres_preconditioner(a.precond)
        q.set_gmres_precision(a.fp32)
        q.set_gmres_restart(100 if a.precond else a.restart)
        q.set_deflation_refresh(a.refresh)

    def method_settings():
        learned_settings()

    def plain_settings():
        q.set_gmres_preconditioner(0)
        q.set_gmres_precision(0)
        q.set_gmres_restart(100)

    builds0 = q.steady_precond_stats()
    q.set_gmres_tolerance(a.rtol)
    learned_settings()
    t = time.perf_counter()
    gen_its = WS.generate(q, net, train, a.ne, a.nc, kd=kd, precond=bool(a.precond))
    t_gen = time.perf_counter() - t
    t = time.perf_counter()
    loss = net.train(a.steps, lr=a.lr, seed=3)
    t_train = time.perf_counter() - t

    e0 = np.zeros(D * D, complex)
    e0[0] = 1.0
    U0 = np.eye(D, kd, dtype=complex)

    def arm_method(th):
        method_settings()
        return WS.solve_guided(q, th, a.ne, a.nc, e0, U0)

    def arm_learned(th):
        learned_settings()
        t0 = time.perf_counter()
        x0, U = WS.proposal_from_factors(net.predict(WS.normalize(th)[None, :])[0], kd)
        dt_p = time.perf_counter() - t0
        B, v, its, res, dt = WS.solve_guided(q, th, a.ne, a.nc, x0, U)
        return B, v, its, res, dt + dt_p  # network inference + proposal + solve

    def finish(r):
        B, v, its, res, dt = r
        x = v.to_numpy()
        v.destroy()
        B.qs.destroy()
        return x, its, res, dt

    # untimed warm-up of every arm on a training point: the first solve of a
    # solver setting in a process loads its kernels and sizes its buffers
    if ncold:
        plain_settings()
        WS.solve_cold(q, train[0], a.ne, a.nc)
    finish(arm_method(train[0]))
    finish(arm_learned(train[0]))

    builds1 = q.steady_precond_stats()
    rows = []
    for k, th in enumerate(held):
        xc, its_c, dt_c = None, -1, float("nan")
        if k < ncold:
            plain_settings()
            xc, its_c, dt_c = WS.solve_cold(q, th, a.ne, a.nc)
        xm, its_m, res_m, dt_m = finish(arm_method(th))
        xl, its_l, res_l, dt_l = finish(arm_learned(th))
        pc = (xc if xc is not None else xm).reshape(D, D, order="F").diagonal().real
        perr = max(np.abs(x.reshape(D, D, order="F").diagonal().real - pc).max() for x in (xm, xl))
        rows.append((its_c, dt_c, its_m, dt_m, its_l, dt_l, perr, max(res_m, res_l)))
    builds2 = q.steady_precond_stats()
    plain_settings()
    q.set_gmres_preconditioner(2)
    q.set_deflation_refresh(1)
    q.set_gmres_tolerance(1e-11)
    r = np.array(rows)
    n = len(held)
    rc = r[:ncold]
    out = {
        "workload": f"tavis_cummings_steady_ne{a.ne}_nc{a.nc}_D{D}",
        "sweep": "2d (omega, delta)" if a.sweep2d else "4d (omega, delta, kappa, gamma)",
        "train_states": a.train, "held_out": n, "kd": kd, "rtol": a.rtol,
        "solver": ("GMRES(100) preconditioned by the "
                   + ("exact inverse" if a.precond == 1 else "Hermitian-part form of the inverse")
                   + " of the no-jump Liouvillian, "
                   + ("fp32-inner/fp64-refined" if a.fp32 else "fp64") + " basis"
                   if a.precond else
                   ("fp32-inner/fp64-refined" if a.fp32 else "fp64") + f" GMRES({a.restart})"
                   + (", deflation refreshed every restart" if a.refresh else "")),
        "generation": {"seconds": t_gen, "mean_iterations": float(np.mean(gen_its))},
        "training": {"steps": a.steps, "seconds": t_train, "loss": loss},
        "method": {"solves_per_s": n / r[:, 3].sum(), "iterations": r[:, 2].astype(int).tolist(),
                   "seconds": [round(float(v), 4) for v in r[:, 3]]},
        "learned": {"solves_per_s": n / r[:, 5].sum(), "iterations": r[:, 4].astype(int).tolist(),
                    "seconds": [round(float(v), 4) for v in r[:, 5]]},
        "learned_vs_method": r[:, 3].sum() / r[:, 5].sum(),
        # per-point time ratios are less sensitive to an occasional slow setup
        "learned_vs_method_median_point": float(np.median(r[:, 3] / r[:, 5])),
        "pop_err_max": float(r[:, 6].max()),
        "residual_max": float(r[:, 7].max()),
    }
    if a.precond:
        nb = builds2[0] - builds0[0]
        out["decompositions"] = {"held_out": builds2[0] - builds1[0], "total": nb,
                                 "mean_seconds": (builds2[1] - builds0[1]) / max(1, nb)}
    if ncold:
        out["cold"] = {"solves_per_s": ncold / rc[:, 1].sum(), "iterations": rc[:, 0].astype(int).tolist(),
                       "points": ncold}
        # per-solve time ratios on the points every arm solved
        out["learned_vs_cold"] = rc[:, 1].sum() / rc[:, 5].sum()
        out["method_vs_cold"] = rc[:, 1].sum() / rc[:, 3].sum()
    net.destroy()
    return out
