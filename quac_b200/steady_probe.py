"""Steady states of a driven Tavis-Cummings sweep: learned warm start
against cold GMRES on held-out parameter points.

    python -m quac_b200.steady_probe [--ne 3] [--nc 4] [--train 48] [--held 12]
                                     [--sweep2d] [--steps 8000] [--fp32 1] [--kd 8]
                                     [--restart 100] [--refresh 1]

Training states are generated by the solver itself (warmstart.generate),
the network is trained on the GPU, then every held-out point is solved
three ways, each to ||(L + e0 vec(I)^T) x - e0|| <= 1e-11:
  cold     plain complex128 GMRES(100) from e0 (steady_state_sys);
  method   the guided solver with the settings of `learned` (basis precision
           --fp32, restart --restart, deflation refresh --refresh, rank
           --kd) started from e0 with the first kd unit vectors as U: the
           method without the network;
  learned  the same solver started from the network's proposal (initial
           state and deflation space).
Prints one JSON line: solves/s of each, the ratios, iteration counts and
the largest population difference against the cold solve.
"""
import argparse
import json
import time

import numpy as np

from . import warmstart as WS


def defaults(**kw):
    """The command-line defaults as an attribute object, overridden by kw."""
    a = argparse.Namespace(ne=3, nc=4, train=48, held=12, sweep2d=False, steps=8000, lr=2e-3, fp32=1, kd=8,
                           seed=5, restart=100, refresh=1)
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ne", type=int, default=3)
    ap.add_argument("--nc", type=int, default=4)
    ap.add_argument("--train", type=int, default=48)
    ap.add_argument("--held", type=int, default=12)
    ap.add_argument("--sweep2d", action="store_true", help="kappa = 0.1 and gamma = 5e-3 fixed")
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--fp32", type=int, default=1)
    ap.add_argument("--kd", type=int, default=8)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--restart", type=int, default=100)
    ap.add_argument("--refresh", type=int, default=1)
    a = ap.parse_args()
    import quac_b200 as q
    q.QuaC_initialize()
    print(json.dumps(run_sweep(q, a)))


def run_sweep(q, a):
    """The measurement described in the module docstring; `a` carries the
    command-line settings as attributes."""
    D = 2 ** a.ne * a.nc
    fixed = {2: 0.1, 3: 5e-3} if a.sweep2d else None
    thetas = WS.sweep_params(a.train + a.held, seed=a.seed, fixed=fixed)
    train, held = thetas[:a.train], thetas[a.train:]
    net = q.WarmStartNet(D, rank=16, hidden=256, batch=min(128, a.train), max_samples=a.train, seed=2)
    def learned_settings():
        q.set_gmres_precision(a.fp32)
        q.set_gmres_restart(a.restart)
        q.set_deflation_refresh(a.refresh)

    def plain_settings():
        q.set_gmres_precision(0)
        q.set_gmres_restart(100)

    learned_settings()
    t = time.perf_counter()
    gen_its = WS.generate(q, net, train, a.ne, a.nc, kd=a.kd)
    t_gen = time.perf_counter() - t
    t = time.perf_counter()
    loss = net.train(a.steps, lr=a.lr, seed=3)
    t_train = time.perf_counter() - t

    # untimed warm-up of every arm on a training point: the first solve of a
    # solver setting in a process loads its kernels and sizes its buffers
    plain_settings()
    WS.solve_cold(q, train[0], a.ne, a.nc)
    learned_settings()
    e0 = np.zeros(D * D, complex)
    e0[0] = 1.0
    for x0, U in ((e0, np.eye(D, a.kd, dtype=complex)),
                  WS.proposal_from_factors(net.predict(WS.normalize(train[0])[None, :])[0], a.kd)):
        B, v, _, _, _ = WS.solve_guided(q, train[0], a.ne, a.nc, x0, U)
        v.destroy()
        B.qs.destroy()

    rows = []
    for th in held:
        plain_settings()
        xc, its_c, dt_c = WS.solve_cold(q, th, a.ne, a.nc)
        learned_settings()
        B, v, its_m, _, dt_m = WS.solve_guided(q, th, a.ne, a.nc, e0, np.eye(D, a.kd, dtype=complex))
        xm = v.to_numpy()
        v.destroy()
        B.qs.destroy()
        t = time.perf_counter()
        x0, U = WS.proposal_from_factors(net.predict(WS.normalize(th)[None, :])[0], a.kd)
        dt_p = time.perf_counter() - t
        B, v, its_l, res, dt_s = WS.solve_guided(q, th, a.ne, a.nc, x0, U)
        xl = v.to_numpy()
        v.destroy()
        B.qs.destroy()
        dt_l = dt_p + dt_s  # network inference + proposal + solve
        pc = xc.reshape(D, D, order="F").diagonal().real
        perr = max(np.abs(x.reshape(D, D, order="F").diagonal().real - pc).max() for x in (xm, xl))
        rows.append((its_c, dt_c, its_m, dt_m, its_l, dt_l, perr, res))
    plain_settings()
    q.set_deflation_refresh(1)
    r = np.array(rows)
    n = len(held)
    out = {
        "workload": f"tavis_cummings_steady_ne{a.ne}_nc{a.nc}_D{D}",
        "sweep": "2d (omega, delta)" if a.sweep2d else "4d (omega, delta, kappa, gamma)",
        "train_states": a.train, "held_out": n, "kd": a.kd,
        "solver": ("fp32-inner/fp64-refined" if a.fp32 else "fp64") + f" GMRES({a.restart})"
                  + (", deflation refreshed every restart" if a.refresh else ""),
        "generation": {"seconds": t_gen, "mean_iterations": float(np.mean(gen_its))},
        "training": {"steps": a.steps, "seconds": t_train, "loss": loss},
        "cold": {"solves_per_s": n / r[:, 1].sum(), "iterations": r[:, 0].astype(int).tolist()},
        "method": {"solves_per_s": n / r[:, 3].sum(), "iterations": r[:, 2].astype(int).tolist()},
        "learned": {"solves_per_s": n / r[:, 5].sum(), "iterations": r[:, 4].astype(int).tolist()},
        "learned_vs_cold": r[:, 1].sum() / r[:, 5].sum(),
        "learned_vs_method": r[:, 3].sum() / r[:, 5].sum(),
        "method_vs_cold": r[:, 1].sum() / r[:, 3].sum(),
        "pop_err_max": float(r[:, 6].max()),
        "residual_max": float(r[:, 7].max()),
    }
    net.destroy()
    return out


if __name__ == "__main__":
    main()
