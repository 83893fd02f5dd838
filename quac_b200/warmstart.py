"""Learned warm start for steady states of parameter sweeps.

Pipeline (driven Tavis-Cummings sweep: Omega ~ U[0, 0.5], Delta ~ U[-1, 1],
kappa ~ U[0.01, 0.2], gamma ~ U[1e-3, 1e-2], g = 0.1):

1. training states come from the solver itself: points are visited along a
   greedy nearest-neighbour chain; the first is solved cold (GMRES(100)
   from e0), every later one starts from the rank-16 factors of the nearest
   point solved so far and is deflated by their leading directions;
2. the network (quac_wsnet_*) learns parameters -> rank-r factors F with
   F F^H ~ rho_ss;
3. a new point is solved from the proposal: initial state F F^H / tr and
   deflation space { u_i u_j^H } from the kd leading left singular vectors
   of F (quac_steady_state_guided), plain GMRES as the fallback.

The guided solve projects the deflation space out of the Krylov process
(Galerkin projection) and, by default, refreshes it at every restart from
the iterate's leading eigenvectors, so a proposal that is only roughly
right still converges toward the exact subspace; the proposal's value is
in the first restarts.  The guided phase is capped and plain GMRES takes
over from its iterate.  The residual ||(L + e0 vec(I)^T) rho - e0|| <= 1e-11
decides every solve.
"""
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
    B = build_tc(q, theta, ne, nc)
    v = q.create_qvec_sys(B.qs)
    v.from_numpy(x0)
    t = time.perf_counter()
    its, res = q.steady_state_guided(B.qs, v, U, maxit_guided)
    dt = time.perf_counter() - t
    return B, v, its, res, dt


def generate(q, net, thetas, ne, nc, kd=8, rank=16, maxit_guided=3000, log=None):
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
            x0, U = proposal_from_factors(near[1], kd)
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
