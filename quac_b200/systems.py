"""Synthetic workloads of the benchmarks and parity tests.

Each builder takes an object ``S`` offering ``op(levels)`` (returning an
operator family with a / dag / n / eye / sig_x / sig_y / sig_z), ``ham(a,
*ops)`` and ``lin(a, *ops)`` -- :class:`Builder` below drives this package,
the CPU oracle's ``OSys`` drives the oracle -- so both receive the same
term list.  Parameters are drawn from seeded numpy generators.
"""
import numpy as np


class Builder:
    """Builds a system through this package's QuaC-style API."""

    def __init__(self, q=None):
        if q is None:
            import quac_b200 as q
        self.q = q
        self.qs = q.initialize_system()
        self.levels = []

    def op(self, levels):
        self.levels.append(levels)
        return self.q.create_op_sys(self.qs, levels)

    def vec(self, levels):
        self.levels.append(levels)
        return self.q.create_vec_op_sys(self.qs, levels)

    def ham(self, a, *ops):
        self.q.add_ham_term(self.qs, a, *ops)

    def lin(self, a, *ops):
        self.q.add_lin_term(self.qs, a, *ops)

    @property
    def D(self):
        return int(np.prod(self.levels))


def jc(S, nc=10, g=0.1, kappa=1e-2, gamma=1e-3):
    """Jaynes-Cummings: emitter (2) created first, cavity (nc) second,
    H = g (a^dag sigma + a sigma^dag), L = kappa a, gamma sigma."""
    qb = S.op(2)
    cav = S.op(nc)
    S.ham(g, cav.dag, qb.a)
    S.ham(g, cav.a, qb.dag)
    S.lin(kappa, cav.a)
    S.lin(gamma, qb.a)
    return qb, cav


def driven_jc(S, nc, delta, g, omega, kappa, gamma=1e-3):
    """Driven JC: H = delta a^dag a + g (a^dag sigma + a sigma^dag) + omega (a + a^dag)."""
    qb = S.op(2)
    cav = S.op(nc)
    S.ham(delta, cav.n)
    S.ham(g, cav.dag, qb.a)
    S.ham(g, cav.a, qb.dag)
    S.ham(omega, cav.a)
    S.ham(omega, cav.dag)
    S.lin(kappa, cav.a)
    S.lin(gamma, qb.a)
    return qb, cav


def tfim(S, n, seed=3, g1=1e-3, gphi=5e-4):
    """Open transverse-field Ising chain: sum J_i Z_i Z_{i+1} + sum h_i X_i with
    J ~ U[0.5, 1.5], h ~ N(0, 0.2^2); decay g1 and dephasing gphi per qubit."""
    rng = np.random.default_rng(seed)
    J = rng.uniform(0.5, 1.5, size=n - 1)
    h = rng.normal(0.0, 0.2, size=n)
    qs = [S.op(2) for _ in range(n)]
    for i in range(n - 1):
        S.ham(J[i], qs[i].sig_z, qs[i + 1].sig_z)
    for i in range(n):
        S.ham(h[i], qs[i].sig_x)
    for i in range(n):
        S.lin(g1, qs[i].a)
        S.lin(gphi, qs[i].n)
    return qs


def tavis_cummings(S, ne=6, nc=8, omega=0.3, delta=0.5, kappa=0.1, gamma=5e-3, g=0.1):
    """Driven Tavis-Cummings: ne two-level emitters and a cavity of nc levels."""
    ems = [S.op(2) for _ in range(ne)]
    cav = S.op(nc)
    S.ham(delta, cav.n)
    for e in ems:
        S.ham(g, cav.dag, e.a)
        S.ham(g, cav.a, e.dag)
    S.ham(omega, cav.a)
    S.ham(omega, cav.dag)
    S.lin(kappa, cav.a)
    for e in ems:
        S.lin(gamma, e.a)
    return ems, cav


def driven_jc_ensemble_params(count, seed=11, nc_lo=5, nc_hi=40):
    """Parameter draws of the driven Jaynes-Cummings ensemble: cavity
    truncation nc ~ U{nc_lo..nc_hi}, detuning ~ U[-0.5, 0.5], g ~ U[0.01, 0.2],
    drive omega ~ U[0, 0.3], kappa log-uniform on [1e-3, 1e-1], gamma = 1e-3."""
    rng = np.random.default_rng(seed)
    nc = rng.integers(nc_lo, nc_hi + 1, size=count)
    delta = rng.uniform(-0.5, 0.5, size=count)
    g = rng.uniform(0.01, 0.2, size=count)
    omega = rng.uniform(0.0, 0.3, size=count)
    kappa = 10.0 ** rng.uniform(-3.0, -1.0, size=count)
    return [dict(nc=int(nc[i]), delta=float(delta[i]), g=float(g[i]), omega=float(omega[i]),
                 kappa=float(kappa[i])) for i in range(count)]


def excited_vacuum(nc):
    """rho0 = |e><e| (x) |0><0| of a driven JC system (emitter first), column-stacked."""
    D = 2 * nc
    rho = np.zeros(D * D, dtype=np.complex128)
    rho[nc * D + nc] = 1.0
    return rho


def noisy_circuit_layers(nq=10, layers=40):
    """Gate lists of the noisy random-circuit workload: in layer l each qubit
    q draws, from default_rng(1000 l + q), one of H, X, RZ(theta), U3(theta,
    phi, lambda) with angles ~ U[0, 2 pi); then CNOTs on a random
    nearest-neighbour matching from default_rng(l) (pairs (i, i+1) from a
    random offset, each pair with probability 1/2, random orientation).
    Returns a list of layers, each a list of (gate, qubits, kw)."""
    out = []
    for l in range(layers):
        layer = []
        for q in range(nq):
            rng = np.random.default_rng(1000 * l + q)
            k = int(rng.integers(4))
            if k == 0:
                layer.append(("HADAMARD", (q,), {}))
            elif k == 1:
                layer.append(("SIGMAX", (q,), {}))
            elif k == 2:
                layer.append(("RZ", (q,), dict(theta=float(rng.uniform(0, 2 * np.pi)))))
            else:
                th, ph, la = rng.uniform(0, 2 * np.pi, size=3)
                layer.append(("U3", (q,), dict(theta=float(th), phi=float(ph), lam=float(la))))
        rng = np.random.default_rng(l)
        off = int(rng.integers(2))
        for i in range(off, nq - 1, 2):
            if rng.uniform() < 0.5:
                c, t = (i, i + 1) if rng.uniform() < 0.5 else (i + 1, i)
                layer.append(("CNOT", (c, t), {}))
        out.append(layer)
    return out


def noisy_qubits(S, nq=10):
    """nq qubits with amplitude damping gamma1 ~ U[5e-4, 2e-3] and dephasing
    gamma_phi ~ U[2e-4, 1e-3] per qubit (default_rng(7))."""
    rng = np.random.default_rng(7)
    g1 = rng.uniform(5e-4, 2e-3, size=nq)
    gp = rng.uniform(2e-4, 1e-3, size=nq)
    qs = [S.op(2) for _ in range(nq)]
    for i in range(nq):
        S.lin(g1[i], qs[i].a)
        S.lin(gp[i], qs[i].n)
    return qs
