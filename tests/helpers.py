"""Shared system builders for the parity tests.

Each builder takes an object S with op(levels) / vec(levels) / ham(a, *ops)
/ lin(a, *ops) -- the oracle's OSys or ProductSystem below -- so that the
oracle and the CUDA product receive the same term list.
"""
import numpy as np


class ProductSystem:
    """Builds a system through the product's Python API (quac_b200)."""

    def __init__(self, q):
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
    """Jaynes-Cummings: emitter (2) created first, cavity (nc) second."""
    qb = S.op(2)
    cav = S.op(nc)
    S.ham(g, cav.dag, qb.a)
    S.ham(g, cav.a, qb.dag)
    S.lin(kappa, cav.a)
    S.lin(gamma, qb.a)
    return qb, cav


def driven_jc(S, nc, delta, g, omega, kappa, gamma=1e-3):
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
    """Open transverse-field Ising chain: sum J ZZ + sum h X, T1/T2 per qubit."""
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


def mixed(S):
    """Mixed radix with every basic operator kind and products."""
    a = S.op(3)
    b = S.op(2)
    c = S.op(5)
    S.ham(0.3, a.dag, c.a)
    S.ham(0.3, a.a, c.dag)
    S.ham(0.25j, b.sig_y)
    S.ham(-0.4, c.n, a.n)
    S.ham(0.1 + 0.05j, b.sig_x, c.dag)
    S.lin(0.2, c.a)
    S.lin(0.05, a.a, b.sig_z)
    S.lin(0.07, b.n)
    S.lin(0.03 + 0.01j, a.dag)
    return a, b, c


def random_state(D, seed=0, hermitian=False):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    if hermitian:
        X = X @ X.conj().T
        X /= np.trace(X)
    return X.reshape(-1, order="F")
