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


from quac_b200.systems import driven_jc, jc, tavis_cummings, tfim  # noqa: F401,E402


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
