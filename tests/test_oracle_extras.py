"""Checks of the oracle pieces that have no reference counterpart.

- `orc_dp5` (Dormand-Prince 5(4)) against the exact solution expm(tL) rho0;
- `oracle/wsnet_oracle.py` (the warm-start network restated in numpy):
  its analytic loss gradient against central finite differences.
"""
import numpy as np
import scipy.linalg as sl

import helpers as H


def test_dp5_oracle_matches_exact_solution(oracle):
    O = oracle.OSys()
    H.driven_jc(O, 6, 0.3, 0.2, 0.1, 0.05)
    A = O.liouvillian()
    D = 12
    x0 = np.zeros(D * D, complex)
    x0[6 * D + 6] = 1.0
    h = O.csr_handle()
    y, nacc, nrej = oracle.dp5(h, x0, 0.0, 3.0, 0.05, atol=1e-11, rtol=1e-11, hmin=1e-4, hmax=1.0)
    oracle.free_csr(h)
    ye = sl.expm(3.0 * A.toarray()) @ x0
    assert np.linalg.norm(y - ye) / np.linalg.norm(ye) < 1e-8
    assert nacc > 10


def test_network_oracle_gradient_matches_finite_differences():
    from oracle import wsnet_oracle as WO
    D, r, Hd, n = 4, 2, 32, 3
    rng = np.random.default_rng(0)
    O = 2 * D * r
    npar = Hd * 32 + Hd + Hd * Hd + Hd + O * Hd + O
    p = rng.normal(scale=0.2, size=npar)
    X = rng.uniform(-1, 1, size=(n, 4))
    rhos = []
    for _ in range(n):
        A = rng.normal(size=(D, 2)) + 1j * rng.normal(size=(D, 2))
        R = A @ A.conj().T
        rhos.append(R / np.trace(R).real)
    rhos = np.array(rhos)
    loss, g = WO.loss_grad(p, X, rhos, D, r, Hd)
    # columns 4..31 of W1 multiply zero-padded inputs: their gradient is zero
    W1g = g[:Hd * 32].reshape(Hd, 32)
    assert np.all(W1g[:, 4:] == 0)
    idx = np.concatenate([np.arange(0, Hd * 32, 32)[:8],                 # W1 (live columns)
                          Hd * 32 + np.arange(4),                         # b1
                          Hd * 32 + Hd + np.arange(0, Hd * Hd, 97)[:8],   # W2
                          npar - O - O * Hd + np.arange(0, O * Hd, 53)[:8],  # W3
                          npar - O + np.arange(4)])                        # b3
    eps = 1e-6
    for k in idx:
        e = np.zeros(npar)
        e[k] = eps
        fd = (WO.loss_grad(p + e, X, rhos, D, r, Hd)[0] - WO.loss_grad(p - e, X, rhos, D, r, Hd)[0]) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), k
