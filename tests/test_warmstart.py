"""Tensor-core dense layers and the learned steady-state warm start.

The TF32 GEMM (tcgen05) is checked against numpy on random matrices to
the TF32 input rounding bound (10-bit mantissa per operand).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(q, A, B, bias, act):
    import torch
    assert A.dtype == B.dtype == np.float32 and (bias is None or bias.dtype == np.float32)
    L = q.lib()
    L.quac_gemm_tf32.restype = ctypes.c_int
    L.quac_gemm_tf32.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4
    a = torch.from_numpy(A).cuda()
    b = torch.from_numpy(B).cuda()
    bi = torch.from_numpy(bias).cuda() if bias is not None else None
    c = torch.zeros((A.shape[0], B.shape[0]), dtype=torch.float32, device="cuda")
    rc = L.quac_gemm_tf32(a.data_ptr(), b.data_ptr(), c.data_ptr(), bi.data_ptr() if bi is not None else None,
                          A.shape[0], B.shape[0], A.shape[1], act)
    assert rc == 0, L.quac_last_error()
    return c.cpu().numpy()


@pytest.mark.parametrize("M,N,K,act", [(128, 128, 32, 0), (300, 200, 96, 1), (2000, 16384 // 16, 256, 0),
                                       (77, 513, 64, 1)])
def test_gemm_tf32_matches_numpy(quac, M, N, K, act):
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = (rng.normal(size=(N, K)) / np.sqrt(K)).astype(np.float32)
    bias = rng.normal(size=N).astype(np.float32)
    C = _gemm(quac, A, B, bias, act)
    ref = A.astype(np.float64) @ B.T.astype(np.float64) + bias
    if act == 1:
        ref = np.tanh(ref)
    # TF32 keeps 10 mantissa bits of each operand: |error| <= 3 * 2^-10 * (|A| |B|^T) (tanh is 1-Lipschitz)
    bound = 3 * 2.0 ** -10 * (np.abs(A).astype(np.float64) @ np.abs(B).T.astype(np.float64)) + 1e-6
    assert np.all(np.abs(C - ref) <= bound)
    assert np.abs(C - ref).max() > 0  # really TF32 tensor-core arithmetic, not an FP32 fallback


# ---------------------------------------------------------------- guided solve
from quac_b200 import systems as Sy  # noqa: E402

TC_POINT = dict(omega=0.403, delta=0.616, kappa=0.108, gamma=0.0036)


def _oracle_steady(oracle, ne, nc, p):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    O = oracle.OSys()
    Sy.tavis_cummings(O, ne=ne, nc=nc, g=0.1, **p)
    L = O.liouvillian().tocsr()
    n = L.shape[0]
    D = int(round(np.sqrt(n)))
    row = sp.csr_matrix((np.eye(D).reshape(-1, order="F"), (np.zeros(n, int), np.arange(n))), shape=(n, n))
    b = np.zeros(n, complex)
    b[0] = 1
    return spla.spsolve((L + row).tocsc(), b), D


@pytest.fixture
def no_precond(quac):
    """The unpreconditioned solver (the deflation flow's setting)."""
    quac.set_gmres_preconditioner(0)
    yield
    quac.set_gmres_preconditioner(2)


def _factors(x, D, r):
    rho = x.reshape(D, D, order="F")
    w, V = np.linalg.eigh((rho + rho.conj().T) / 2)
    idx = np.argsort(-w)[:r]
    return V[:, idx], w[idx]


def test_guided_steady_state_with_exact_subspace(quac, oracle, no_precond):
    ne, nc = 3, 4
    xs, D = _oracle_steady(oracle, ne, nc, TC_POINT)
    B = Sy.Builder(quac)
    Sy.tavis_cummings(B, ne=ne, nc=nc, g=0.1, **TC_POINT)
    quac.construct_matrix(B.qs)
    cold = quac.create_qvec_sys(B.qs)
    its_cold = quac.steady_state_sys(B.qs, cold)
    U, w = _factors(xs, D, 16)
    x0 = (U * np.maximum(w, 0)) @ U.conj().T
    x0 = (x0 / np.trace(x0)).reshape(-1, order="F")
    g = quac.create_qvec_sys(B.qs)
    g.from_numpy(x0)
    its, res = quac.steady_state_guided(B.qs, g, U[:, :8])
    y = g.to_numpy()
    print(f"cold {its_cold} iterations, guided {its} iterations, residual {res:.2e}")
    assert res <= 1e-11
    assert 5 * its < its_cold
    assert np.linalg.norm(y - xs) / np.linalg.norm(xs) < 1e-8
    cold.destroy()
    g.destroy()
    B.qs.destroy()


def test_guided_steady_state_falls_back_to_plain_gmres(quac, oracle, no_precond):
    ne, nc = 3, 4
    xs, D = _oracle_steady(oracle, ne, nc, TC_POINT)
    B = Sy.Builder(quac)
    Sy.tavis_cummings(B, ne=ne, nc=nc, g=0.1, **TC_POINT)
    quac.construct_matrix(B.qs)
    rng = np.random.default_rng(1)
    U, _ = np.linalg.qr(rng.normal(size=(D, 4)) + 1j * rng.normal(size=(D, 4)))
    g = quac.create_qvec_sys(B.qs)
    x0 = np.zeros(D * D, complex)
    x0[0] = 1.0
    g.from_numpy(x0)
    its, res = quac.steady_state_guided(B.qs, g, U, maxit_guided=50)
    assert res <= 1e-11 and its > 50
    assert np.linalg.norm(g.to_numpy() - xs) / np.linalg.norm(xs) < 1e-8
    g.destroy()
    B.qs.destroy()


def test_deflation_refresh_finds_the_subspace_itself(quac, oracle, no_precond):
    """Started from e0 with an arbitrary U, the guided solve refreshes U
    from the iterate at every restart (one Rayleigh-Ritz step); it meets
    the residual bar in far fewer iterations than plain GMRES(100), and
    with refresh off the same start gains little or nothing."""
    ne, nc = 3, 4
    xs, D = _oracle_steady(oracle, ne, nc, TC_POINT)
    B = Sy.Builder(quac)
    Sy.tavis_cummings(B, ne=ne, nc=nc, g=0.1, **TC_POINT)
    quac.construct_matrix(B.qs)
    cold = quac.create_qvec_sys(B.qs)
    its_cold = quac.steady_state_sys(B.qs, cold)
    e0 = np.zeros(D * D, complex)
    e0[0] = 1.0
    out = {}
    for mode in (1, 0):
        quac.set_deflation_refresh(mode)
        try:
            g = quac.create_qvec_sys(B.qs)
            g.from_numpy(e0)
            its, res = quac.steady_state_guided(B.qs, g, np.eye(D, 8, dtype=complex))
        finally:
            quac.set_deflation_refresh(1)
        y = g.to_numpy()
        assert res <= 1e-11
        assert np.linalg.norm(y - xs) / np.linalg.norm(xs) < 1e-8
        out[mode] = its
        g.destroy()
    print(f"cold {its_cold}, refresh on {out[1]}, refresh off {out[0]} iterations")
    assert 3 * out[1] < its_cold
    assert out[1] < out[0]
    # kd up to 16 is accepted, 17 is not
    g = quac.create_qvec_sys(B.qs)
    g.from_numpy(e0)
    its16, res16 = quac.steady_state_guided(B.qs, g, np.eye(D, 16, dtype=complex))
    assert res16 <= 1e-11
    with pytest.raises(quac.QuacError):
        quac.steady_state_guided(B.qs, g, np.eye(D, 17, dtype=complex))
    g.destroy()
    cold.destroy()
    B.qs.destroy()


def _residual(oracle, ne, nc, p, x):
    import scipy.sparse as sp
    O = oracle.OSys()
    Sy.tavis_cummings(O, ne=ne, nc=nc, g=0.1, **p)
    L = O.liouvillian().tocsr()
    n = L.shape[0]
    D = int(round(np.sqrt(n)))
    row = sp.csr_matrix((np.eye(D).reshape(-1, order="F"), (np.zeros(n, int), np.arange(n))), shape=(n, n))
    b = np.zeros(n, complex)
    b[0] = 1
    return np.linalg.norm((L + row) @ x - b)


@pytest.mark.parametrize("guided", [False, True], ids=["cold", "guided"])
def test_fp32_inner_gmres_reaches_fp64_tolerance(quac, oracle, guided):
    """complex64 Krylov basis, complex128 residual at every restart: the
    answer meets the same complex128 residual bar as the plain solver."""
    ne, nc = 3, 4
    xs, D = _oracle_steady(oracle, ne, nc, TC_POINT)
    B = Sy.Builder(quac)
    Sy.tavis_cummings(B, ne=ne, nc=nc, g=0.1, **TC_POINT)
    quac.construct_matrix(B.qs)
    g = quac.create_qvec_sys(B.qs)
    quac.set_gmres_precision(1)
    try:
        if guided:
            U, w = _factors(xs, D, 16)
            x0 = (U * np.maximum(w, 0)) @ U.conj().T
            g.from_numpy((x0 / np.trace(x0)).reshape(-1, order="F"))
            its, res = quac.steady_state_guided(B.qs, g, U[:, :8])
            assert res <= 1e-11
        else:
            its = quac.steady_state_sys(B.qs, g)
    finally:
        quac.set_gmres_precision(0)
    y = g.to_numpy()
    r = _residual(oracle, ne, nc, TC_POINT, y)
    print(f"fp32-inner {'guided' if guided else 'cold'}: {its} iterations, residual {r:.2e}")
    assert r <= 2e-11
    assert np.linalg.norm(y - xs) / np.linalg.norm(xs) < 1e-8
    pops = y.reshape(D, D, order="F").diagonal().real
    assert np.abs(pops - xs.reshape(D, D, order="F").diagonal().real).max() < 1e-8
    with pytest.raises(quac.QuacError):
        quac.set_gmres_precision(2)
    g.destroy()
    B.qs.destroy()


# ------------------------------------------------------------ network kernels
def _random_states(rng, n, D):
    out = []
    for _ in range(n):
        A = rng.normal(size=(D, 3)) + 1j * rng.normal(size=(D, 3))
        rho = A @ A.conj().T
        out.append(rho / np.trace(rho).real)
    return np.array(out)


def test_network_gradients_match_cpu_oracle(quac):
    from oracle import wsnet_oracle as WO
    D, r, H, n = 8, 4, 32, 6
    rng = np.random.default_rng(3)
    net = quac.WarmStartNet(D, rank=r, hidden=H, batch=8, max_samples=n, seed=11)
    B = Sy.Builder(quac)
    for _ in range(3):
        B.op(2)
    X = rng.uniform(-1, 1, size=(n, 4))
    rhos = _random_states(rng, n, D)
    for k in range(n):
        v = quac.create_dm_sys(B.qs)
        v.from_numpy(rhos[k].reshape(-1, order="F"))
        net.add_sample(X[k], v)
        v.destroy()
    p = net.get_params()
    # round the targets like the device copy (complex64)
    rhos32 = rhos.astype(np.complex64).astype(np.complex128)
    loss_ref, g_ref = WO.loss_grad(p, X.astype(np.float32).astype(np.float64), rhos32, D, r, H)
    loss, g = net.loss_grad(n)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    W1, b1, W2, b2, W3, b3 = WO.unpack(np.arange(p.size), D, r, H)
    for name, ix in zip(["W1", "b1", "W2", "b2", "W3", "b3"], [W1, b1, W2, b2, W3, b3]):
        ix = np.asarray(ix).ravel().astype(int)
        gr, gg = g_ref[ix], g[ix]
        # TF32 operands (10-bit mantissa) in all six GEMMs of the pass
        assert np.linalg.norm(gg - gr) <= 3e-2 * np.linalg.norm(gr) + 1e-7, name
    # one Adam epoch lowers the loss on this batch
    net.train(30, lr=1e-2, seed=1)
    loss_after, _ = net.loss_grad(n)
    assert loss_after < loss
    net.destroy()
    B.qs.destroy()


def test_trained_network_proposals_and_measured_gain(quac):
    """Sweep of (Omega, Delta) at fixed kappa = 0.1, gamma = 5e-3 for 3
    emitters + 4 cavity levels, 48 solver-generated training states, the
    unpreconditioned deflation flow.  The trained network's proposals are
    much closer to the held-out steady states than an untrained network's;
    the solves started from them meet the residual bar and agree with cold
    solves on populations to 1e-8; and the network saves iterations over
    the method without it (the same guided solver from e0 with the first
    eight unit vectors as its initial deflation space) on at least four of
    the six held-out points, with a median per-point ratio below 1.  (A
    total over six points is decided by single outliers: on a point whose
    steady state is nearly e0 the method needs 8 iterations and a proposed
    deflation space can cost thousands.)"""
    from quac_b200 import warmstart as WS
    ne, nc = 3, 4
    D = 2 ** ne * nc
    thetas = WS.sweep_params(54, seed=5, fixed={2: 0.1, 3: 5e-3})
    train, held = thetas[:48], thetas[48:]
    net = quac.WarmStartNet(D, rank=16, hidden=256, batch=64, max_samples=48, seed=2)
    untrained = quac.WarmStartNet(D, rank=16, hidden=256, batch=64, max_samples=1, seed=2)
    quac.set_gmres_preconditioner(0)  # the deflation flow of unpreconditioned GMRES
    try:
        _run_deflation_flow(quac, WS, net, untrained, train, held, ne, nc, D)
    finally:
        quac.set_gmres_preconditioner(2)
        net.destroy()
        untrained.destroy()


def _run_deflation_flow(quac, WS, net, untrained, train, held, ne, nc, D):
    WS.generate(quac, net, train, ne, nc, kd=8)
    loss = net.train(8000, lr=2e-3, seed=3)
    e0 = np.zeros(D * D, complex)
    e0[0] = 1.0
    cold_its, method_its, learned_its, err_tr, err_un = [], [], [], [], []
    for th in held:
        xc, its_c, _ = WS.solve_cold(quac, th, ne, nc)
        B, v, its_m, res_m, _ = WS.solve_guided(quac, th, ne, nc, e0, np.eye(D, 8, dtype=complex))
        xm = v.to_numpy()
        v.destroy()
        B.qs.destroy()
        xl, its_l, res, _ = WS.solve_learned(quac, net, th, ne, nc, kd=8)
        assert res <= 1e-11 and res_m <= 1e-11
        pc = xc.reshape(D, D, order="F").diagonal().real
        for x in (xl, xm):
            assert np.abs(x.reshape(D, D, order="F").diagonal().real - pc).max() < 1e-8
        for n_, out in ((net, err_tr), (untrained, err_un)):
            x0, _ = WS.proposal_from_factors(n_.predict(WS.normalize(th)[None, :])[0], 8)
            out.append(np.linalg.norm(x0 - xc) / np.linalg.norm(xc))
        cold_its.append(its_c)
        method_its.append(its_m)
        learned_its.append(its_l)
    print(f"train loss {loss:.3e}; proposal error trained {np.round(err_tr, 3)} untrained {np.round(err_un, 3)}; "
          f"iterations cold {cold_its} method {method_its} learned {learned_its}")
    assert loss < 1e-2
    assert 3 * np.mean(err_tr) < np.mean(err_un)
    wins = sum(l < m for l, m in zip(learned_its, method_its))
    assert wins >= 4, (learned_its, method_its)
    assert np.median(np.array(learned_its) / np.array(method_its)) < 1.0


def test_preconditioned_flow(quac):
    """The preconditioned flow (the default): 48 solver-generated training
    states of the (Omega, Delta) sweep train the network; every held-out
    point is then solved to the 1e-11 residual bar cold (no
    preconditioner), by the method (preconditioned, from e0) and learned
    (preconditioned, from the network's proposal, complex64 basis with
    complex128 refinement).  Populations agree to 1e-8; each preconditioned
    solve decomposes its own H_eff once; the preconditioner cuts the
    iterations of the cold solves by more than 5x; the proposal may cost a
    few iterations against e0 (an exact no-jump preconditioner leaves the
    start little to do), at most 2x in total."""
    from quac_b200 import warmstart as WS
    out = WS.measure_sweep(quac, WS.sweep_settings(sweep2d=True, train=48, held=6, precond=1, cold_sample=2))
    print({k: out[k] for k in ("method", "learned", "cold", "decompositions", "learned_vs_method")})
    assert out["residual_max"] <= 1e-11
    assert out["pop_err_max"] < 1e-8
    assert out["decompositions"]["held_out"] == 12
    assert sum(out["learned"]["iterations"]) <= 2 * sum(out["method"]["iterations"])
    assert 5 * max(out["method"]["iterations"][:2]) < min(out["cold"]["iterations"])
