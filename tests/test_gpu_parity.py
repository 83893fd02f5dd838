"""CUDA path against the oracle (run on a B200: pytest -m gpu).

Tolerances: complex128 arithmetic throughout; the matrix-free kernel sums
the same products as the assembled CSR in a different order, so results
agree to ~1e-14 relative.  The bar in these tests is 1e-12 relative for one
L.x, 1e-10 relative for integrated states, 1e-12 for
gates and observables.
"""
import numpy as np
import pytest

import fixture_systems as F
import helpers as H
from conftest import golden_csr

pytestmark = pytest.mark.gpu


def _lrho(q, S, x):
    q.construct_matrix(S.qs)
    return q.lrho_apply_host(S.qs, x)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("case", F.CASES, ids=lambda c: f"{c[0]}-{c[1]}op-{c[2]}-{'c' if c[3] else 'r'}")
def test_lrho_matches_golden_fixture(quac, golden, case):
    fam, nop, kind, cplx = case
    S = H.ProductSystem(quac)
    stems = F.build(S, fam, nop, kind, cplx)
    ref = sum(golden_csr(golden, s) for s in stems)
    x = np.random.default_rng(7).normal(size=ref.shape[0]) + 1j * np.random.default_rng(8).normal(size=ref.shape[0])
    y = _lrho(quac, S, x)
    assert _rel(y, ref @ x) < 1e-12
    S.qs.destroy()


@pytest.mark.parametrize("build", [
    lambda S: H.jc(S),
    lambda S: H.driven_jc(S, 13, 0.2, 0.1, 0.3, 0.05),
    lambda S: H.tfim(S, 6),
    lambda S: H.tfim(S, 8),
    lambda S: H.tavis_cummings(S, ne=3, nc=5),
    lambda S: H.mixed(S),
], ids=["jc", "driven_jc13", "tfim6", "tfim8", "tc3x5", "mixed3x2x5"])
def test_lrho_matches_oracle(quac, oracle, build):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    build(S)
    build(O)
    A = O.liouvillian()
    for seed in range(2):
        x = H.random_state(S.D, seed=seed)
        y = _lrho(quac, S, x)
        assert _rel(y, A @ x) < 1e-12
    S.qs.destroy()


def test_lrho_device_entry_point(quac, oracle):
    import torch
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, 7)
    H.tfim(O, 7)
    quac.construct_matrix(S.qs)
    x = H.random_state(S.D, seed=3)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    quac.lrho_apply_device(S.qs, xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    assert _rel(yd.cpu().numpy(), O.liouvillian() @ x) < 1e-12
    S.qs.destroy()


def test_rk4_fixed_step_matches_oracle(quac, oracle):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    qb, cav = H.jc(S)
    H.jc(O)
    quac.construct_matrix(S.qs)
    rho = quac.create_qvec_sys(S.qs)
    quac.add_to_qvec(rho, 1.0, 10, 10)
    quac.assemble_qvec(rho)
    quac.set_ts_options(rk_type="4", adapt_type="none")
    try:
        quac.time_step_sys(S.qs, rho, 0.0, 2.0, 0.01, 100000)
    finally:
        quac.set_ts_options(rk_type="3bs", adapt_type="basic")
    y = rho.to_numpy()
    h = O.csr_handle()
    x0 = np.zeros(400, dtype=complex)
    x0[10 * 20 + 10] = 1.0
    yo = oracle.rk4(h, x0, 0.01, 200)
    oracle.free_csr(h)
    assert _rel(y, yo) < 1e-10
    n_q = quac.get_expectation_value_qvec(rho, qb.n)
    assert abs(n_q - oracle.expect_dm([2, 10], yo, (0, 0, -1))) < 1e-12
    rho.destroy()
    S.qs.destroy()


def test_bs3_adaptive_matches_oracle(quac, oracle):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.driven_jc(S, 8, 0.3, 0.2, 0.1, 0.05)
    H.driven_jc(O, 8, 0.3, 0.2, 0.1, 0.05)
    quac.construct_matrix(S.qs)
    rho = quac.create_qvec_sys(S.qs)
    D = S.D
    quac.add_to_qvec(rho, 1.0, 8, 8)
    quac.assemble_qvec(rho)
    quac.time_step_sys(S.qs, rho, 0.0, 3.0, 0.05, 100000)
    y = rho.to_numpy()
    h = O.csr_handle()
    x0 = np.zeros(D * D, dtype=complex)
    x0[8 * D + 8] = 1.0
    yo, nacc, nrej = oracle.bs3(h, x0, 0.0, 3.0, 0.05)
    oracle.free_csr(h)
    assert _rel(y, yo) < 1e-10
    rho.destroy()
    S.qs.destroy()


@pytest.mark.parametrize("adapt", ["basic", "none"])
def test_dp5_matches_oracle(quac, oracle, adapt):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.driven_jc(S, 8, 0.3, 0.2, 0.1, 0.05)
    H.driven_jc(O, 8, 0.3, 0.2, 0.1, 0.05)
    quac.construct_matrix(S.qs)
    rho = quac.create_qvec_sys(S.qs)
    D = S.D
    quac.add_to_qvec(rho, 1.0, 8, 8)
    quac.assemble_qvec(rho)
    quac.set_ts_options(rk_type="5dp", adapt_type=adapt)
    try:
        quac.time_step_sys(S.qs, rho, 0.0, 3.0, 0.05, 100000)
    finally:
        quac.set_ts_options(rk_type="3bs", adapt_type="basic")
    y = rho.to_numpy()
    h = O.csr_handle()
    x0 = np.zeros(D * D, dtype=complex)
    x0[8 * D + 8] = 1.0
    if adapt == "basic":
        yo, nacc, nrej = oracle.dp5(h, x0, 0.0, 3.0, 0.05)
    else:
        # fixed step: the controller accepts everything (hmin = hmax = dt)
        yo, nacc, nrej = oracle.dp5(h, x0, 0.0, 3.0, 0.05, atol=1e300, hmin=0.05, hmax=0.05)
        assert nacc == 60 and nrej == 0
    oracle.free_csr(h)
    assert _rel(y, yo) < 1e-10
    rho.destroy()
    S.qs.destroy()


def test_t1_decay_known_answer_gpu(quac):
    q = quac
    qs = q.initialize_system()
    vop = q.create_vec_op_sys(qs, 2)
    q.add_lin_term(qs, 1.0, vop[0], vop[1])
    dm = q.create_qvec_sys(qs)
    q.add_to_qvec(dm, 1.0, 1, 1)
    q.assemble_qvec(dm)
    q.construct_matrix(qs)
    q.time_step_sys(qs, dm, 0.0, 1.0, 0.05, 200)
    v = q.get_expectation_value_qvec(dm, vop[1], vop[1])
    assert abs(v.real - np.exp(-1)) < 1e-4
    dm.destroy()
    qs.destroy()


def test_circuit_events_during_time_step(quac):
    """time_step_tests.c:337-396: unscheduled circuit gates use in-place
    qubit numbering (qubit 0 = last subsystem)."""
    q = quac
    qs = q.initialize_system()
    op2 = q.create_op_sys(qs, 2)
    op3 = q.create_op_sys(qs, 2)
    q.add_ham_term(qs, 1.0, op2.n)
    q.add_lin_term(qs, 1.0, op2)
    q.add_lin_term(qs, 1.0, op3)
    dm = q.create_qvec_sys(qs)
    q.add_to_qvec(dm, 1.0, 0, 0)
    q.assemble_qvec(dm)
    q.construct_matrix(qs)
    circ = q.create_circuit(5)
    q.add_gate_to_circuit_sys(circ, 0.0, "SIGMAX", 0)
    q.add_gate_to_circuit_sys(circ, 0.1, "SIGMAX", 1)
    q.apply_circuit_to_sys(qs, circ, 0.1)
    q.time_step_sys(qs, dm, 0.0, 1.1, 0.05, 200)
    assert abs(q.get_expectation_value_qvec(dm, op2.n).real - np.exp(-0.9)) < 5e-4
    assert abs(q.get_expectation_value_qvec(dm, op3.n).real - np.exp(-1.0)) < 5e-4
    dm.destroy()
    qs.destroy()


GATE_CASES = [("HADAMARD", [1], {}), ("SIGMAX", [2], {}), ("SIGMAY", [0], {}), ("SIGMAZ", [1], {}),
              ("EYE", [0], {}), ("RX", [2], dict(theta=0.37)), ("RY", [1], dict(theta=-1.2)),
              ("RZ", [0], dict(theta=2.1)), ("U3", [1], dict(theta=0.4, phi=1.3, lam=-0.8)),
              ("U2", [2], dict(theta=np.pi / 2, phi=0.2, lam=0.9)),
              ("U1", [0], dict(theta=0.0, phi=0.0, lam=0.6)),
              ("CNOT", [0, 2], {}), ("CNOT", [2, 0], {}), ("CXZ", [1, 0], {}), ("CZX", [0, 1], {}),
              ("CZ", [2, 1], {}), ("CmZ", [1, 2], {}), ("CZ_ARP", [0, 2], {})]


@pytest.mark.parametrize("gate,qubits,kw", GATE_CASES, ids=lambda v: str(v))
def test_superop_gate_matches_oracle(quac, oracle, gate, qubits, kw):
    q = quac
    qs = q.initialize_system()
    for _ in range(3):
        q.create_op_sys(qs, 2)
    dm = q.create_dm_sys(qs)
    x = H.random_state(8, seed=11)
    dm.from_numpy(x)
    c = q.create_circuit(1)
    c.add_gate(0.0, gate, *qubits, theta=kw.get("theta", 0.0), phi=kw.get("phi", 0.0),
               lam=kw.get("lam", 0.0))
    q.apply_circuit_to_qvec(qs, c, dm)
    ref = oracle.gate_superop([2, 2, 2], x, gate, qubits, **kw)
    assert _rel(dm.to_numpy(), ref) < 1e-12
    dm.destroy()
    qs.destroy()


INPLACE_CASES = [("HADAMARD", [1], {}), ("SIGMAX", [2], {}), ("RZ", [0], dict(theta=0.8)),
                 ("U3", [2], dict(theta=0.4, phi=1.3, lam=-0.8)), ("CNOT", [0, 2], {}),
                 ("CNOT", [2, 1], {}), ("CZ_ARP", [1, 2], {}), ("SQiSWP", [0, 1], {})]


@pytest.mark.parametrize("gate,qubits,kw", INPLACE_CASES, ids=lambda v: str(v))
def test_inplace_gate_matches_oracle(quac, oracle, gate, qubits, kw):
    q = quac
    qs = q.initialize_system()
    for _ in range(3):
        q.create_op_sys(qs, 2)
    dm = q.create_dm_sys(qs)
    x = H.random_state(8, seed=12)
    dm.from_numpy(x)
    args = list(qubits)
    if gate == "RZ":
        args.append(kw["theta"])
    if gate == "U3":
        args += [kw["theta"], kw["phi"], kw["lam"]]
    q.apply_gate2(dm, gate, *args)
    ref = oracle.gate_inplace([2] * 6, x, gate, qubits, **kw)
    assert _rel(dm.to_numpy(), ref) < 1e-12
    dm.destroy()
    qs.destroy()


def test_observables_match_numpy(quac, oracle):
    q = quac
    S = H.ProductSystem(q)
    a, b, c = H.mixed(S)
    dm = q.create_dm_sys(S.qs)
    D = S.D
    x = H.random_state(D, seed=5, hermitian=True)
    dm.from_numpy(x)
    for ops, trip in [((c.n,), [(0, 2, -1)]), ((a.dag, c.a), [(-1, 0, -1), (1, 2, -1)]),
                      ((b.sig_x,), [(3, 1, -1)])]:
        got = q.get_expectation_value_qvec(dm, *ops)
        ref = oracle.expect_dm(S.levels, x, *trip)
        assert abs(got - ref) < 1e-12
    assert abs(q.get_trace_qvec(dm) - np.trace(x.reshape(D, D, order="F"))) < 1e-12
    wf = q.create_arb_qvec(D, q.WAVEFUNCTION)
    psi = np.random.default_rng(3).normal(size=D) + 1j * np.random.default_rng(4).normal(size=D)
    psi /= np.linalg.norm(psi)
    wf.from_numpy(psi)
    f, _ = q.get_fidelity_qvec(dm, wf)
    R = x.reshape(D, D, order="F")
    assert abs(f - (psi.conj() @ R @ psi).real) < 1e-12
    dm.destroy()
    wf.destroy()
    S.qs.destroy()


def test_steady_state_matches_direct_solve(quac, oracle):
    import scipy.sparse.linalg as sla
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tavis_cummings(S, ne=2, nc=4)
    H.tavis_cummings(O, ne=2, nc=4)
    quac.construct_matrix(S.qs)
    x = quac.create_qvec_sys(S.qs)
    its = quac.steady_state_sys(S.qs, x)
    assert its > 0
    D = S.D
    A = O.liouvillian().tolil()
    for i in range(D):
        A[0, i * (D + 1)] += 1.0
    b = np.zeros(D * D, dtype=complex)
    b[0] = 1
    xd = sla.spsolve(A.tocsr(), b)
    xg = x.to_numpy()
    # GMRES stops on the residual (rtol 1e-11 as solver.c:176); the error
    # against the direct solve is bounded by the conditioning, so the bar is
    # the residual plus population agreement at 1e-8
    assert np.linalg.norm(A.tocsr() @ xg - b) < 1e-10
    pops = lambda v: np.real(np.diag(v.reshape(D, D, order="F")))
    assert np.max(np.abs(pops(xg) - pops(xd))) < 1e-8
    x.destroy()
    S.qs.destroy()


@pytest.mark.parametrize("ne,nc,params", [
    (3, 4, dict(omega=0.3, delta=0.2, kappa=0.1, gamma=5e-3)),
    (3, 4, dict(omega=0.45, delta=-0.7, kappa=0.02, gamma=1e-3)),
    (4, 6, dict(omega=0.2, delta=0.5, kappa=0.15, gamma=2e-3))], ids=["tc32", "tc32-slow", "tc96"])
def test_steady_state_preconditioned_vs_plain(quac, oracle, ne, nc, params):
    """The no-jump-inverse preconditioner, exact (1) and from the Hermitian
    part of H_eff (2): the same residual and populations against a direct
    solve, in at least ten times fewer iterations than the unpreconditioned
    GMRES(100)."""
    import scipy.sparse.linalg as sla
    its, xs = {}, {}
    for pre in (0, 1, 2):
        S = H.ProductSystem(quac)
        H.tavis_cummings(S, ne=ne, nc=nc, **params)
        quac.construct_matrix(S.qs)
        x = quac.create_qvec_sys(S.qs)
        quac.set_gmres_preconditioner(pre)
        try:
            its[pre] = quac.steady_state_sys(S.qs, x)
        finally:
            quac.set_gmres_preconditioner(2)
        xs[pre] = x.to_numpy()
        x.destroy()
        S.qs.destroy()
    O = oracle.OSys()
    H.tavis_cummings(O, ne=ne, nc=nc, **params)
    D = O.D
    A = O.liouvillian().tolil()
    for i in range(D):
        A[0, i * (D + 1)] += 1.0
    A = A.tocsr()
    b = np.zeros(D * D, dtype=complex)
    b[0] = 1
    xd = sla.spsolve(A.tocsc(), b)
    pops = lambda v: np.real(np.diag(v.reshape(D, D, order="F")))
    for pre in (0, 1, 2):
        assert its[pre] > 0
        assert np.linalg.norm(A @ xs[pre] - b) < 1e-10
        assert np.max(np.abs(pops(xs[pre]) - pops(xd))) < 1e-8
    assert 10 * its[1] <= its[0], its
    assert 10 * its[2] <= its[0], its


def test_legacy_steady_state_uses_preconditioner(quac):
    """steady_state(Vec) and steady_state_sys share the solver; the option is
    process-wide and defaults to on (the Hermitian-part form)."""
    assert quac.lib().quac_set_gmres_preconditioner(2) == 0


def test_monitor_called_every_step(quac):
    q = quac
    S = H.ProductSystem(q)
    qb, cav = H.jc(S, nc=4)
    q.construct_matrix(S.qs)
    rho = q.create_qvec_sys(S.qs)
    q.add_to_qvec(rho, 1.0, 4, 4)
    q.assemble_qvec(rho)
    seen = []
    q.set_ts_monitor_sys(S.qs, lambda step, t, vec: seen.append((step, t)))
    q.set_ts_options(rk_type="4", adapt_type="none")
    try:
        q.time_step_sys(S.qs, rho, 0.0, 0.1, 0.01, 1000)
    finally:
        q.set_ts_options(rk_type="3bs", adapt_type="basic")
        q.set_ts_monitor_sys(S.qs, None)
    assert [s for s, _ in seen] == list(range(11))
    assert abs(seen[-1][1] - 0.1) < 1e-12
    rho.destroy()
    S.qs.destroy()


def qubit_zoo(S, n=7):
    """All-qubit system exercising the bit-mask kernel: complex coefficients,
    sigma_y, products over several qubits, conditions (ladder operators),
    multi-qubit diagonal jumps, |i><j| pairs and high-bit partners."""
    qs = [S.op(2) for _ in range(n)]
    S.ham(0.7, qs[0].sig_x)
    S.ham(0.3j, qs[1].sig_y, qs[n - 1].sig_z)
    S.ham(0.2 - 0.1j, qs[2].dag, qs[n - 2].a)
    S.ham(0.4, qs[n - 1].sig_x, qs[3].sig_x)
    S.ham(-0.25, qs[0].sig_z, qs[n - 1].sig_z)
    S.ham(0.15, qs[4].n, qs[1].sig_x)
    S.lin(0.05, qs[0].a)
    S.lin(0.02, qs[n - 1].a, qs[2].sig_z)
    S.lin(0.03, qs[3].n)
    S.lin(0.04, qs[1].n, qs[5].n)
    S.lin(0.01 + 0.002j, qs[n - 3].dag)
    S.lin(0.06, qs[2].sig_x)
    S.ham(0.12, qs[0].sig_x, qs[n - 1].sig_x)   # flips in two bit groups
    S.lin(0.015, qs[n - 1].a, qs[0].dag)
    return qs


def tfim_real(S, n):
    return H.tfim(S, n)


def tfim_pump(S, n):
    """Real-coefficient system that exercises every canonical single-bit
    slot (X fields, decay, pumping) plus general and cross-group terms."""
    qs = H.tfim(S, n)
    for q in qs[::3]:
        S.lin(2e-3, q.dag)
    S.ham(0.11, qs[0].sig_x, qs[n - 1].sig_x)
    S.ham(0.07, qs[1].sig_x, qs[2].sig_x)
    S.lin(0.01, qs[n - 2].a, qs[0].a)
    return qs


@pytest.mark.parametrize("n,build", [(6, qubit_zoo), (7, qubit_zoo), (9, qubit_zoo),
                                     (6, tfim_real), (10, tfim_real), (7, tfim_pump),
                                     (11, tfim_pump)],
                         ids=["zoo6", "zoo7", "zoo9", "tfim6", "tfim10", "pump7", "pump11"])
def test_qubit_kernel_matches_oracle(quac, oracle, n, build):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    build(S, n)
    build(O, n)
    quac.construct_matrix(S.qs)
    A = O.liouvillian()
    for seed in range(2):
        x = H.random_state(S.D, seed=seed)
        assert _rel(quac.lrho_apply_host(S.qs, x), A @ x) < 1e-12
    S.qs.destroy()


@pytest.mark.parametrize("n", [8, 11])
def test_qubit_and_generic_kernels_agree(quac, n):
    ys = []
    for path in (0, 1, 2):
        quac.set_kernel_path(path)
        S = H.ProductSystem(quac)
        qubit_zoo(S, n)
        quac.construct_matrix(S.qs)
        x = H.random_state(S.D, seed=9)
        ys.append(quac.lrho_apply_host(S.qs, x))
        S.qs.destroy()
    quac.set_kernel_path(0)
    assert _rel(ys[0], ys[1]) < 1e-13
    assert _rel(ys[2], ys[1]) < 1e-13


def test_full_size_tfim12_properties(quac, oracle):
    """D = 4096 (the benchmarked system): the oracle cannot hold the whole
    superoperator quickly, so check (a) a row block against the oracle's
    assembled rows, (b) trace preservation Tr(L x) = 0, (c) Hermiticity
    preservation L(x^dag) = (L x)^dag, (d) linearity."""
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, 12)
    H.tfim(O, 12)
    quac.construct_matrix(S.qs)
    D = S.D
    rng = np.random.default_rng(21)
    X = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    x = X.reshape(-1, order="F")
    y = quac.lrho_apply_host(S.qs, x)
    r0, r1 = 37 * D, 41 * D + 17
    Ablk = O.liouvillian(rows=(r0, r1))
    assert _rel(y[r0:r1], Ablk @ x) < 1e-12
    Y = y.reshape(D, D, order="F")
    assert abs(np.trace(Y)) < 1e-9 * np.abs(Y).max() * D
    yh = quac.lrho_apply_host(S.qs, X.conj().T.reshape(-1, order="F"))
    assert _rel(yh.reshape(D, D, order="F"), Y.conj().T) < 1e-13
    x2 = rng.normal(size=D * D) + 0j
    y2 = quac.lrho_apply_host(S.qs, x2)
    y12 = quac.lrho_apply_host(S.qs, 0.3 * x + 2.0 * x2)
    assert _rel(y12, 0.3 * y + 2.0 * y2) < 1e-13
    S.qs.destroy()


def test_rk4_horner_equals_classical(quac):
    outs = []
    for form in ("4", "4classic"):
        S = H.ProductSystem(quac)
        H.tfim(S, 8)
        quac.construct_matrix(S.qs)
        rho = quac.create_dm_sys(S.qs)
        rho.from_numpy(H.random_state(S.D, seed=4, hermitian=True))
        quac.set_ts_options(rk_type=form, adapt_type="none")
        quac.time_step_sys(S.qs, rho, 0.0, 1.0, 0.01, 10 ** 6)
        outs.append(rho.to_numpy())
        rho.destroy()
        S.qs.destroy()
    quac.set_ts_options(rk_type="3bs", adapt_type="basic")
    assert _rel(outs[0], outs[1]) < 1e-13


def test_multipass_rk4_tfim9_matches_oracle(quac, oracle):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, 9)
    H.tfim(O, 9)
    quac.construct_matrix(S.qs)
    D = S.D
    x0 = H.random_state(D, seed=6, hermitian=True)
    rho = quac.create_dm_sys(S.qs)
    rho.from_numpy(x0)
    quac.set_ts_options(rk_type="4", adapt_type="none")
    quac.time_step_sys(S.qs, rho, 0.0, 0.2, 0.01, 10 ** 6)
    quac.set_ts_options(rk_type="3bs", adapt_type="basic")
    h = O.csr_handle()
    yo = oracle.rk4(h, x0, 0.01, 20)
    oracle.free_csr(h)
    assert _rel(rho.to_numpy(), yo) < 1e-12
    rho.destroy()
    S.qs.destroy()


# complex64 contraction (multi-pass kernel): one L.x is held to 2e-6
# relative (float rounding of tiles, coefficients and ~40 accumulated terms);
# an integration keeps its FP64 state, so trace and populations stay within
# 1e-6 of the complex128 run over a short horizon.
def test_fp32_contraction_lx_matches_oracle(quac, oracle):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, 9)
    H.tfim(O, 9)
    quac.construct_matrix(S.qs)
    x = H.random_state(S.D, seed=4, hermitian=True)
    quac.set_lrho_precision(1)
    try:
        y32 = quac.lrho_apply_host(S.qs, x)
    finally:
        quac.set_lrho_precision(0)
    y64 = quac.lrho_apply_host(S.qs, x)
    ref = O.liouvillian() @ x
    assert _rel(y64, ref) < 1e-12
    e = _rel(y32, ref)
    assert 1e-10 < e < 2e-6
    S.qs.destroy()


def test_fp32_contraction_integration_error(quac):
    outs = []
    for prec in (0, 1):
        S = H.ProductSystem(quac)
        H.tfim(S, 9)
        quac.construct_matrix(S.qs)
        D = S.D
        rho = quac.create_dm_sys(S.qs)
        quac.add_to_qvec(rho, 1.0, 0, 0)
        quac.assemble_qvec(rho)
        quac.set_lrho_precision(prec)
        quac.set_ts_options(rk_type="5dp", adapt_type="basic", rtol=1e-8, atol=1e-8)
        try:
            quac.time_step_sys(S.qs, rho, 0.0, 2.0, 0.01, 10 ** 6)
        finally:
            quac.set_lrho_precision(0)
            quac.set_ts_options(rk_type="3bs", adapt_type="basic", rtol=5e-7, atol=5e-7)
        outs.append(rho.to_numpy().reshape(D, D, order="F"))
        rho.destroy()
        S.qs.destroy()
    a, b = outs
    assert abs(np.trace(b) - 1.0) < 1e-6
    assert np.abs(a.diagonal().real - b.diagonal().real).max() < 1e-6


# Hermitian mode (12-qubit TFIM, Hermitian start): the blocks below the block
# diagonal are written as conjugate transposes instead of being computed; the
# result must agree with the full computation to rounding for every scheme.
@pytest.mark.parametrize("rk,adapt", [("4", "none"), ("3bs", "basic"), ("5dp", "basic")])
def test_hermitian_mode_matches_full_computation(quac, rk, adapt):
    outs, counts = [], []
    for mode in (1, 0):
        S = H.ProductSystem(quac)
        H.tfim(S, 12)
        quac.construct_matrix(S.qs)
        D = S.D
        rho = quac.create_dm_sys(S.qs)
        rho.from_numpy(H.random_state(D, seed=21, hermitian=True))
        quac.set_hermitian_mode(mode)
        quac.set_ts_options(rk_type=rk, adapt_type=adapt)
        c0 = quac.hermitian_apply_count()
        try:
            quac.time_step_sys(S.qs, rho, 0.0, 0.05, 0.01, 10 ** 6)
        finally:
            quac.set_hermitian_mode(1)
            quac.set_ts_options(rk_type="3bs", adapt_type="basic")
        counts.append(quac.hermitian_apply_count() - c0)
        outs.append(rho.to_numpy())
        rho.destroy()
        S.qs.destroy()
    assert counts[0] > 0 and counts[1] == 0
    assert _rel(outs[0], outs[1]) < 1e-12
    y = outs[0].reshape(4096, 4096, order="F")
    assert np.array_equal(y, y.conj().T) or np.abs(y - y.conj().T).max() < 1e-15 * np.abs(y).max()


def test_hermitian_mode_not_used_for_non_hermitian_state(quac):
    S = H.ProductSystem(quac)
    H.tfim(S, 12)
    quac.construct_matrix(S.qs)
    rho = quac.create_dm_sys(S.qs)
    rho.from_numpy(H.random_state(S.D, seed=22, hermitian=False))
    quac.set_ts_options(rk_type="4", adapt_type="none")
    c0 = quac.hermitian_apply_count()
    try:
        quac.time_step_sys(S.qs, rho, 0.0, 0.02, 0.01, 10 ** 6)
    finally:
        quac.set_ts_options(rk_type="3bs", adapt_type="basic")
    assert quac.hermitian_apply_count() == c0
    rho.destroy()
    S.qs.destroy()


def _herm_state(D, seed):
    """Hermitian (not necessarily positive) test state, cheap at any size."""
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    return ((X + X.conj().T) / 2).reshape(-1, order="F")


# Hermitian mode at every size with two or more passes: tile pairs in the
# first pass (TFIM, canonical terms), general and cross-group terms in both
# passes (pump), three passes (13 qubits)
@pytest.mark.parametrize("n,build", [(7, tfim_real), (8, tfim_real), (10, tfim_real), (9, tfim_pump),
                                     (11, tfim_pump), (13, tfim_real)],
                         ids=["tfim7", "tfim8", "tfim10", "pump9", "pump11", "tfim13"])
def test_hermitian_mode_all_sizes_matches_full_computation(quac, n, build):
    outs, counts = [], []
    x0 = None
    for mode in (1, 0):
        S = H.ProductSystem(quac)
        build(S, n)
        quac.construct_matrix(S.qs)
        D = S.D
        if x0 is None:
            x0 = _herm_state(D, seed=23)
        rho = quac.create_dm_sys(S.qs)
        rho.from_numpy(x0)
        quac.set_hermitian_mode(mode)
        quac.set_ts_options(rk_type="4", adapt_type="none")
        c0 = quac.hermitian_apply_count()
        try:
            quac.time_step_sys(S.qs, rho, 0.0, 0.03, 0.01, 10 ** 6)
        finally:
            quac.set_hermitian_mode(1)
            quac.set_ts_options(rk_type="3bs", adapt_type="basic")
        counts.append(quac.hermitian_apply_count() - c0)
        outs.append(rho.to_numpy())
        rho.destroy()
        S.qs.destroy()
    assert counts[0] >= 12 and counts[0] % 4 == 0 and counts[1] == 0
    assert _rel(outs[0], outs[1]) < 1e-12
    D = 1 << n
    y = outs[0].reshape(D, D, order="F")
    assert np.array_equal(y, y.conj().T)


def test_hermitian_mode_lx_d4096_matches_oracle_rows(quac, oracle):
    """The benchmarked kernel path (12-qubit TFIM, Hermitian mode: tile
    pairs in the high pass, blocks I <= J and their mirrors in the low pass)
    against the oracle's assembled rows, for a low and a high column range
    (the high one written entirely by the mirror epilogue)."""
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, 12)
    H.tfim(O, 12)
    quac.construct_matrix(S.qs)
    D = S.D
    x = _herm_state(D, seed=24)
    quac.set_hermitian_mode(2)
    c0 = quac.hermitian_apply_count()
    try:
        y = quac.lrho_apply_host(S.qs, x)
    finally:
        quac.set_hermitian_mode(1)
    assert quac.hermitian_apply_count() == c0 + 1
    for c_lo, c_hi in [(2, 5), (4000, 4004)]:
        r0, r1 = c_lo * D, c_hi * D
        Ablk = O.liouvillian(rows=(r0, r1))
        assert _rel(y[r0:r1], Ablk @ x) < 1e-12
    Y = y.reshape(D, D, order="F")
    assert np.array_equal(Y, Y.conj().T)
    yfull = quac.lrho_apply_host(S.qs, x)
    assert _rel(y, yfull) < 1e-13
    S.qs.destroy()


@pytest.mark.parametrize("build", [tfim_real, tfim_pump], ids=["tfim13", "pump13"])
def test_three_pass_lx_d8192_matches_oracle_rows(quac, oracle, build):
    """13 qubits: three passes, the middle one over bits 6-11 with fixed bits
    on both sides of its free ones (its TMA box takes the low fixed bits
    into the element dimension, selected by the innermost coordinate).
    L.x of a random (non-Hermitian) vector against the oracle's rows for a
    low and a high column range."""
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    build(S, 13)
    build(O, 13)
    quac.construct_matrix(S.qs)
    D = S.D
    rng = np.random.default_rng(25)
    x = rng.normal(size=D * D) + 1j * rng.normal(size=D * D)
    y = quac.lrho_apply_host(S.qs, x)
    for c_lo, c_hi in [(3, 5), (8189, 8192)]:
        r0, r1 = c_lo * D, c_hi * D
        Ablk = O.liouvillian(rows=(r0, r1))
        assert _rel(y[r0:r1], Ablk @ x) < 1e-12
    S.qs.destroy()
