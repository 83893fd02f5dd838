"""Time-dependent terms (add_ham_term_time_dep / add_lin_term_time_dep,
qsystem.c:491-552, applied as in _time_dep_mat_mult, qsystem.c:1300-1330).

  * the reference's own known-answer test (time_dep_tests.c:130-220): a
    qubit driven by pi e^{-alpha t} sigma_x from |0>, sigma_x/y/z after
    every step against the analytic rotation, within 1e-4, default adaptive
    Bogacki-Shampine;
  * fixed-step RK4 against the oracle's restatement of the time-dependent
    right-hand side (oracle.rk4_time_dep) at 1e-10, density matrix with a
    time-dependent drive and a time-dependent decay rate, and wavefunction
    form;
  * host-side checks (no GPU): the API records the terms.
"""
import numpy as np
import pytest

import helpers as H


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.gpu
def test_time_dep_wf_rabi_known_answer(quac):
    q = quac
    alpha, omega = 0.1, 2 * np.pi
    qs = q.initialize_system()
    op2 = q.create_op_sys(qs, 2)
    pulse = lambda t: np.exp(-alpha * t)
    q.add_ham_term_time_dep(qs, 0.5 * omega, pulse, op2)
    q.add_ham_term_time_dep(qs, 0.5 * omega, pulse, op2.dag)
    wf = q.create_qvec_sys(qs)
    q.add_to_qvec(wf, 1.0, 0)
    q.assemble_qvec(wf)
    q.construct_matrix(qs)
    diffs = []

    def monitor(step, t, vec):
        th = omega * (1 - np.exp(-alpha * t)) / alpha
        sz = q.get_expectation_value_qvec(wf, op2.sig_z)
        sy = q.get_expectation_value_qvec(wf, op2.sig_y)
        sx = q.get_expectation_value_qvec(wf, op2.sig_x)
        diffs.append(max(abs(sz - np.cos(th)), abs(sy + np.sin(th)), abs(sx)))

    q.set_ts_monitor_sys(qs, monitor)
    q.time_step_sys(qs, wf, 0.0, 20.0, 0.01, 10 ** 6)
    q.set_ts_monitor_sys(qs, None)
    assert len(diffs) > 100
    assert max(diffs) < 1e-4
    wf.destroy()
    qs.destroy()


def _drive(t):
    return np.cos(1.3 * t) * np.exp(-0.2 * t)


def _ramp(t):
    return 1.0 + 0.5 * np.sin(0.7 * t)


def _build_dm(S):
    qb = S.op(2)
    cav = S.op(5)
    S.ham(0.3, cav.n)
    S.ham(0.1, cav.dag, qb.a)
    S.ham(0.1, cav.a, qb.dag)
    S.lin(0.02, qb.a)
    return qb, cav


@pytest.mark.gpu
def test_time_dep_dm_rk4_matches_oracle(quac, oracle):
    q = quac
    S = H.ProductSystem(q)
    qb, cav = _build_dm(S)
    q.add_ham_term_time_dep(S.qs, 0.4, _drive, cav)
    q.add_ham_term_time_dep(S.qs, 0.4, _drive, cav.dag)
    q.add_lin_term_time_dep(S.qs, 0.05, _ramp, cav)
    q.construct_matrix(S.qs)
    D = S.D
    rho = q.create_qvec_sys(S.qs)
    q.add_to_qvec(rho, 1.0, 5, 5)
    q.assemble_qvec(rho)
    q.set_ts_options(rk_type="4", adapt_type="none")
    try:
        q.time_step_sys(S.qs, rho, 0.0, 2.0, 0.01, 10 ** 6)
    finally:
        q.set_ts_options(rk_type="3bs", adapt_type="basic")
    O = oracle.OSys()
    _build_dm(O)
    h0 = O.csr_handle()
    hk = []
    for kind, build, a, f in [("h", lambda T, c: T.ham(1.0, c.a), 0.4, _drive),
                              ("h", lambda T, c: T.ham(1.0, c.dag), 0.4, _drive),
                              ("l", lambda T, c: T.lin(1.0, c.a), 0.05, _ramp)]:
        T = oracle.OSys()
        T.op(2)
        c = T.op(5)
        build(T, c)
        hk.append((T.csr_handle(), a, f))
    x0 = np.zeros(D * D, dtype=complex)
    x0[5 * D + 5] = 1.0
    yo = oracle.rk4_time_dep(h0, hk, x0, 0.0, 0.01, 200)
    oracle.free_csr(h0)
    for h, _, _ in hk:
        oracle.free_csr(h)
    assert _rel(rho.to_numpy(), yo) < 1e-10
    rho.destroy()
    S.qs.destroy()


@pytest.mark.gpu
def test_time_dep_wf_rk4_matches_oracle(quac, oracle):
    q = quac
    S = H.ProductSystem(q)
    a = S.op(3)
    b = S.op(2)
    S.ham(0.5, a.n)
    S.ham(0.2, a.dag, b.a)
    S.ham(0.2, a.a, b.dag)
    q.add_ham_term_time_dep(S.qs, 0.3 + 0.1j, _drive, a)
    q.add_ham_term_time_dep(S.qs, 0.3 - 0.1j, _drive, a.dag)
    q.construct_matrix(S.qs)
    wf = q.create_qvec_sys(S.qs)
    q.add_to_qvec(wf, 1.0, 1)
    q.assemble_qvec(wf)
    q.set_ts_options(rk_type="4", adapt_type="none")
    try:
        q.time_step_sys(S.qs, wf, 0.0, 1.5, 0.01, 10 ** 6)
    finally:
        q.set_ts_options(rk_type="3bs", adapt_type="basic")
    O = oracle.OSys()
    oa, ob = O.op(3), O.op(2)
    O.ham(0.5, oa.n)
    O.ham(0.2, oa.dag, ob.a)
    O.ham(0.2, oa.a, ob.dag)
    h0 = O.csr_handle(mode=oracle.MODE_WF)
    hk = []
    for c, f in [(0.3 + 0.1j, lambda T, x: T.ham(1.0, x.a)), (0.3 - 0.1j, lambda T, x: T.ham(1.0, x.dag))]:
        T = oracle.OSys()
        x = T.op(3)
        T.op(2)
        f(T, x)
        hk.append((T.csr_handle(mode=oracle.MODE_WF), c, _drive))
    x0 = np.zeros(6, dtype=complex)
    x0[1] = 1.0
    yo = oracle.rk4_time_dep(h0, hk, x0, 0.0, 0.01, 150)
    oracle.free_csr(h0)
    for h, _, _ in hk:
        oracle.free_csr(h)
    assert _rel(wf.to_numpy(), yo) < 1e-10
    wf.destroy()
    S.qs.destroy()


def test_time_dep_terms_recorded_on_host(quac):
    q = quac
    qs = q.initialize_system()
    op = q.create_op_sys(qs, 2)
    q.add_ham_term_time_dep(qs, 1.0, lambda t: 1.0, op)
    assert qs._ptr.contents.num_time_dep == 1 and not qs.dm_equations
    q.add_lin_term_time_dep(qs, 0.1, lambda t: 1.0, op)
    assert qs._ptr.contents.num_time_dep == 2 and qs.dm_equations
    q.clear_mat_terms_sys(qs)
    assert qs._ptr.contents.num_time_dep == 0
    qs.destroy()
