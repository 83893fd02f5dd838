"""Monte-Carlo wavefunction trajectories (use_mcwf_solver, qsystem.c:358-403,
1139-1235; effective Hamiltonian kron.c:664-700).

  * the reference's known-answer tests (time_step_tests.c:103-191,
    287-335): T1 decay of a qubit and of a qubit + three-level system, 1000
    trajectories, <n> within 2/sqrt(1000) of the analytic value, also with
    the run split into ten restarts;
  * trajectory by trajectory against the oracle's restatement of the same
    algorithm (oracle.McwfEnsemble: the same random stream, integrator,
    jump location and jump choice): every final state to 1e-10, the same
    jump counts, adaptive BS3 and fixed RK4;
  * the effective Hamiltonian against the oracle's MCWF operator;
  * host-side checks (no GPU): use_mcwf_solver's argument checks.
"""
import numpy as np
import pytest

import helpers as H


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _t1(q, restarts=1, seed=42):
    qs = q.initialize_system()
    op2 = q.create_op_sys(qs, 2)
    q.add_ham_term(qs, 1.0, op2.n)
    q.add_lin_term(qs, 1.0, op2)
    q.use_mcwf_solver(qs, 1000, seed)
    wf = q.create_qvec_sys(qs)
    q.add_to_qvec(wf, 1.0, 1)
    q.assemble_qvec(wf)
    q.construct_matrix(qs)
    for i in range(restarts):
        q.time_step_sys(qs, wf, i / restarts, (i + 1) / restarts, 0.01, 1000)
    v = q.get_expectation_value_qvec(wf, op2.n).real
    wf.destroy()
    qs.destroy()
    return v


@pytest.mark.gpu
@pytest.mark.parametrize("restarts", [1, 10])
def test_mcwf_t1_decay_known_answer(quac, restarts):
    assert abs(_t1(quac, restarts) - np.exp(-1)) < 2 / np.sqrt(1000)


@pytest.mark.gpu
def test_mcwf_t1_decay_two_systems_known_answer(quac):
    q = quac
    qs = q.initialize_system()
    op3 = q.create_op_sys(qs, 3)
    op2 = q.create_op_sys(qs, 2)
    q.add_ham_term(qs, 1.0, op2.n)
    q.add_lin_term(qs, 1.0, op2)
    q.add_lin_term(qs, 1.0, op3)
    q.use_mcwf_solver(qs, 1000, 7)
    wf = q.create_qvec_sys(qs)
    q.add_to_qvec(wf, 1.0, 5)
    q.assemble_qvec(wf)
    assert abs(q.get_expectation_value_qvec(wf, op2.n) - 1.0) < 1e-12  # not spawned yet: plain WF
    q.construct_matrix(qs)
    q.time_step_sys(qs, wf, 0.0, 1.0, 0.05, 2000)
    assert abs(q.get_expectation_value_qvec(wf, op2.n).real - np.exp(-1)) < 2 / np.sqrt(1000)
    assert abs(q.get_expectation_value_qvec(wf, op3.n).real - 2 * np.exp(-1)) < 2 / np.sqrt(1000)
    wf.destroy()
    qs.destroy()


def _driven(S):
    qb = S.op(2)
    cav = S.op(4)
    S.ham(0.4, cav.n)
    S.ham(0.3, cav.dag, qb.a)
    S.ham(0.3, cav.a, qb.dag)
    S.ham(0.2, cav.a)
    S.ham(0.2, cav.dag)
    S.lin(0.3, cav.a)
    S.lin(0.1, qb.a)
    S.lin(0.05, qb.n)
    return qb, cav


@pytest.mark.gpu
@pytest.mark.parametrize("rk,adapt,scheme", [("3bs", "basic", 0), ("4", "none", 2)], ids=["bs3", "rk4"])
def test_mcwf_trajectories_match_oracle(quac, oracle, rk, adapt, scheme):
    q = quac
    ntraj, seed = 256, 2024
    S = H.ProductSystem(q)
    qb, cav = _driven(S)
    q.use_mcwf_solver(S.qs, ntraj, seed)
    wf = q.create_qvec_sys(S.qs)
    q.add_to_qvec(wf, 1.0, 4)  # |1> (excited emitter) x |0>
    q.assemble_qvec(wf)
    q.construct_matrix(S.qs)
    q.set_ts_options(rk_type=rk, adapt_type=adapt)
    try:
        q.time_step_sys(S.qs, wf, 0.0, 2.5, 0.02, 10 ** 6)
        q.time_step_sys(S.qs, wf, 2.5, 5.0, 0.02, 10 ** 6)
    finally:
        q.set_ts_options(rk_type="3bs", adapt_type="basic")
    states, stats = q.mcwf_states(wf)
    O = oracle.OSys()
    _, ocav = _driven(O)
    psi0 = np.zeros(8, complex)
    psi0[4] = 1.0
    E = oracle.McwfEnsemble(O, psi0, ntraj, seed)
    E.run(0.0, 2.5, 0.02, scheme=scheme)
    E.run(2.5, 5.0, 0.02, scheme=scheme)
    assert np.array_equal(stats[:, 1], E.stats[1::2])
    assert stats[:, 1].sum() > ntraj // 4  # jumps happened
    for i in range(ntraj):
        assert _rel(states[i], E.psi[i]) < 1e-10, i
    got = q.get_expectation_value_qvec(wf, cav.n)
    assert abs(got - E.expectation([2, 4], ocav.n)) < 1e-10
    E.free()
    wf.destroy()
    S.qs.destroy()


def test_mcwf_argument_checks(quac):
    q = quac
    qs = q.initialize_system()
    op = q.create_op_sys(qs, 2)
    q.add_ham_term(qs, 1.0, op.n)
    with pytest.raises(q.QuacError):
        q.use_mcwf_solver(qs, 10, 1)  # no Lindblad term
    q.add_lin_term(qs, 1.0, op)
    with pytest.raises(q.QuacError):
        q.use_mcwf_solver(qs, 1, 1)  # fewer than 2 trajectories
    q.use_mcwf_solver(qs, 10, 1)
    assert qs._ptr.contents.mcwf_solver == 1
    qs.destroy()
