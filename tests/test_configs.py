"""Benchmark configurations end to end against the oracle, and the qvec /
legacy entry points around them (run on a B200: pytest -m gpu).

  config 1  Jaynes-Cummings 2 x 10, fixed RK4 dt = 0.01 to t = 200 with the
            populations read every step (the simple_jc_test monitor form)
  config 2  noisy 10-qubit random circuit: superoperator gates and 1.0 time
            unit of adaptive BS3 per layer, fidelity against the ideal state
  config 3  complex64 contraction against the complex128 oracle (trace,
            populations, fidelity), on the 8-qubit chain the oracle runs
  legacy    create_op / add_to_ham / add_lin / steady_state(Vec) and
            get_populations (operators.c, solver.c, dm_utilities.c)
  qvec      read_qvec_dm_binary on the reference's rand_dm.dat, element
            read-back, PETSc-binary write, set_qvec_from_init_excited_op,
            get_bitstring_probs

Bars: 1e-10 relative for complex128 integrations, 1e-12 for single reads.
"""
import os

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _jc_pops(levels, x):
    """(emitter, cavity) populations of a column-stacked JC state (emitter =
    subsystem 0, the most significant digit)."""
    D = int(np.prod(levels))
    d = x.reshape(D, D, order="F").diagonal().real.reshape(levels)
    return d[1, :].sum(), (d.sum(axis=0) * np.arange(levels[1])).sum()


def test_config1_jc_rk4_t200_populations_match_oracle(quac, oracle):
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    qb, cav = H.jc(S)
    H.jc(O)
    quac.construct_matrix(S.qs)
    rho = quac.create_qvec_sys(S.qs)
    quac.add_to_qvec(rho, 1.0, 10, 10)
    quac.assemble_qvec(rho)
    got = {}

    def monitor(step, t, vec):
        if step % 1000 == 0:
            got[step] = (quac.get_expectation_value_qvec(rho, qb.n).real,
                         quac.get_expectation_value_qvec(rho, cav.n).real)

    quac.set_ts_monitor_sys(S.qs, monitor)
    quac.set_ts_options(rk_type="4", adapt_type="none")
    try:
        quac.time_step_sys(S.qs, rho, 0.0, 200.0, 0.01, 10 ** 6)
    finally:
        quac.set_ts_options(rk_type="3bs", adapt_type="basic")
        quac.set_ts_monitor_sys(S.qs, None)
    assert sorted(got) == list(range(0, 20001, 1000))
    h = O.csr_handle()
    y = np.zeros(400, dtype=complex)
    y[10 * 20 + 10] = 1.0
    for step in range(0, 20001, 1000):
        if step:
            y = oracle.rk4(h, y, 0.01, 1000)
        pe, pc = _jc_pops([2, 10], y)
        ge, gc = got[step]
        assert abs(ge - pe) <= 1e-10 * abs(pe) + 1e-14, (step, ge, pe)
        assert abs(gc - pc) <= 1e-10 * abs(pc) + 1e-14, (step, gc, pc)
    oracle.free_csr(h)
    assert _rel(rho.to_numpy(), y) < 1e-10
    rho.destroy()
    S.qs.destroy()


@pytest.mark.parametrize("batch", [1000, 7])
def test_config1_observable_monitor_matches_oracle(quac, oracle, batch):
    """The same run through the device-side observable monitor (one-CTA
    kernel, many steps per launch): both populations after every one of the
    20,000 steps; every 1000th against the oracle to 1e-10, the rest against
    the final state's by continuity of the record."""
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    qb, cav = H.jc(S)
    H.jc(O)
    quac.construct_matrix(S.qs)
    rho = quac.create_qvec_sys(S.qs)
    quac.add_to_qvec(rho, 1.0, 10, 10)
    quac.assemble_qvec(rho)
    rec = []
    quac.set_observable_monitor(S.qs, [(qb.n,), (cav.n,)], lambda st, tm, v: rec.append((st, tm, v)), batch=batch)
    quac.set_ts_options(rk_type="4", adapt_type="none")
    c0 = quac.kernel_launch_count()
    try:
        quac.time_step_sys(S.qs, rho, 0.0, 200.0, 0.01, 10 ** 6)
    finally:
        quac.set_ts_options(rk_type="3bs", adapt_type="basic")
        quac.set_observable_monitor(S.qs, None, None)
    launches = quac.kernel_launch_count() - c0
    steps = np.concatenate([r[0] for r in rec])
    times = np.concatenate([r[1] for r in rec])
    vals = np.concatenate([r[2] for r in rec])
    assert np.array_equal(steps, np.arange(1, 20001))
    assert abs(times[-1] - 200.0) < 1e-12 and np.all(np.diff(times) > 0)
    assert launches <= 20000 // batch + 2  # many steps per launch
    h = O.csr_handle()
    y = np.zeros(400, dtype=complex)
    y[10 * 20 + 10] = 1.0
    for k in range(1000, 20001, 1000):
        y = oracle.rk4(h, y, 0.01, 1000)
        pe, pc = _jc_pops([2, 10], y)
        assert abs(vals[k - 1, 0].real - pe) <= 1e-10 * abs(pe) + 1e-14
        assert abs(vals[k - 1, 1].real - pc) <= 1e-10 * abs(pc) + 1e-14
    oracle.free_csr(h)
    assert _rel(rho.to_numpy(), y) < 1e-10
    rho.destroy()
    S.qs.destroy()


@pytest.mark.parametrize("layers", [5])
def test_config2_noisy_circuit_matches_oracle(quac, oracle, layers):
    """Each layer: the drawn gates on rho (superoperator convention) and 1.0
    time unit of BS3 (dt0 = 0.1), both against the oracle step for step;
    the state after every layer to 1e-10 and the fidelity against the ideal
    (noiseless) state from both sides."""
    from quac_b200.systems import noisy_circuit_layers, noisy_qubits
    nq = 10
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    noisy_qubits(S, nq)
    noisy_qubits(O, nq)
    quac.construct_matrix(S.qs)
    D = S.D
    rho = quac.create_dm_sys(S.qs)
    quac.add_to_qvec(rho, 1.0, 0, 0)
    quac.assemble_qvec(rho)
    spec = noisy_circuit_layers(nq, layers)
    h = O.csr_handle()
    y = np.zeros(D * D, dtype=complex)
    y[0] = 1.0
    ideal = y.copy()
    levels = [2] * nq
    t = 0.0
    c0 = quac.hermitian_apply_count()
    for layer in spec:
        c = quac.create_circuit(len(layer))
        for g, qbits, kw in layer:
            c.add_gate(0.0, g, *qbits, **kw)
            y = oracle.gate_superop(levels, y, g, list(qbits), **kw)
            ideal = oracle.gate_superop(levels, ideal, g, list(qbits), **kw)
        quac.apply_circuit_to_qvec(S.qs, c, rho)
        quac.time_step_sys(S.qs, rho, t, t + 1.0, 0.1, 10 ** 6)
        y, _, _ = oracle.bs3(h, y, t, t + 1.0, 0.1)
        t += 1.0
        got = rho.to_numpy()
        assert _rel(got, y) < 1e-10
        fid_gpu = float(np.vdot(ideal, got).real)
        fid_orc = float(np.vdot(ideal, y).real)
        assert abs(fid_gpu - fid_orc) < 1e-10
    oracle.free_csr(h)
    # the benchmarked path: these integrations ran in Hermitian mode
    assert quac.hermitian_apply_count() > c0
    assert 0.5 < fid_orc < 1.0
    rho.destroy()
    S.qs.destroy()


def test_config3_fp32_contraction_errors_against_oracle(quac, oracle):
    """The precision form of config 3 on the 8-qubit chain the oracle can
    integrate: DP5 at rtol = atol = 1e-8 to t = 5 with complex64
    contraction against the oracle's complex128 DP5, per result."""
    n = 8
    S = H.ProductSystem(quac)
    O = oracle.OSys()
    H.tfim(S, n)
    H.tfim(O, n)
    quac.construct_matrix(S.qs)
    D = S.D
    x0 = np.zeros(D * D, dtype=complex)
    x0[0] = 1.0
    out = {}
    for prec in (0, 1):
        rho = quac.create_dm_sys(S.qs)
        rho.from_numpy(x0)
        quac.set_lrho_precision(prec)
        quac.set_ts_options(rk_type="5dp", adapt_type="basic", rtol=1e-8, atol=1e-8)
        try:
            quac.time_step_sys(S.qs, rho, 0.0, 5.0, 0.01, 10 ** 6)
        finally:
            quac.set_lrho_precision(0)
            quac.set_ts_options(rk_type="3bs", adapt_type="basic", rtol=5e-7, atol=5e-7)
        out[prec] = rho.to_numpy().reshape(D, D, order="F")
        rho.destroy()
    h = O.csr_handle()
    yo, _, _ = oracle.dp5(h, x0, 0.0, 5.0, 0.01, atol=1e-8, rtol=1e-8)
    oracle.free_csr(h)
    Y = yo.reshape(D, D, order="F")
    assert _rel(out[0], Y) < 1e-10
    B = out[1]
    # fidelity F = (Tr sqrt(sqrt(A) B sqrt(A)))^2 against the oracle state
    w, V = np.linalg.eigh(Y)
    sa = (V * np.sqrt(np.clip(w, 0, None))) @ V.conj().T
    ev = np.linalg.eigvalsh(sa @ ((B + B.conj().T) / 2) @ sa)
    fid = float(np.sum(np.sqrt(np.clip(ev, 0, None))) ** 2)
    assert abs(np.trace(B) - np.trace(Y)) < 1e-6
    assert np.abs(B.diagonal().real - Y.diagonal().real).max() < 1e-6
    assert abs(fid - 1.0) < 1e-6


def test_legacy_steady_state_matches_direct_solve(quac, oracle):
    """steady_state(Vec) on the legacy global system (create_op, add_to_ham,
    add_to_ham_mult2, add_lin; solver.c:33-221, operators.c:290-337,
    679-719), with get_populations (dm_utilities.c:1157-1325)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    q = quac
    qb = q.create_op(2)
    cav = q.create_op(5)
    q.add_to_ham(0.2, cav.n)
    q.add_to_ham_mult2(0.1, cav.dag, qb)
    q.add_to_ham_mult2(0.1, cav, qb.dag)
    q.add_to_ham(0.15, cav)
    q.add_to_ham(0.15, cav.dag)
    q.add_lin(0.05, cav)
    q.add_lin(2e-3, qb)
    rho = q.create_full_dm()
    q.steady_state(rho)
    x = rho.to_numpy()
    O = oracle.OSys()
    oq, oc = O.op(2), O.op(5)
    O.ham(0.2, oc.n)
    O.ham(0.1, oc.dag, oq.a)
    O.ham(0.1, oc.a, oq.dag)
    O.ham(0.15, oc.a)
    O.ham(0.15, oc.dag)
    O.lin(0.05, oc.a)
    O.lin(2e-3, oq.a)
    L = O.liouvillian().tocsr()
    D = 10
    n = D * D
    A = (L + sp.csr_matrix((np.eye(D).reshape(-1, order="F"), (np.zeros(n, int), np.arange(n))),
                           shape=(n, n))).tocsc()
    b = np.zeros(n, complex)
    b[0] = 1.0
    xs = spla.spsolve(A, b)
    assert _rel(x, xs) < 1e-8
    pops = q.get_populations(rho)
    X = xs.reshape(D, D, order="F").diagonal().real.reshape(2, 5)
    assert abs(pops[0] - X[1, :].sum()) < 1e-9
    assert abs(pops[1] - (X.sum(axis=0) * np.arange(5)).sum()) < 1e-9
    assert abs(q.get_dm_element(rho, 3, 3) - xs[3 * D + 3]) < 1e-9
    rho.destroy()


def test_legacy_time_step_matches_time_step_sys(quac):
    """time_step(Vec) on the legacy global system (solver.c:236-510) after
    QuaC_clear (quac.c:60-80) gives the state time_step_sys gives for the
    same terms, and calls the set_ts_monitor callback at every step."""
    q = quac
    q.QuaC_clear()
    qb = q.create_op(2)
    cav = q.create_op(5)
    q.add_to_ham(0.2, cav.n)
    q.add_to_ham_mult2(0.1, cav.dag, qb)
    q.add_to_ham_mult2(0.1, cav, qb.dag)
    q.add_to_ham(0.15, cav)
    q.add_to_ham(0.15, cav.dag)
    q.add_lin(0.05, cav)
    q.add_lin(2e-3, qb)
    rho = q.create_full_dm()
    q.add_value_to_dm(rho, 5, 5, 1.0)  # emitter excited, cavity empty
    q.assemble_dm(rho)
    steps = []
    q.set_ts_monitor(lambda step, t, vec: steps.append((step, t)))
    try:
        q.time_step(rho, 0.0, 2.0, 0.05, 10 ** 6)
    finally:
        q.set_ts_monitor(None)
    x = rho.to_numpy()
    rho.destroy()
    q.QuaC_clear()
    S = H.ProductSystem(q)
    sq, sc = S.op(2), S.op(5)
    S.ham(0.2, sc.n)
    S.ham(0.1, sc.dag, sq.a)
    S.ham(0.1, sc.a, sq.dag)
    S.ham(0.15, sc.a)
    S.ham(0.15, sc.dag)
    S.lin(0.05, sc.a)
    S.lin(2e-3, sq.a)
    q.construct_matrix(S.qs)
    r2 = q.create_qvec_sys(S.qs)
    q.add_to_qvec(r2, 1.0, 5, 5)
    q.assemble_qvec(r2)
    q.time_step_sys(S.qs, r2, 0.0, 2.0, 0.05, 10 ** 6)
    assert _rel(x, r2.to_numpy()) < 1e-12
    assert len(steps) > 1 and steps[-1][1] == pytest.approx(2.0)
    r2.destroy()
    S.qs.destroy()


def test_read_reference_dm_binary_and_elements(quac, golden, tmp_path):
    """read_qvec_dm_binary on the reference's own rand_dm.dat bytes and the
    element read-back of qvec_utilities_tests.c:788-870 (column stacking:
    element (1, 0) at vector index 1); print_qvec_file writes the same bytes."""
    src = tmp_path / "rand_dm.dat"
    src.write_bytes(golden["rand_dm_dat__raw"].tobytes())
    dm = quac.read_qvec_dm_binary(str(src))
    assert dm.n == 16
    for (r, c), v in {(0, 0): 0.21986779173439994, (1, 0): -0.16336963153116132 - 0.05584012449039134j,
                      (3, 1): 0.0056141822506085995 + 0.041200982904222694j,
                      (3, 3): 0.25891270101644115}.items():
        assert abs(quac.get_dm_element_qvec(dm, r, c) - v) < 1e-12
        assert abs(quac.get_dm_element_qvec(dm, c, r) - np.conj(v)) < 1e-12
    assert np.array_equal(dm.to_numpy(), golden["rand_dm_dat__val"])
    out = tmp_path / "back.dat"
    quac.print_qvec_file(dm, str(out))
    assert out.read_bytes() == src.read_bytes()
    probs = quac.get_bitstring_probs(dm)
    assert np.allclose(probs, golden["rand_dm_dat__val"].reshape(4, 4, order="F").diagonal().real, atol=0)
    dm.destroy()
    wsrc = tmp_path / "rand_wf.dat"
    wsrc.write_bytes(golden["rand_wf_dat__raw"].tobytes())
    wf = quac.read_qvec_wf_binary(str(wsrc))
    assert np.array_equal(wf.to_numpy(), golden["rand_wf_dat__val"])
    assert np.allclose(quac.get_bitstring_probs(wf), np.abs(golden["rand_wf_dat__val"]) ** 2, atol=0)
    wf.destroy()


def test_set_qvec_from_init_excited_op(quac):
    """qvec_utilities.c:2540-2566: the initial excitations of the subsystems
    select one basis state through n_after strides (subsystem 0 = most
    significant digit); a density matrix gets |i><i|."""
    q = quac
    qs = q.initialize_system()
    a, b, c = q.create_op_sys(qs, 3), q.create_op_sys(qs, 2), q.create_op_sys(qs, 4)
    q.add_lin_term(qs, 0.1, a)
    q.set_init_excited_op(a, 2)
    q.set_init_excited_op(b, 1)
    q.set_init_excited_op(c, 3)
    q.construct_matrix(qs)
    rho = q.create_qvec_sys(qs)
    q.set_qvec_from_init_excited_op(qs, rho)
    q.assemble_qvec(rho)
    i = 2 * (2 * 4) + 1 * 4 + 3
    D = 24
    x = rho.to_numpy()
    assert x[i * D + i] == 1.0 and np.count_nonzero(x) == 1
    assert q.get_dm_element_qvec(rho, i, i) == 1.0
    rho.destroy()
    qs.destroy()


@pytest.mark.parametrize("kind", ["wf", "dm"])
def test_add_to_qvec_fock_op_expectations(quac, kind):
    """tests/qvec_utilities_tests.c test_get_expectation_value_wf_real /
    _dm_real: |11> set through add_to_qvec_fock_op on two qubits gives
    <n1> = <n2> = 1 and <qd1^dag qd2> = <qd2^dag qd1> = 0."""
    q = quac
    qs = q.initialize_system()
    qd1, qd2 = q.create_op_sys(qs, 2), q.create_op_sys(qs, 2)
    v = q.create_wf_sys(qs) if kind == "wf" else q.create_dm_sys(qs)
    q.add_to_qvec_fock_op(1.0, v, qd1, 1, qd2, 1)
    q.assemble_qvec(v)
    assert q.get_expectation_value_qvec(v, qd1.n) == 1.0
    assert q.get_expectation_value_qvec(v, qd2.n) == 1.0
    assert q.get_expectation_value_qvec(v, qd1.dag, qd2) == 0.0
    assert q.get_expectation_value_qvec(v, qd2.dag, qd1) == 0.0
    x = v.to_numpy()
    assert np.count_nonzero(x) == 1 and x[3 if kind == "wf" else 3 * 4 + 3] == 1.0
    v.destroy()
    qs.destroy()


def test_circuit_events_inside_time_step_match_oracle(quac, oracle):
    """Gates scheduled at times inside one time_step_sys run (in-place
    engine, quantum_circuits.c:17-120): the integration stops on every
    event time, applies the gates and continues the same controller,
    against the oracle's restatement (oracle.bs3_events) step for step."""
    q = quac
    S = H.ProductSystem(q)
    O = oracle.OSys()
    for T in (S, O):
        qs_ = [T.op(2) for _ in range(3)]
        T.ham(0.4, qs_[0].sig_x)
        T.ham(0.25, qs_[1].sig_z, qs_[2].sig_z)
        T.lin(0.05, qs_[0].a)
        T.lin(0.02, qs_[2].n)
    q.construct_matrix(S.qs)
    rho = q.create_qvec_sys(S.qs)
    q.add_to_qvec(rho, 1.0, 0, 0)
    q.assemble_qvec(rho)
    circ = q.create_circuit(5)
    gates = [(0.3, "HADAMARD", (0,), {}), (0.3, "CNOT", (0, 2), {}), (0.85, "RZ", (1,), dict(theta=0.7)),
             (1.4, "U3", (2,), dict(theta=0.3, phi=1.1, lam=-0.4)), (1.4, "SIGMAX", (1,), {})]
    for t, g, qb, kw in gates:
        q.add_gate_to_circuit_sys(circ, t, g, *qb, **kw)
    q.apply_circuit_to_sys(S.qs, circ, 0.0)
    q.time_step_sys(S.qs, rho, 0.0, 2.0, 0.05, 10 ** 6)
    dims = [2] * 6
    evs = [(t, (lambda g, qb, kw: (lambda y: oracle.gate_inplace(dims, y, g, list(qb), **kw)))(g, qb, kw))
           for t, g, qb, kw in gates]
    h = O.csr_handle()
    x0 = np.zeros(64, dtype=complex)
    x0[0] = 1.0
    yo, _ = oracle.bs3_events(h, x0, 0.0, 2.0, 0.05, evs)
    oracle.free_csr(h)
    assert _rel(rho.to_numpy(), yo) < 1e-10
    # RY has no in-place form in the reference either
    # (quantum_circuits.c:3007-3035): the run stops with its message
    bad = q.create_circuit(1)
    q.add_gate_to_circuit_sys(bad, 2.5, "RY", 1, theta=0.7)
    q.apply_circuit_to_sys(S.qs, bad, 0.0)
    with pytest.raises(q.QuacError, match="get_gate_func_wf"):
        q.time_step_sys(S.qs, rho, 2.0, 3.0, 0.05, 10 ** 6)
    rho.destroy()
    S.qs.destroy()
