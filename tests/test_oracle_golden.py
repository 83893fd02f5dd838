"""The oracle against the reference's own golden data (no GPU).

- 48 superoperator fixtures of matrix_construction_test_*.c (Frobenius
  <= 1e-9, the reference tests' bar, t_helpers.h DELTA) plus the 12 MCWF
  effective-Hamiltonian fixtures no reference test reads;
- the shipped conj(a) form of kron.c:723 misses the complex fixtures;
- qvec_utilities_tests.c:788-870 known answers (column-stacked rho);
- quantum_gates_test_sys.c known answers (qubit 0 = most significant);
- time_step_tests.c:337-396 ordering (in-place qubit 0 = last subsystem);
- T1 decay known answer (time_step_tests.c:24-101).
"""
import numpy as np
import pytest
import scipy.sparse as sp

import fixture_systems as F
from conftest import golden_csr


@pytest.mark.parametrize("case", F.CASES, ids=lambda c: f"{c[0]}-{c[1]}op-{c[2]}-{'c' if c[3] else 'r'}")
def test_superoperator_fixture(oracle, golden, case):
    fam, nop, kind, cplx = case
    S = oracle.OSys()
    stems = F.build(S, fam, nop, kind, cplx)
    mode = oracle.MODE_WF if fam == "ham_only" else oracle.MODE_DM
    A = S.liouvillian(mode=mode)
    ref = sum(golden_csr(golden, s) for s in stems)
    assert sp.linalg.norm(A - ref) <= 1e-9


@pytest.mark.parametrize("nop", [1, 2, 3])
@pytest.mark.parametrize("kind", ["basic", "pauli"])
@pytest.mark.parametrize("cplx", [False, True])
def test_mcwf_fixture(oracle, golden, nop, kind, cplx):
    S = oracle.OSys()
    F.build(S, "ham_lin", nop, kind, cplx)
    A = S.liouvillian(mode=oracle.MODE_MCWF)
    stem = f"mcwf_{nop}op_{'b' if kind == 'basic' else 'p'}{'c' if cplx else 'r'}"
    assert sp.linalg.norm(A - golden_csr(golden, stem)) <= 1e-9


def test_shipped_conj_form_misses_complex_fixture(oracle, golden):
    S = oracle.OSys()
    F.build(S, "ham", 1, "basic", True)
    A = S.liouvillian(conj_compat=True)
    assert sp.linalg.norm(A - golden_csr(golden, "ham_1op_bc")) > 1.0


def test_rand_dm_column_stacking(golden):
    v = golden["rand_dm_dat__val"]
    D = 4
    el = lambda r, c: v[D * c + r]
    assert np.isclose(el(0, 0).real, 0.21986779173439994)
    assert np.isclose(el(1, 0), -0.16336963153116132 - 0.05584012449039134j)
    assert np.isclose(el(0, 1), np.conj(el(1, 0)))
    assert np.isclose(el(3, 1), 0.0056141822506085995 + 0.041200982904222694j)
    assert np.isclose(el(3, 3).real, 0.25891270101644115)


def _superop_matrix(oracle, levels, gate, qubits, **kw):
    D = int(np.prod(levels))
    cols = []
    for k in range(D):
        e = np.zeros(D, dtype=complex)
        e[k] = 1
        cols.append(oracle.gate_superop(levels, e, gate, qubits, is_dm=False, **kw))
    return np.array(cols).T


def test_gate_kat_sigmaz_qubit0_is_msb(oracle):
    U = _superop_matrix(oracle, [2, 2], "SIGMAZ", [0])
    assert np.allclose(np.diag(U), [1, 1, -1, -1])
    U = _superop_matrix(oracle, [2, 2], "SIGMAZ", [1])
    assert np.allclose(np.diag(U), [1, -1, 1, -1])


def test_gate_kat_cnot_control_first(oracle):
    U = _superop_matrix(oracle, [2, 2], "CNOT", [0, 1])
    ref = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]])
    assert np.allclose(U, ref)
    U = _superop_matrix(oracle, [2, 2], "CNOT", [1, 0])
    ref = np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]])
    assert np.allclose(U, ref)


def test_gate_kat_hadamard_and_cxz(oracle):
    U = _superop_matrix(oracle, [2], "HADAMARD", [0])
    assert np.allclose(U, np.array([[1, 1], [1, -1]]) / np.sqrt(2))
    U = _superop_matrix(oracle, [2, 2], "CXZ", [0, 1])
    ref = np.eye(4, dtype=complex)
    ref[2:, 2:] = [[0, -1], [1, 0]]
    assert np.allclose(U, ref)


def test_superop_gate_is_u_rho_udag(oracle):
    rng = np.random.default_rng(1)
    levels = [2, 3, 2]
    D = 12
    X = rng.normal(size=(D, D)) + 1j * rng.normal(size=(D, D))
    for gate, q, kw in [("U3", [2], dict(theta=0.3, phi=1.1, lam=-0.4)), ("CNOT", [2, 0], {}),
                        ("RZ", [0], dict(theta=0.7))]:
        out = oracle.gate_superop(levels, X.reshape(-1, order="F"), gate, q, **kw)
        U = _superop_matrix(oracle, levels, gate, q, **kw)
        assert np.allclose(out.reshape(D, D, order="F"), U @ X @ U.conj().T)


def test_inplace_qubit0_is_last_subsystem(oracle):
    # |00><00| on two qubits; SIGMAX on in-place qubit 0 flips the last subsystem
    rho = np.zeros(16, dtype=complex)
    rho[0] = 1
    out = oracle.gate_inplace([2, 2, 2, 2], rho, "SIGMAX", [0])
    D = 4
    assert np.isclose(out[D * 1 + 1], 1.0)


def test_inplace_rz_column_not_conjugated(oracle):
    # the reference's RZ kernel ignores conj_gate: rho_11 picks up e^{2i theta}
    rho = np.zeros(4, dtype=complex)
    rho[3] = 1
    th = 0.3
    out = oracle.gate_inplace([2, 2], rho, "RZ", [0], theta=th)
    assert np.isclose(out[3], np.exp(2j * th))
    sup = oracle.gate_superop([2], rho, "RZ", [0], theta=th)
    assert np.isclose(sup[3], 1.0)


def test_t1_decay_known_answer(oracle):
    S = oracle.OSys()
    o = S.op(2)
    S.lin(1.0, o.a)
    h = S.csr_handle()
    rho = np.zeros(4, dtype=complex)
    rho[3] = 1.0
    y, nacc, nrej = oracle.bs3(h, rho, 0.0, 1.0, 0.05)
    oracle.free_csr(h)
    assert abs(oracle.expect_dm([2], y, o.n).real - np.exp(-1)) < 1e-4


def test_rk4_fixed_step_matches_expm(oracle):
    import scipy.linalg as sl
    S = oracle.OSys()
    q, c = S.op(2), S.op(5)
    S.ham(0.1, c.dag, q.a)
    S.ham(0.1, c.a, q.dag)
    S.lin(1e-2, c.a)
    S.lin(1e-3, q.a)
    A = S.liouvillian().toarray()
    h = S.csr_handle()
    rho = np.zeros(100, dtype=complex)
    rho[5 * 10 + 5] = 1.0
    y = oracle.rk4(h, rho, 0.01, 500)
    oracle.free_csr(h)
    assert np.allclose(y, sl.expm(A * 5.0) @ rho, atol=1e-10)


def test_gmres_steady_state_matches_direct(oracle):
    import scipy.sparse.linalg as sla
    S = oracle.OSys()
    q, c = S.op(2), S.op(4)
    S.ham(0.3, c.dag, q.a)
    S.ham(0.3, c.a, q.dag)
    S.ham(0.2, c.a)
    S.ham(0.2, c.dag)
    S.lin(0.1, c.a)
    S.lin(0.01, q.a)
    x, its = oracle.steady_state(S, rtol=1e-12)
    A = S.liouvillian().tolil()
    D = 8
    for i in range(D):
        A[0, i * (D + 1)] += 1.0
    b = np.zeros(D * D, dtype=complex)
    b[0] = 1
    xd = sla.spsolve(A.tocsr(), b)
    assert np.allclose(x, xd, atol=1e-9)
    assert abs(np.trace(x.reshape(D, D, order="F")) - 1) < 1e-9
