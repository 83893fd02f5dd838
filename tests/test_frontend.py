"""Circuit front ends (qasm_parser.c): OpenQASM 2 (qiskit and cirq qubit
orders, timed form), ProjectQ command logs and Quil.  Parsing runs on the
host; the GPU test applies a parsed circuit to a density matrix against
the oracle's gates."""
import math

import numpy as np
import pytest

GATES = None


def _g(quac):
    return quac.GATES


QASM = """OPENQASM 2.0;
include "qelib1.inc";
qreg qr[3];
creg cr[3];
h qr[0];
cx qr[0],qr[1];
// a comment line
rz(pi/4) qr[2];
u3(0.3,-pi/2,2*pi/3) qr[1];

barrier qr[0],qr[1];
u2(pi/2,-0.25) qr[2];
u1(-3*pi/4) qr[0];
rx(-pi) qr[1];
"""


def test_qiskit_qasm_read(quac, tmp_path):
    f = tmp_path / "c.qasm"
    f.write_text(QASM)
    nq, c = quac.qiskit_qasm_read(str(f))
    G = quac.GATES
    gates = quac.circuit_gates(c)
    assert nq == 3
    want = [(1, G["HADAMARD"], (2,), 0, 0, 0), (2, G["CNOT"], (2, 1), 0, 0, 0),
            (3, G["RZ"], (0,), math.pi / 4, 0, 0), (4, G["U3"], (1,), 0.3, -math.pi / 2, 2 * math.pi / 3),
            (6, G["U2"], (0,), math.pi / 2, math.pi / 2, -0.25), (7, G["U1"], (2,), 0, 0, -3 * math.pi / 4),
            (8, G["RX"], (1,), -math.pi, 0, 0)]
    assert len(gates) == len(want)
    for g, w in zip(gates, want):
        assert g[1:3] == w[1:3] and g[0] == w[0]
        assert np.allclose(g[3:], w[3:], atol=1e-15)
    c.destroy()


def test_cirq_and_timed_qasm_read(quac, tmp_path):
    f = tmp_path / "c.qasm"
    f.write_text(QASM)
    nq, c = quac.cirq_qasm_read(str(f))
    assert nq == 3 and quac.circuit_gates(c)[1][2] == (0, 1)  # file qubit order kept
    c.destroy()
    f2 = tmp_path / "t.qasm"
    f2.write_text('OPENQASM 2.0;\ninclude "qelib1.inc";\nqreg qr[2];\nh qr[0] @0.5;\ncx qr[0],qr[1] @1.25;\n'
                  'rz(pi) qr[1] @2.0;\n')
    nq, c = quac.qiskit_tqasm_read(str(f2))
    gates = quac.circuit_gates(c)
    assert nq == 2 and [g[0] for g in gates] == [0.5, 1.25, 2.0]
    assert gates[1][2] == (0, 1) and abs(gates[2][3] - math.pi) < 1e-15
    c.destroy()


def test_projectq_qasm_read(quac, tmp_path):
    f = tmp_path / "p.txt"
    f.write_text("Allocate | Qureg[0]\nAllocate | Qureg[1]\nH | Qureg[0]\nCX | ( Qureg[0], Qureg[1] )\n"
                 "Rz(0.5) | Qureg[1]\nRx(-1.25) | Qureg[0]\nDeallocate | Qureg[0]\nDeallocate | Qureg[1]\n")
    nq, c = quac.projectq_qasm_read(str(f))
    G = quac.GATES
    gates = quac.circuit_gates(c)
    assert nq == 2
    assert [(g[0], g[1], g[2]) for g in gates] == [(1, G["HADAMARD"], (0,)), (2, G["CNOT"], (0, 1)),
                                                    (3, G["RZ"], (1,)), (4, G["RX"], (0,))]
    assert gates[2][3] == 0.5 and gates[3][3] == -1.25
    c.destroy()


def test_quil_read(quac, tmp_path):
    f = tmp_path / "p.quil"
    f.write_text("PRAGMA INITIAL_REWIRING \"PARTIAL\"\nH 0\nCNOT 1 0\nRX(pi/2) 2\nRZ(-3*pi/4) 1\nCZ 2 1\n")
    nq, c = quac.quil_read(str(f))
    G = quac.GATES
    gates = quac.circuit_gates(c)
    assert nq == 3
    assert [(g[0], g[1], g[2]) for g in gates] == [(1, G["HADAMARD"], (0,)), (2, G["CNOT"], (1, 0)),
                                                    (3, G["RX"], (2,)), (4, G["RZ"], (1,)), (5, G["CZ"], (2, 1))]
    assert abs(gates[2][3] - math.pi / 2) < 1e-15 and abs(gates[3][3] + 3 * math.pi / 4) < 1e-15
    c.destroy()


def test_reader_errors(quac, tmp_path):
    f = tmp_path / "bad.qasm"
    f.write_text('OPENQASM 2.0;\nqreg qr[2];\nfoo qr[0];\n')
    with pytest.raises(quac.QuacError):
        quac.qiskit_qasm_read(str(f))
    with pytest.raises(quac.QuacError):
        quac.quil_read(str(tmp_path / "missing.quil"))


@pytest.mark.gpu
def test_parsed_circuit_on_density_matrix_matches_oracle(quac, oracle, tmp_path):
    """The qiskit file applied with apply_circuit_to_qvec (superoperator
    convention) against the oracle's gates in the same order."""
    f = tmp_path / "c.qasm"
    f.write_text(QASM)
    nq, c = quac.qiskit_qasm_read(str(f))
    qs = quac.initialize_system()
    ops = [quac.create_op_sys(qs, 2) for _ in range(nq)]
    quac.add_lin_term(qs, 1e-3, ops[0])
    quac.construct_matrix(qs)
    rho = quac.create_dm_sys(qs)
    quac.add_to_qvec(rho, 1.0, 0, 0)
    quac.assemble_qvec(rho)
    quac.apply_circuit_to_qvec(qs, c, rho)
    y = np.zeros(64, complex)
    y[0] = 1.0
    for t, g, qb, th, ph, la in quac.circuit_gates(c):
        y = oracle.gate_superop([2] * nq, y, int(g), list(qb), theta=th, phi=ph, lam=la)
    assert np.linalg.norm(rho.to_numpy() - y) < 1e-12
    rho.destroy()
    c.destroy()
    qs.destroy()
