"""Front-end types on the CPU: operator canonicalisation, circuit validation and monomial expansion
(conventions of the reference's src/monoprop/{majorana,pauli,circuit}.py)."""

import numpy as np
import pytest

from monoprop_b200 import Circuit, ExpGate, Majorana, MajoranaOperator, Pauli, PauliOperator, expand_monomials
from monoprop_b200 import workloads as W


def test_majorana_canonicalisation_sign_and_pairs():
    assert Majorana.from_unsorted(2, 1) == (Majorana(1, 2), -1.0)
    assert Majorana.from_unsorted(3, 1, 2) == (Majorana(1, 2, 3), 1.0)
    assert Majorana.from_unsorted(1, 2, 1) == (Majorana(2), -1.0)
    op = MajoranaOperator({(1, 0): 1.0, (0, 1): 2.0}, num_modes=1)
    assert op.terms == {(0, 1): 1.0 + 0j}
    with pytest.raises(ValueError):
        MajoranaOperator({(0, 4): 1.0}, num_modes=2)


def test_pauli_slots_roundtrip():
    p = Pauli("XYZ", (3, 0, 5))
    assert p.string == "YXZ" and p.qubits == (0, 3, 5)
    assert p.slots() == (1, 6, 10, 11)
    assert Pauli.from_slots(p.slots()) == p
    assert PauliOperator({Pauli("ZZ", (1, 2)): 0.5}, 3).get_local_operator().terms == {(2, 3, 4, 5): 0.5 + 0j}


def test_expand_monomials_matches_workload_arrays():
    wl = W.line20()
    n = 20
    gates = []
    for slots in wl.gate_slots:
        q = sorted({s // 2 for s in slots})
        gates.append(ExpGate(PauliOperator({Pauli("ZZ" if len(slots) == 4 else "X", q): -0.5}, n)))
    circ = Circuit(gates, n, wl.params)
    monos, g, mapping, gidx = expand_monomials(circ.gates, circ.resolved_mapping, n)
    assert monos == wl.gate_slots
    assert np.array_equal(g, wl.gen_coeffs) and np.array_equal(mapping, wl.param_map)
    assert gidx == list(range(wl.n_layers))


def test_majorana_generator_normalisation():
    # exp(+i t H) with H = i m0 m1 (Hermitian): engine g = -coeff / i^C(2,2) = -(i)/i = -1
    gate = ExpGate(MajoranaOperator({(0, 1): 1j}, 2))
    assert gate.layers() == [((0, 1), -1.0)]
    with pytest.raises(ValueError):
        ExpGate(MajoranaOperator({(0, 1): 1.0}, 2)).layers()  # non-Hermitian generator
    with pytest.raises(ValueError):
        ExpGate(MajoranaOperator({(0, 1): 1j, (1, 2): 1j}, 2))  # non-commuting terms


def test_circuit_mapping_rules():
    g0 = ExpGate(PauliOperator({"X": 1.0}, 1), index=0)
    g1 = ExpGate(PauliOperator({"Z": 1.0}, 1), index=0)
    c = Circuit([g0, g1], 1, [0.3])
    assert c.resolved_mapping == (0, 0) and c.n_parameters == 1
    with pytest.raises(ValueError):
        Circuit([g0, ExpGate(PauliOperator({"Z": 1.0}, 1))], 1)  # mixed explicit/default index
    with pytest.raises(ValueError):
        Circuit([ExpGate(PauliOperator({"X": 1.0}, 1), index=1)], 1)  # gap in indices
    d = Circuit.from_dense_arrays([(0, 1), (2, 3), (1, 2)], [1.0, -1.0, 0.5], [0, 0, 1], 2, [0.1, 0.2])
    assert len(d) == 2 and d.resolved_mapping == (0, 1)
    monos, g, mapping, gidx = expand_monomials(d.gates, d.resolved_mapping, 2)
    assert monos == [(0, 1), (2, 3), (1, 2)] and g == [1.0, -1.0, 0.5] and mapping == [0, 0, 1]
    assert gidx == [0, 0, 1]
