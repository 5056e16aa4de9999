"""The front-end (PauliPropagator / MajoranaPropagator over the _core module) on the GPU.

Mirrors the reference's own Python tests for the propagate path: the analytic truncation cases of
tests/test_coeff_trunc.py:59-96 and :142-227, the exact energies of tests/test_infinite_cutoff.py
(from the golden copies of its fixtures), and from_circuit on a qubit circuit against the oracle.
"""

import numpy as np
import pytest

import oracle
from monoprop_b200 import Circuit, ExpGate, MajoranaOperator, MajoranaPropagator, Pauli, PauliOperator, PauliPropagator
from monoprop_b200 import workloads as W
from oracle import golden

pytestmark = pytest.mark.gpu


def check_dicts(d1, d2):
    d1 = d1.terms if isinstance(d1, MajoranaOperator) else d1
    assert len(d1) == len(d2), (d1, d2)
    for k in d1:
        assert k in d2, k
        assert np.isclose(d1[k], d2[k]), (k, d1[k], d2[k])


@pytest.mark.parametrize("cutoff, upper_atol, lower_atol, kept", [
    (4, None, None, True), (1, 0.49, None, True), (1, 1.0, None, False), (4, None, 0.9, False),
    (10, None, 0.1, True)])
def test_coeff_trunc(cutoff, upper_atol, lower_atol, kept):
    op = MajoranaOperator({(0, 1): 1.0j}, num_modes=5)
    circuit = Circuit.from_dense_arrays(initial_state=[], majoranas=[(1, 2, 3, 4)], parameters=[np.pi / 6],
                                        gen_coeffs=[1.0], param_inds=[0], system_size=5)
    cos_pi6, sin_pi6 = 0.5, -0.8660254037844386
    expected = {(0, 1): 1j * cos_pi6, (0, 2, 3, 4): sin_pi6} if kept else {(0, 1): 1j * cos_pi6}
    mp = MajoranaPropagator(op, [], cutoff=cutoff, upper_atol=upper_atol, lower_atol=lower_atol)
    mp.propagate(circuit)
    check_dicts(mp.evolved_operator(), expected)


@pytest.mark.parametrize("upper_atol, lower_atol", [(None, None), (None, 1e-6), (None, 1e-10), (1e-4, None),
                                                    (1e-4, 1e-6), (1e-4, 1e-10), (1e-10, None), (1e-10, 1e-10)])
def test_evolution_small_coeffs(upper_atol, lower_atol):
    p = 1e-5
    init = {(0, 1): 1.0j, (0, 2): 1e-7j}
    circuit = Circuit.from_dense_arrays(initial_state=[], majoranas=[(1, 2)], parameters=[p], gen_coeffs=[1.0],
                                        param_inds=[0], system_size=2)
    final = {(0, 1): init[(0, 1)] * np.cos(2 * p) - init[(0, 2)] * np.sin(2 * p),
             (0, 2): init[(0, 2)] * np.cos(2 * p) + init[(0, 1)] * np.sin(2 * p)}
    mp = MajoranaPropagator(MajoranaOperator(init, num_modes=2), [], cutoff=4, upper_atol=upper_atol,
                            lower_atol=lower_atol)
    mp.propagate(circuit)
    assert mp.size() == 2
    check_dicts(mp.evolved_operator(), final)


@pytest.mark.parametrize("name", [c for c in golden.REF_CASES if not c.endswith("atol1e-10")])
def test_infinite_cutoff_exact_energy(name):
    g = golden.load(name)
    wl = golden.fixture_workload(g, name)
    circuit = Circuit.from_dense_arrays(wl.gate_slots, wl.gen_coeffs, wl.param_map, wl.num_modes, wl.params,
                                        wl.initial_state)
    op = MajoranaOperator(wl.observable, wl.num_modes)
    mp = MajoranaPropagator.from_circuit(circuit, op, cutoff=2 * wl.num_modes)
    assert np.isclose(mp.expectation_value(), float(g["exact_energy"]), atol=1e-12)
    value, grad = mp.expectation_value_and_gradient()
    assert np.isclose(value, float(g["exact_energy"]), atol=1e-12) and len(grad) == 0


def test_pauli_from_circuit_matches_oracle():
    wl = W.line20()
    n = 20
    gates = []
    for slots in wl.gate_slots:
        if len(slots) == 4:  # RZZ(t) = exp(+i t (-1/2) Z Z)
            q = sorted({s // 2 for s in slots})
            gates.append(ExpGate(PauliOperator({Pauli("ZZ", q): -0.5}, n)))
        else:  # RX(t) = exp(+i t (-1/2) X)
            gates.append(ExpGate(PauliOperator({Pauli("X", slots[0] // 2): -0.5}, n)))
    circuit = Circuit(gates, n, wl.params, [])
    obs = PauliOperator({Pauli("Z", 10): 1.0}, n)
    pp = PauliPropagator.from_circuit(circuit, obs, cutoff=8, lower_atol=1e-4)
    ref = oracle.run_port(wl)
    assert pp.size() == ref.keys.shape[0]
    assert abs(pp.expectation_value() - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))
    evolved = pp.evolved_operator(atol=0.0)
    # atol = 0 keeps every stored term plus the (zero) identity core term, as the reference does
    assert len(evolved.terms) == pp.size() + 1 and evolved.terms[Pauli("")] == 0.0


@pytest.mark.parametrize("name", ["ref_rx_rz_ry_rz_exact", "ref_random_exact"])
def test_graph_exact_energy_and_gradient(name):
    """build_graph + replayed functionals (tests/test_infinite_cutoff.py:39-108 of the reference): the
    exact energy and gradient at infinite cutoff, and central finite differences at cutoff 4."""
    g = golden.load(name)
    wl = golden.fixture_workload(g, name)
    circuit = Circuit.from_dense_arrays(wl.gate_slots, wl.gen_coeffs, wl.param_map, wl.num_modes, wl.params,
                                        wl.initial_state)
    op = MajoranaOperator(wl.observable, wl.num_modes)
    mp = MajoranaPropagator(op, wl.initial_state, cutoff=2 * wl.num_modes)
    mp.build_graph(circuit)
    assert np.isclose(mp.expval_functional()(wl.params), float(g["exact_energy"]), atol=1e-12)
    ev, grad = mp.expval_and_grad(wl.params)
    assert np.isclose(ev, float(g["exact_energy"]), atol=1e-12)
    assert np.allclose(grad, g["exact_gradient"], atol=1e-10)

    prng = np.random.default_rng(0)
    mp4 = MajoranaPropagator(op, wl.initial_state, cutoff=4)
    mp4.build_graph(circuit)
    fn = mp4.expval_functional()
    xk = prng.random(size=len(wl.params))
    eps = 1e-6
    fd = np.zeros_like(xk)
    for i in range(len(xk)):
        old = xk[i]
        xk[i] = old + eps
        ep = fn(xk)
        xk[i] = old - eps
        em = fn(xk)
        fd[i] = (ep - em) / (2 * eps)
        xk[i] = old
    assert np.allclose(mp4.grad(xk), fd, atol=1e-6)


def test_contract_partially():
    """contract_partially (monomial_propagator.py:478-510): the graph replayed at new parameters as raw
    coefficients; inplace consumes the graph, after which a plain propagate is allowed."""
    g = golden.load("ref_random_exact")
    wl = golden.fixture_workload(g, "ref_random_exact")
    circuit = Circuit.from_dense_arrays(wl.gate_slots, wl.gen_coeffs, wl.param_map, wl.num_modes, wl.params,
                                        wl.initial_state)
    op = MajoranaOperator(wl.observable, wl.num_modes)
    mp = MajoranaPropagator(op, wl.initial_state, cutoff=4)
    mp.build_graph(circuit)
    theta = np.asarray(wl.params) * 0.7 + 0.05
    coefs = mp.contract_partially(theta, inplace=False)
    assert coefs.shape == (mp.size(),) and mp.graph_layers() > 0
    ev = mp.expectation_value(theta)
    evolved = mp.evolved_operator(theta, atol=0.0)
    assert np.allclose(np.sort(np.abs(coefs)), np.sort([abs(c) for k, c in evolved.terms.items() if len(k)]),
                       atol=1e-12)
    again = mp.contract_partially(theta, inplace=True)
    assert np.array_equal(np.sort(again), np.sort(coefs))
    assert mp.graph_layers() == 0
    assert abs(mp.expectation_value() - ev) <= 1e-12 * max(1.0, abs(ev))
    mp.propagate(circuit)  # no graph left: a plain propagation continues from the contracted operator
