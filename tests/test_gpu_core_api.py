"""The rest of the `_core` surface the reference front-end calls, on the GPU.

* expectation_value_functional / expectation_value_and_gradient_functional (binder.h:137-146): equal to
  expectation_value[_and_gradient] at the same parameters; pared (pare_threshold 1e-10, PareGraph.cpp)
  equal to unpared, as the reference's tests/test_infinite_cutoff.py:39-108 require; stale after the
  operator is re-weighted; a wrong parameter count raises;
* update_initial_operator (MPOperator.h:193-232): the graph replay is linear in the initial operator, so
  re-weighted replays combine linearly; a term outside the store raises OperatorTermNotFound; after a
  plain propagate the current operator becomes the given one;
* parameter_mapping (rw, per layer or per gate), graph_size, operator_memory_breakdown,
  graph_memory_bytes and __deepcopy__.
"""

import copy

import numpy as np
import pytest

import oracle
from monoprop_b200 import Circuit, MajoranaOperator, MajoranaPropagator, _core
from monoprop_b200 import workloads as W
from oracle import golden

pytestmark = pytest.mark.gpu


def fixture_propagator(name="ref_random_exact", cutoff=4):
    g = golden.load(name)
    wl = golden.fixture_workload(g, name)
    circuit = Circuit.from_dense_arrays(wl.gate_slots, wl.gen_coeffs, wl.param_map, wl.num_modes, wl.params,
                                        wl.initial_state)
    mp = MajoranaPropagator(MajoranaOperator(wl.observable, wl.num_modes), wl.initial_state, cutoff=cutoff)
    mp.build_graph(circuit)
    return wl, mp


def core_hubbard(L=300, lower_atol=1e-5):
    """A _core propagator (the reference's class layout) with the 6x6 Hubbard prefix as a graph."""
    wl = W.hubbard6x6()
    cls = getattr(_core, "MonomialPropagator096")
    obs = {k: complex(v) for k, v in wl.observable.items()}
    p = cls(obs, wl.cutoff, wl.initial_state, lower_atol=lower_atol, cutoff_type="length", logical_num_modes=72)
    P = int(wl.param_map[:L].max()) + 1
    p.build_graph([list(m) for m in wl.gate_slots[:L]], list(map(int, wl.param_map[:L])), list(wl.gen_coeffs[:L]),
                  None, list(wl.params[:P]))
    return wl, p, list(wl.params[:P])


@pytest.mark.parametrize("name", ["ref_random_exact", "ref_rx_rz_ry_rz_exact"])
def test_functionals_match_direct_calls_and_paring_is_exact(name):
    wl, mp = fixture_propagator(name, cutoff=2 * golden.fixture_workload(golden.load(name), name).num_modes)
    theta = np.asarray(wl.params) * 0.9 + 0.03
    ev = mp.expectation_value(theta)
    ev_g, grad = mp.expectation_value_and_gradient(theta)
    for pare in (None, 1e-10):
        f = mp.expval_functional(pare_threshold=pare)
        fg = mp.expval_and_grad_functional(pare_threshold=pare)
        assert abs(f(theta) - ev) <= 1e-12 * max(1.0, abs(ev))
        v, g = fg(theta)
        assert abs(v - ev_g) <= 1e-12 * max(1.0, abs(ev_g))
        assert np.max(np.abs(g - grad)) <= 1e-11 * max(1.0, np.max(np.abs(grad)))
    exact = float(golden.load(name)["exact_energy"])
    assert abs(mp.expval_functional(pare_threshold=1e-10)(wl.params) - exact) <= 1e-12


def test_paring_on_a_truncated_graph():
    """The 6x6 Hubbard prefix (truncation active): pared and unpared replays agree on <O> and gradient at
    shifted parameters, and the plain expectation after a pared functional is unpared again."""
    wl, p, theta = core_hubbard()
    t2 = list(np.asarray(theta) * 1.05 + 0.01)
    ev = p.expectation_value(t2)
    ev1, g1 = p.expectation_value_and_gradient(t2)
    pared = p.expectation_value_functional(1e-10)
    pared_g = p.expectation_value_and_gradient_functional(1e-10)
    assert abs(pared(t2) - ev) <= 1e-13 * max(1.0, abs(ev))
    v, g = pared_g(t2)
    assert abs(v - ev1) <= 1e-13 * max(1.0, abs(ev1))
    assert np.max(np.abs(np.asarray(g) - np.asarray(g1))) <= 1e-11 * max(1.0, np.max(np.abs(g1)))
    # a threshold above every reference-state weight pares everything; a plain call is exact again after
    p.expectation_value_functional(2.0)(t2)
    assert abs(p.expectation_value(t2) - ev) <= 1e-13 * max(1.0, abs(ev))
    coefs = np.asarray(p.contract_partially(t2, False))
    pared(t2)
    assert np.array_equal(np.asarray(p.contract_partially(t2, False)), coefs)


def test_functional_errors_and_staleness():
    wl, p, theta = core_hubbard(L=200)
    f = p.expectation_value_functional()
    with pytest.raises(RuntimeError, match="Invalid functional call"):
        f(theta[:-1])
    f(theta)
    p.update_initial_operator({(): 0.5 + 0j, (0, 1): 0.25j})
    with pytest.raises(RuntimeError, match="MP object has been modified"):
        f(theta)
    p.expectation_value_functional()(theta)  # a new functional is fine


def test_update_initial_operator_is_linear_in_the_replay():
    """Re-weighting the initial operator of a built graph: E(a O1 + b O2) = a E(O1) + b E(O2) over terms
    that are in the store, with the core term carried separately."""
    wl = W.ising100()
    L = 600
    obs = {k: complex(v) for k, v in wl.observable.items()}
    p = _core.MonomialPropagator128(obs, wl.cutoff, [], lower_atol=wl.lower_atol, cutoff_type="support",
                                    logical_num_modes=100, basis="pauli")
    P = int(wl.param_map[:L].max()) + 1
    theta = list(wl.params[:P])
    p.build_graph([list(m) for m in wl.gate_slots[:L]], list(map(int, wl.param_map[:L])), list(wl.gen_coeffs[:L]),
                  None, theta)
    keys = sorted(obs)
    o1 = {k: 0.01 + 0j for k in keys[:50]}
    o2 = {k: 0.01 + 0j for k in keys[50:]}
    t2 = list(np.asarray(theta) * 0.97)
    p.update_initial_operator(o1)
    e1 = p.expectation_value(t2)
    p.update_initial_operator(o2)
    e2 = p.expectation_value(t2)
    both = {**{k: 2.0 * v for k, v in o1.items()}, **{k: -0.5 * v for k, v in o2.items()}, (): 0.125 + 0j}
    p.update_initial_operator(both)
    e12 = p.expectation_value(t2)
    assert abs(e12 - (0.125 + 2.0 * e1 - 0.5 * e2)) <= 1e-12
    # X on 12 qubits: above the weight cutoff of 10, so never stored
    absent = tuple(range(0, 24, 2))
    with pytest.raises(RuntimeError, match=r"Operator term \[0, 2, 4, .*, 22\] not found in the operator"):
        p.update_initial_operator({absent: 1.0 + 0j})


def test_update_initial_operator_after_propagate():
    """Without a graph the current (evolved) operator becomes the given one: <0|O|0> is then the core plus
    the Z-only terms' coefficients (reference state |0...0>)."""
    wl = W.line20()
    obs = {k: complex(v) for k, v in wl.observable.items()}
    p = _core.MonomialPropagator032(obs, wl.cutoff, [], lower_atol=wl.lower_atol, cutoff_type="support",
                                    logical_num_modes=20, basis="pauli")
    p.propagate([list(m) for m in wl.gate_slots], list(map(int, wl.param_map)), list(wl.gen_coeffs),
                list(wl.params), None)
    terms = p.evolved_operator([], 0.0)
    zonly = [k for k in terms if len(k) and len(k) % 2 == 0
             and all(k[i] % 2 == 0 and k[i + 1] == k[i] + 1 for i in range(0, len(k), 2))][:5]
    other = [k for k in terms if len(k) and k not in zonly][:5]
    new = {**{k: 0.1 * (i + 1) + 0j for i, k in enumerate(zonly)}, **{k: 7.0 + 0j for k in other}, (): 0.5 + 0j}
    p.update_initial_operator(new)
    assert abs(p.expectation_value([]) - (0.5 + sum(0.1 * (i + 1) for i in range(len(zonly))))) <= 1e-12
    got = p.evolved_operator([], 1e-14)
    assert {k for k in got if len(k)} == set(zonly) | set(other)


def test_parameter_mapping_per_layer_and_per_gate():
    """Relabelling the graph's parameters: with theta2 permuted accordingly, the replay is unchanged."""
    wl, p, theta = core_hubbard(L=200)
    m = p.parameter_mapping
    assert m == list(map(int, wl.param_map[:200]))
    ev = p.expectation_value(theta)
    n = len(theta)
    perm = np.random.default_rng(3).permutation(n)  # new index of old parameter j is perm[j]
    p.parameter_mapping = [int(perm[j]) for j in m]
    theta2 = np.zeros(n)
    theta2[perm] = theta
    assert abs(p.expectation_value(list(theta2)) - ev) <= 1e-13 * max(1.0, abs(ev))
    assert p.n_gates() == 200  # no gate_indices: one gate per layer
    p.parameter_mapping = m  # per layer == per gate here; back to the original
    assert abs(p.expectation_value(theta) - ev) <= 1e-13 * max(1.0, abs(ev))
    with pytest.raises(RuntimeError, match="parameter_mapping has 3 entries"):
        p.parameter_mapping = [0, 1, 2]


def test_graph_size_memory_and_deepcopy():
    wl, p, theta = core_hubbard(L=300)
    cos_only, pairs = p.graph_size()
    # the anticommuting terms of every gate are either cos-only or pair members (the oracle's per-gate counts)
    wl3 = W.hubbard6x6()
    import dataclasses

    wl3 = dataclasses.replace(wl3, gate_slots=wl3.gate_slots[:300], gen_coeffs=wl3.gen_coeffs[:300],
                              param_map=wl3.param_map[:300], params=wl3.params[:len(theta)])
    counts = oracle.run_port(wl3).counts.astype(np.int64)
    assert cos_only + 2 * pairs - int(counts[:, 3].sum()) == int(counts[:, 1].sum())
    b = p.operator_memory_breakdown()
    parts = ("operator_terms_bytes", "op_coeffs_bytes", "state_coeffs_bytes", "indexing_bytes",
             "init_operator_bytes", "initial_state_bytes", "inverted_index_bytes")
    assert b["total_bytes"] == sum(b[k] for k in parts) == p.operator_memory_bytes()
    assert b["operator_terms_bytes"] >= 24 * p.size() and p.graph_memory_bytes() > 0
    q = copy.deepcopy(p)
    t2 = list(np.asarray(theta) * 0.9)
    assert q.expectation_value(t2) == p.expectation_value(t2)
    assert q.graph_size() == p.graph_size() and q.size() == p.size()
    q.update_initial_operator({(0, 1): 1.0j})
    assert q.expectation_value(t2) != p.expectation_value(t2)  # the copy is independent
    assert abs(p.expectation_value(t2) - q.expectation_value(t2)) > 0.0
    p.contract_partially(t2, True)
    assert p.graph_memory_bytes() == 0 and q.graph_layers() == 300
