"""Graphs, functionals and gradients in the Schrodinger picture on the GPU.

The reference replays a Schrodinger graph from the dense reference state: every stored monomial starts at
its reference-state score, appended ones included (MPOperator.h:169-181), and each recorded pair rotates
both ways, the appended partner cos-scaled like every anticommuting term below the post-insert count
(Evolution.cpp:471-511, Engine.h:628-633). <O> dots the observable into the evolved state, so the adjoint
starts from the observable, and paring keeps the observable's terms above the threshold
(MonomialPropagator.inl:950-964). Checked against the reference's own graphs
(``tests/golden/graph_*_s*.npz``: its replay at the build parameters and at shifted ones, its gradient
there, and central finite differences of its replay), as the reference's own tests build them
(tests/test_infinite_cutoff.py:72-105: cutoff 4, schrodinger_cutoff 6; tests/test_only_rotate_k.py:32:
cutoff 6, schrodinger_cutoff 8 with only_rotate_len_k).
"""

import dataclasses

import numpy as np
import pytest

from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from oracle import golden

pytestmark = pytest.mark.gpu

#: graph fixture -> (base problem, cutoff or None for the workload's own, schrodinger_cutoff, only_rotate_len_k)
CASES = {
    "ref_lih_fermionic_spin_exact_c4_s6": ("ref_lih_fermionic_spin_exact", 4, 6, None),
    "ref_lih_fermionic_spin_exact_c6_s8_k4": ("ref_lih_fermionic_spin_exact", 6, 8, 4),
    "line20_L200_s4": ("line20", None, 4, None),
}


def _case(name):
    """(workload, layers) of graph fixture ``name``: the reference's fermionic test problem with its test's
    cutoffs, or the 20-qubit line circuit (200 layers)."""
    base, cutoff, sc, k = CASES[name]
    if base == "line20":
        wl = W.line20()
        L = 200
    else:
        wl = golden.fixture_workload(golden.load(base), base)
        wl = dataclasses.replace(wl, cutoff=cutoff)
        L = wl.n_layers
    extra = {**wl.extra, "schrodinger_cutoff": sc}
    if k is not None:
        extra["only_rotate_len_k"] = k
    return dataclasses.replace(wl, extra=extra), L


def _propagator(wl):
    from monoprop_b200.propagators import dispatch

    ops = {tuple(key): complex(v) for key, v in wl.observable.items()}
    return dispatch(wl.num_modes)(initial_operator=ops, cutoff=wl.cutoff, initial_state=list(wl.initial_state),
                                  cutoff_type=wl.cutoff_type, lower_atol=wl.lower_atol,
                                  schrodinger_cutoff=int(wl.extra["schrodinger_cutoff"]),
                                  logical_num_modes=wl.num_modes, basis=wl.basis)


def _built(name):
    wl, L = _case(name)
    p = _propagator(wl)
    P = int(wl.param_map[:L].max()) + 1
    p.build_graph([list(m) for m in wl.gate_slots[:L]], list(map(int, wl.param_map[:L])), list(wl.gen_coeffs[:L]),
                  None, list(wl.params[:P]), wl.extra.get("only_rotate_len_k"))
    return wl, L, P, p


@pytest.mark.parametrize("name", sorted(CASES))
def test_schrodinger_graph_matches_reference(name):
    """<O> of the replay at the build parameters and at shifted ones, and the gradient there, against the
    reference's graph; the gradient also against central finite differences of the reference's replay
    (per angle, 1e-7 relative + 1e-9)."""
    g = golden.load("graph_" + name)
    wl, L, P, p = _built(name)
    assert p.schrodinger
    ev0 = p.expectation_value(list(wl.params[:P]))
    assert abs(ev0 - float(g["expectation_build"])) <= 1e-10 * max(1.0, abs(float(g["expectation_build"])))
    ev, grad = p.expectation_value_and_gradient(list(g["params"]))
    grad = np.asarray(grad)
    assert abs(ev - float(g["expectation"])) <= 1e-10 * max(1.0, abs(float(g["expectation"])))
    assert np.max(np.abs(grad - g["grad"])) <= 1e-9 * max(1.0, np.max(np.abs(g["grad"])))
    fd = g["fd"]
    assert np.all(np.abs(grad[g["fd_idx"]] - fd) <= 1e-7 * np.abs(fd) + 1e-9)
    assert p.size() == int(g["terms"])


@pytest.mark.parametrize("name", ["ref_lih_fermionic_spin_exact_c4_s6", "line20_L200_s4"])
def test_schrodinger_pared_functional_equals_unpared(name):
    """Paring against the observable at 1e-10 drops no term that reaches <O> (the reference's own check,
    tests/test_infinite_cutoff.py:38-67): the pared functionals give the unpared values."""
    wl, L, P, p = _built(name)
    theta = list(wl.params[:P] + 0.05 * np.random.default_rng(3).standard_normal(P))
    full = p.expectation_value_and_gradient_functional(None)(theta)
    pared_ev = p.expectation_value_functional(1e-10)(theta)
    pared = p.expectation_value_and_gradient_functional(1e-10)(theta)
    assert abs(pared_ev - full[0]) <= 1e-12 * max(1.0, abs(full[0]))
    assert abs(pared[0] - full[0]) <= 1e-12 * max(1.0, abs(full[0]))
    assert np.max(np.abs(np.asarray(pared[1]) - np.asarray(full[1]))) <= 1e-11 * max(1.0, np.max(np.abs(full[1])))


@pytest.mark.parametrize("name", sorted(golden.SCHRODINGER))
def test_schrodinger_graph_replay_is_the_propagation(name):
    """At its build parameters the replayed state is the propagated state: the replay of the graph from the
    dense reference state gives the reference's Schrodinger propagation (tests/golden/<name>.npz: key set
    bit-exact, coefficient sums and <O> within 1e-10)."""
    wl, L = golden.schrodinger_workload(name)
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    eng.graph_build(circ)
    ev = eng.graph_expectation(circ)
    keys, coefs = eng.export()
    circ.close()
    eng.close()
    golden.check_against(golden.load(name), keys, coefs, ev)


@pytest.mark.parametrize("pair_log", [-1, 0])
def test_schrodinger_adjoint_equals_graph_gradient(pair_log):
    """The engine's adjoint in the Schrodinger picture (forward pair log replayed by the frozen kernels, or,
    without the log, the streaming kernels in replay mode redoing each append from its score) gives the
    graph's gradient at the same angles, per circuit layer."""
    wl, L = _case("line20_L200_s4")
    eng = _native.engine_for(wl)
    eng.set_pair_log(pair_log)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    ev = eng.adjoint_forward(circ, 48)
    ga = eng.adjoint_backward(circ)
    eng.graph_build(circ)
    ev_g, gg = eng.graph_gradient(circ)
    circ.close()
    eng.close()
    assert abs(ev - ev_g) <= 1e-13 * max(1.0, abs(ev))
    assert np.max(np.abs(ga - gg)) <= 1e-11 * max(1.0, np.max(np.abs(gg)))
    assert np.count_nonzero(np.abs(gg) > 1e-9) > 10
