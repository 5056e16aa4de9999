"""only_rotate_len_k on the GPU: terms with more than k set slots take no part in a gate.

The reference (Scan.h:146-157,376-391, FusedApply.h:46-52) skips them in the cos set and in the emit
pass, and a partner outside the set receives its sine term unscaled. Checked against the golden fixtures
generated by the reference with only_rotate_len_k, against the oracle on seeded random circuits (Pauli
and Majorana), and through the _core module (validation message); graphs and gradients built with only_rotate_len_k
against the reference's own graph and its finite differences.
"""

import dataclasses

import numpy as np
import pytest

import oracle
from monoprop_b200 import _native
from monoprop_b200.encoding import canonical_order
from oracle import golden
from oracle.golden import random_workload

pytestmark = pytest.mark.gpu


def run(wl, n_layers=None):
    k = wl.extra.get("only_rotate_len_k")
    eng = _native.engine_for(wl)
    try:
        eng.set_only_rotate_len_k(k)
        L = wl.n_layers if n_layers is None else n_layers
        eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
        keys, coefs = eng.export()
        return keys, coefs, eng.expectation()
    finally:
        eng.close()


@pytest.mark.parametrize("name", sorted(golden.LEN_K))
def test_len_k_matches_reference_golden(name):
    wl, L = golden.len_k_workload(name)
    keys, coefs, ev = run(wl, L)
    golden.check_against(golden.load(name), keys, coefs, ev)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
@pytest.mark.parametrize("k", [2, 4, 6])
def test_len_k_matches_oracle(seed, basis, k):
    base = random_workload(seed, basis)
    wl = dataclasses.replace(base, extra={**base.extra, "only_rotate_len_k": k})
    ref = oracle.run_port(wl)
    keys, coefs, ev = run(wl)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert np.all(np.abs(coefs[ia] - ref.coefs[ib]) <= 1e-10 * np.maximum(np.abs(ref.coefs[ib]), 1e-300) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_len_k_cleared_and_guards():
    wl, _ = golden.len_k_workload("line20_k6")
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words(), wl.angles())
    eng.set_only_rotate_len_k(6)
    with pytest.raises(_native.MpxInvalid):
        eng.set_only_rotate_len_k(2 * wl.num_modes + 1)
    eng.set_only_rotate_len_k(None)  # cleared: a plain propagation again
    eng.propagate_circuit(circ)
    plain = oracle.run_port(dataclasses.replace(wl, extra={}))
    assert eng.size() == plain.keys.shape[0]
    circ.close()
    eng.close()


def test_core_propagate_only_rotate_len_k():
    from monoprop_b200 import _core
    from monoprop_b200.propagators import dispatch

    wl, _ = golden.len_k_workload("line20_k6")
    ops = {tuple(k): complex(v) for k, v in wl.observable.items()}
    p = dispatch(wl.num_modes)(initial_operator=ops, cutoff=wl.cutoff, initial_state=[], cutoff_type="support",
                               lower_atol=wl.lower_atol, logical_num_modes=wl.num_modes, basis="pauli")
    monos = [list(m) for m in wl.gate_slots]
    with pytest.raises(RuntimeError, match="only_rotate_len_k=0 is out of range"):
        p.propagate(monos, list(wl.param_map), list(wl.gen_coeffs), list(wl.params), only_rotate_len_k=0)
    p.propagate(monos, list(wl.param_map), list(wl.gen_coeffs), list(wl.params), only_rotate_len_k=6)
    g = golden.load("line20_k6")
    assert p.size() == int(g["n"])
    assert abs(p.expectation_value([]) - float(g["expectation"])) <= 1e-10
    assert _core.MAX_NUM_MODES >= wl.num_modes


LEN_K_GRAPHS = {"hubbard6x6_L300_k4": ("hubbard6x6", 300, 4), "ising100_L600_k6": ("ising100", 600, 6)}


def _core_graph(name):
    """A _core propagator (the reference's class layout) holding the graph of LEN_K_GRAPHS[name], built with
    only_rotate_len_k at the workload's parameters."""
    from monoprop_b200 import workloads as W
    from monoprop_b200.propagators import dispatch

    base, L, k = LEN_K_GRAPHS[name]
    wl = W.BY_NAME[base]()
    ops = {tuple(key): complex(v) for key, v in wl.observable.items()}
    p = dispatch(wl.num_modes)(initial_operator=ops, cutoff=wl.cutoff, initial_state=list(wl.initial_state),
                               cutoff_type=wl.cutoff_type, lower_atol=wl.lower_atol, logical_num_modes=wl.num_modes,
                               basis=wl.basis)
    P = int(wl.param_map[:L].max()) + 1
    p.build_graph([list(m) for m in wl.gate_slots[:L]], list(map(int, wl.param_map[:L])), list(wl.gen_coeffs[:L]),
                  None, list(wl.params[:P]), k)
    return wl, L, k, P, p


@pytest.mark.parametrize("name", sorted(LEN_K_GRAPHS))
def test_len_k_graph_matches_reference(name):
    """build_graph(..., only_rotate_len_k=k) (binder.h:102-110): the replay at the build parameters, and
    <O> and the gradient at shifted parameters, against the reference's own graph (tests/golden/graph_*_k*.npz),
    plus per-angle central finite differences of the reference's replay (1e-7 relative + 1e-9)."""
    g = golden.load("graph_" + name)
    wl, L, k, P, p = _core_graph(name)
    ev0 = p.expectation_value(list(wl.params[:P]))
    assert abs(ev0 - float(g["expectation_build"])) <= 1e-10 * max(1.0, abs(float(g["expectation_build"])))
    ev, grad = p.expectation_value_and_gradient(list(g["params"]))
    grad = np.asarray(grad)
    assert abs(ev - float(g["expectation"])) <= 1e-10 * max(1.0, abs(float(g["expectation"])))
    assert np.max(np.abs(grad - g["grad"])) <= 1e-9 * max(1.0, np.max(np.abs(g["grad"])))
    fd = g["fd"]
    assert np.all(np.abs(grad[g["fd_idx"]] - fd) <= 1e-7 * np.abs(fd) + 1e-9)


def test_len_k_graph_replay_matches_reference_replay():
    """At its build parameters the replayed graph is the reference's replay (graph_replay_hubbard6x6_L400_k4.npz:
    keys bit-exact, every coefficient within 1e-10). The reference recomputes each layer's cos set with no
    length filter (MonomialPropagator.inl:872-895), so its replay scales the terms outside the
    only_rotate_len_k set and departs from its own propagation there (hubbard6x6_L400_k4.npz), while <O>
    agrees with the propagation."""
    from monoprop_b200 import workloads as W

    wl = W.hubbard6x6()
    wl = dataclasses.replace(wl, extra={**wl.extra, "only_rotate_len_k": 4})
    L = 400
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    eng.set_only_rotate_len_k(4)
    eng.graph_build(circ)
    eng.set_only_rotate_len_k(None)
    ev = eng.graph_expectation(circ)
    keys, coefs = eng.export()
    circ.close()
    eng.close()
    golden.check_against(golden.load("graph_replay_hubbard6x6_L400_k4"), keys, coefs, ev)
    assert abs(ev - float(golden.load("hubbard6x6_L400_k4")["expectation"])) <= 1e-10


@pytest.mark.parametrize("pair_log", [-1, 0])
def test_len_k_adjoint_equals_graph_gradient(pair_log):
    """The engine's adjoint with only_rotate_len_k (forward pair log replayed by the frozen kernels, or,
    without the log, the streaming kernels in replay mode) gives the graph's gradient at the same angles."""
    from monoprop_b200 import workloads as W

    wl = W.hubbard6x6()
    L, k = 300, 4
    eng = _native.engine_for(wl)
    eng.set_pair_log(pair_log)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    eng.set_only_rotate_len_k(k)
    ev = eng.adjoint_forward(circ, 64)
    eng.set_only_rotate_len_k(None)  # the backward pass keeps the forward pass's k
    ga = eng.adjoint_backward(circ)
    eng.set_only_rotate_len_k(k)
    eng.graph_build(circ)
    eng.set_only_rotate_len_k(None)
    ev_g, gg = eng.graph_gradient(circ)
    circ.close()
    eng.close()
    assert abs(ev - ev_g) <= 1e-13 * max(1.0, abs(ev))
    assert np.max(np.abs(ga - gg)) <= 1e-11 * max(1.0, np.max(np.abs(gg)))
