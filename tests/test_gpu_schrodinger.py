"""The Schrodinger picture on the GPU (schrodinger_cutoff, MonomialPropagator.inl:146-179,595-620).

The store starts as every fully paired monomial up to the cutoff holding its reference-state score, the
gates run first to last at the negated angle, an appended partner starts from its own score
(FusedApply.h:39-83), and <O> is the observable dotted into the evolved state (MPFunctions.cpp:196-205).
Checked against the unmodified reference's fixtures (tests/golden/*_s4.npz: keys bit-exact,
coefficients and <O> within 1e-10 relative) and against the oracle on random circuits with truncation
active, through the shared-memory path (small stores) and the streaming kernels alike.
"""

import dataclasses

import numpy as np
import pytest

import oracle
from monoprop_b200 import _core, _native
from monoprop_b200.encoding import canonical_order
from oracle import golden
from oracle.golden import random_workload

pytestmark = pytest.mark.gpu


def run_engine(wl, n_layers=None, **kw):
    eng = _native.engine_for(wl, **kw)
    L = wl.n_layers if n_layers is None else n_layers
    try:
        eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
        keys, coefs = eng.export()
        ev = eng.expectation()
    finally:
        eng.close()
    return keys, coefs, ev


@pytest.mark.parametrize("name", sorted(golden.SCHRODINGER))
def test_schrodinger_matches_reference_golden(name):
    wl, L = golden.schrodinger_workload(name)
    keys, coefs, ev = run_engine(wl, L)
    golden.check_against(golden.load(name), keys, coefs, ev)


@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
def test_schrodinger_matches_oracle_random(seed, basis):
    base = random_workload(seed, basis)
    wl = dataclasses.replace(base, extra={**base.extra, "schrodinger_cutoff": base.cutoff + 1})
    ref = oracle.run_port(wl)
    keys, coefs, ev = run_engine(wl)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert keys.shape == ref.keys.shape and np.array_equal(keys[ia], ref.keys[ib])
    a, b = coefs[ia], ref.coefs[ib]
    assert np.all(np.abs(a - b) <= 1e-10 * np.maximum(np.abs(a), np.abs(b)) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_schrodinger_streaming_from_a_tiny_capacity():
    """Growth from a tiny store (streaming kernels from the first gate on) gives the same state."""
    wl, L = golden.schrodinger_workload("line20_L100_s4")
    k1, c1, e1 = run_engine(wl, L)
    k2, c2, e2 = run_engine(wl, L, capacity_hint=1)
    i1, i2 = canonical_order(k1), canonical_order(k2)
    assert np.array_equal(k1[i1], k2[i2]) and np.array_equal(c1[i1], c2[i2])
    assert abs(e1 - e2) <= 1e-14 * max(1.0, abs(e1))


def test_core_schrodinger_surface():
    """The _core class with schrodinger_cutoff: the reference's property, <O> over the evolved state, the
    observable re-weighted by update_initial_operator, no core term in evolved_operator, and a graph built
    in this picture (its replays are checked in test_gpu_schrodinger_graph.py)."""
    wl, L = golden.schrodinger_workload("hubbard6x6_L200_s4")
    g = golden.load("hubbard6x6_L200_s4")
    obs = {k: complex(v) for k, v in wl.observable.items()}
    p = _core.MonomialPropagator096(obs, wl.cutoff, wl.initial_state, schrodinger_cutoff=4, lower_atol=wl.lower_atol,
                                    cutoff_type="length", logical_num_modes=72)
    assert p.schrodinger is True
    P = int(wl.param_map[:L].max()) + 1
    p.propagate([list(m) for m in wl.gate_slots[:L]], list(map(int, wl.param_map[:L])), list(wl.gen_coeffs[:L]),
                list(wl.params[:P]), None)
    ev = p.expectation_value([])
    assert abs(ev - float(g["expectation"])) <= 1e-10 * max(1.0, abs(float(g["expectation"])))
    # the state's identity monomial (score 1, never rotated) is a stored term; the observable's core term is
    # not added in this picture (binder.h:200-221)
    assert p.evolved_operator([], 0.0)[()] == 1.0
    # <O> is linear in the observable: doubling its non-core part doubles <O> - core
    p.update_initial_operator({(): 0.5 + 0j, (0, 1): 1.0j})
    assert abs((p.expectation_value([]) - 0.5) - 2 * (ev - 0.5)) <= 1e-12
    P10 = int(wl.param_map[:10].max()) + 1
    p.build_graph([list(m) for m in wl.gate_slots[:10]], list(map(int, wl.param_map[:10])),
                  list(wl.gen_coeffs[:10]), None, list(wl.params[:P10]))
    assert p.graph_layers() == 10
    ev_g, grad = p.expectation_value_and_gradient(list(wl.params[:P10]))
    assert np.isfinite(ev_g) and len(grad) == P10
