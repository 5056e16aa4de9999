"""Edge cases of the engine on the GPU, against the oracle where there is a result to compare.

Empty observable, empty circuit, identity (empty-generator) layers, an observable that is only a core
term, wide keys (W = 7: 224 fermionic modes, 448 Majorana slots) and the failure paths that need no device fault: a capacity beyond
the 32-bit term index, invalid arguments, a backward pass without its forward pass.
"""

import numpy as np
import pytest

import oracle
from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from monoprop_b200.encoding import canonical_order
from oracle.golden import random_workload

pytestmark = pytest.mark.gpu


def same(wl):
    ref = oracle.run_port(wl)
    eng = _native.engine_for(wl)
    eng.propagate(wl.gen_words(), wl.angles())
    keys, coefs = eng.export()
    ev = eng.expectation()
    eng.close()
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert np.all(np.abs(coefs[ia] - ref.coefs[ib]) <= 1e-10 * np.maximum(np.abs(coefs[ia]), 1e-300) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_empty_circuit_and_identity_layers():
    wl = W.line20(layers=2)
    same(W.Workload("empty", wl.basis, wl.num_modes, [], np.zeros(0), np.zeros(0, np.int64), np.zeros(0),
                    wl.observable, [], wl.cutoff, wl.cutoff_type, wl.lower_atol))
    slots = list(wl.gate_slots)
    slots[3] = ()
    slots[10] = ()
    same(W.Workload("identity", wl.basis, wl.num_modes, slots, wl.gen_coeffs, wl.param_map, wl.params,
                    wl.observable, [], wl.cutoff, wl.cutoff_type, wl.lower_atol))


def test_core_only_observable():
    wl = W.line20(layers=1)
    eng = _native.Engine(basis="pauli", cutoff_type="support", cutoff=8, num_modes=20,
                         keys=np.zeros((0, 1), np.uint64), coefs=np.zeros(0), core=0.75,
                         state_mask=np.zeros(1, np.uint64), lower_atol=1e-4)
    eng.propagate(wl.gen_words(), wl.angles())
    assert eng.size() == 0 and eng.expectation() == 0.75
    eng.close()


@pytest.mark.parametrize("seed", range(4))
def test_wide_keys_224_modes(seed):
    base = random_workload(seed, "majorana")
    rng = np.random.default_rng(seed)
    n = 224  # 448 Majorana slots -> W = 7
    shift = lambda m: tuple(sorted((s * 37 + 5) % (2 * n) for s in m))  # noqa: E731
    obs = {shift(k): v for k, v in base.observable.items()}
    slots = [shift(m) for m in base.gate_slots]
    state = sorted(set(int(x) for x in rng.integers(0, n, size=6)))
    wl = W.Workload(f"wide_{seed}", "majorana", n, slots, base.gen_coeffs, base.param_map, base.params, obs, state,
                    base.cutoff, base.cutoff_type, base.lower_atol, base.upper_atol)
    assert wl.words == 7
    same(wl)


def test_capacity_beyond_term_index_is_rejected():
    wl = W.line20(layers=1)
    with pytest.raises(_native.MpxError) as ei:
        _native.engine_for(wl, capacity_hint=1 << 33)
    assert ei.value.status == 4  # MPX_ERR_CAPACITY


def test_invalid_arguments_and_state_errors():
    wl = W.line20(layers=1)
    with pytest.raises(_native.MpxInvalid):
        _native.Engine(basis="pauli", cutoff_type="length", cutoff=8, num_modes=20,
                       keys=np.zeros((1, 1), np.uint64), coefs=np.ones(1), core=0.0, state_mask=np.zeros(1, np.uint64))
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words(), wl.angles())
    with pytest.raises(_native.MpxError) as ei:
        eng.adjoint_backward(circ)  # no forward pass recorded
    assert ei.value.status == 5
    with pytest.raises(_native.MpxError) as ei:
        eng.graph_expectation(circ)  # no graph built
    assert ei.value.status == 5
    with pytest.raises(ValueError):
        eng.propagate(wl.gen_words(), wl.angles()[:-1])
    circ.close()
    eng.close()
