"""only_rotate_len_k on the GPU: terms with more than k set slots take no part in a gate.

The reference (Scan.h:146-157,376-391, FusedApply.h:46-52) skips them in the cos set and in the emit
pass, and a partner outside the set receives its sine term unscaled. Checked against the golden fixtures
generated by the reference with only_rotate_len_k, against the oracle on seeded random circuits (Pauli
and Majorana), and through the _core module (validation message, gradient/graph rejection).
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
        eng.adjoint_forward(circ)
    with pytest.raises(_native.MpxInvalid):
        eng.graph_build(circ)
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
