"""basis_change on the GPU (Majorana): the structural cutoff of every emitted partner is judged on its
image XOR_{slot s in P} row_s (MonomialPropagatorCommon.h:44-62, change_basis MajoranaAlgebra.h:179-189).

Checked against golden fixtures from the reference, against the oracle on seeded random circuits with
three kinds of rows, through the _core module (constructor, property, the reference's messages), and
for the adjoint gradient (the replayed emit decisions use the same image) against finite differences.
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
    eng = _native.engine_for(wl)  # applies wl.extra["basis_change"]
    try:
        L = wl.n_layers if n_layers is None else n_layers
        eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
        keys, coefs = eng.export()
        return keys, coefs, eng.expectation()
    finally:
        eng.close()


@pytest.mark.parametrize("name", sorted(golden.BASIS_CHANGE))
def test_basis_change_matches_reference_golden(name):
    wl, L = golden.basis_change_workload(name)
    keys, coefs, ev = run(wl, L)
    golden.check_against(golden.load(name), keys, coefs, ev)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("kind", ["jw", "perm", "rand"])
def test_basis_change_matches_oracle(seed, kind):
    base = random_workload(seed, "majorana")
    wl = dataclasses.replace(base, extra={**base.extra,
                                          "basis_change": golden.basis_pattern(kind, base.num_modes, 100 + seed)})
    ref = oracle.run_port(wl)
    keys, coefs, ev = run(wl)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert np.all(np.abs(coefs[ia] - ref.coefs[ib]) <= 1e-10 * np.maximum(np.abs(ref.coefs[ib]), 1e-300) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_core_basis_change_surface():
    from monoprop_b200.propagators import dispatch

    wl, L = golden.basis_change_workload("hubbard6x6_L400_bcjw")
    ops = {tuple(k): complex(v) for k, v in wl.observable.items()}
    cls = dispatch(wl.num_modes)
    kw = dict(initial_operator=ops, cutoff=wl.cutoff, initial_state=list(wl.initial_state), cutoff_type="length",
              lower_atol=wl.lower_atol, logical_num_modes=wl.num_modes, basis="majorana")
    with pytest.raises(ValueError, match="basis_change must have exactly 2\\*logical_num_modes"):
        cls(basis_change=[[0]], **kw)
    with pytest.raises(ValueError, match="Pauli basis does not accept a basis_change"):
        dispatch(4)(initial_operator={(0,): 1.0}, cutoff=2, initial_state=[], cutoff_type="support",
                    logical_num_modes=4, basis="pauli", basis_change=[[s] for s in range(8)])
    p = cls(basis_change=wl.extra["basis_change"], **kw)
    assert p.basis_change == wl.extra["basis_change"]
    monos = [list(m) for m in wl.gate_slots[:L]]
    n_params = int(wl.param_map[:L].max()) + 1  # the reference requires exactly max(mapping) + 1 parameters
    p.propagate(monos, list(wl.param_map[:L]), list(wl.gen_coeffs[:L]), list(wl.params[:n_params]))
    g = golden.load("hubbard6x6_L400_bcjw")
    assert p.size() == int(g["n"])
    assert abs(p.expectation_value([]) - float(g["expectation"])) <= 1e-10
    p.basis_change = None
    assert p.basis_change is None


def test_basis_change_gradient_finite_differences():
    base = random_workload(3, "majorana")
    wl = dataclasses.replace(base, lower_atol=None, upper_atol=None,
                             extra={**base.extra, "basis_change": golden.basis_pattern("rand", base.num_modes, 5)})
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words(), wl.angles())
    ev = eng.adjoint_forward(circ)
    grad = eng.adjoint_backward(circ)
    ang = wl.angles()
    h = 1e-5
    for layer in range(0, wl.n_layers, max(1, wl.n_layers // 12)):
        vals = []
        for d in (h, -h):
            a = ang.copy()
            a[layer] += d
            eng.reset()
            eng.propagate(wl.gen_words(), a)
            vals.append(eng.expectation())
        fd = (vals[0] - vals[1]) / (2 * h)
        # per angle: 1e-7 relative, plus 1e-9 for the central difference's own error at h = 1e-5
        assert abs(fd - grad[layer]) <= 1e-7 * abs(fd) + 1e-9, (layer, fd, grad[layer])
    assert np.isfinite(ev)
    circ.close()
    eng.close()


@pytest.mark.parametrize("seed", range(3))
def test_basis_change_with_only_rotate_len_k(seed):
    """Both options at once (the sweep variant that checks the term length and judges the image)."""
    base = random_workload(seed, "majorana")
    wl = dataclasses.replace(base, extra={**base.extra, "only_rotate_len_k": 4,
                                          "basis_change": golden.basis_pattern("rand", base.num_modes, 200 + seed)})
    ref = oracle.run_port(wl)
    eng = _native.engine_for(wl)
    eng.set_only_rotate_len_k(4)
    eng.propagate(wl.gen_words(), wl.angles())
    keys, coefs = eng.export()
    ev = eng.expectation()
    eng.close()
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert np.all(np.abs(coefs[ia] - ref.coefs[ib]) <= 1e-10 * np.maximum(np.abs(ref.coefs[ib]), 1e-300) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))
