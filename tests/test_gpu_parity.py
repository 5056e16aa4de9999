"""CUDA engine vs the oracle on the same seeded inputs (bit-exact sets, coefficients within 1e-10).

The oracle is the C restatement in oracle/ (pinned bit-exact against the unmodified reference engine in
tests/test_oracle.py). Tolerance: keys must match exactly; coefficients |a-b| <= 1e-10*max(|a|,|b|) +
1e-15 (they are expected to be bit-identical: the kernels reproduce the reference's FMA contraction);
<O> within 1e-10 relative.
"""

import numpy as np
import pytest

import oracle
from monoprop_b200 import _native, workloads as W
from monoprop_b200.encoding import canonical_order

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def compare(wl, n_layers=None):
    ref = oracle.run_port(wl, n_layers=n_layers)
    eng = _native.engine_for(wl)
    L = wl.n_layers if n_layers is None else n_layers
    eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
    keys, coefs = eng.export()
    ev = eng.expectation()
    st = eng.gate_stats()
    eng.close()
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert keys.shape == ref.keys.shape
    assert np.array_equal(keys[ia], ref.keys[ib])
    a, b = coefs[ia], ref.coefs[ib]
    tol = RTOL * np.maximum(np.abs(a), np.abs(b)) + 1e-15
    assert np.all(np.abs(a - b) <= tol), float(np.max(np.abs(a - b)))
    assert abs(ev - ref.expectation) <= RTOL * max(1.0, abs(ref.expectation))
    # per-gate counters agree with the oracle's
    np.testing.assert_array_equal(st.n, ref.counts[:, 0])
    np.testing.assert_array_equal(st.anti, ref.counts[:, 1])
    np.testing.assert_array_equal(st.emitted, ref.counts[:, 2])
    np.testing.assert_array_equal(st.appended, ref.counts[:, 3])
    return keys, coefs, ev


def test_line20_full():
    compare(W.line20())


def test_ising100_prefix():
    compare(W.ising100(), n_layers=900)


def test_hubbard_prefix():
    compare(W.hubbard6x6(), n_layers=600)


def test_ising50_depth5():
    compare(W.ising50(5))


@pytest.mark.parametrize("name", ["line20", "hubbard6x6", "ising100"])
def test_term_gate_update_counts(name):
    """The engine's per-gate counters sum to the oracle's term-gate update count of each bench workload."""
    wl = W.BY_NAME[name]()
    eng = _native.engine_for(wl)
    eng.propagate(wl.gen_words(), wl.angles())
    assert eng.gate_stats().term_gate_updates == W.TERM_GATE_UPDATES[name]
    eng.close()
