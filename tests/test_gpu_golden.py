"""CUDA engine (through the C ABI) against the reference's golden fixtures and the oracle.

* seeded workloads and the reference's own exact-energy fixtures (tests/golden/, generated from the
  unmodified reference engine): keys bit-exact, coefficients and <O> within 1e-10 relative, exact
  energies within 1e-12 (tests/test_infinite_cutoff.py:39-68 of the reference);
* random small Pauli and Majorana circuits with truncation active, against the oracle port;
* engine life cycle: reset, device-resident circuits with replaced angles, store growth from a tiny
  initial capacity.
"""

import numpy as np
import pytest

import oracle
from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from monoprop_b200.encoding import canonical_order
from oracle import golden
from oracle.golden import random_workload

pytestmark = pytest.mark.gpu

SEEDED = {"line20": (W.line20, None), "line20_L200": (W.line20, 200), "hubbard6x6_L400": (W.hubbard6x6, 400),
          "ising100_L600": (W.ising100, 600), "ising50_d2": (lambda: W.ising50(2), None),
          "ising50_d3": (lambda: W.ising50(3), None), "ising100_L1200": (W.ising100, 1200)}


def run_engine(wl, n_layers=None, **kw):
    eng = _native.engine_for(wl, **kw)
    L = wl.n_layers if n_layers is None else n_layers
    eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
    keys, coefs = eng.export()
    ev = eng.expectation()
    eng.close()
    return keys, coefs, ev


@pytest.mark.parametrize("name", golden.SEEDED)
def test_engine_matches_reference_golden(name):
    make, L = SEEDED[name]
    keys, coefs, ev = run_engine(make(), L)
    golden.check_against(golden.load(name), keys, coefs, ev)


@pytest.mark.parametrize("name", golden.REF_CASES)
def test_engine_reproduces_reference_fixture(name):
    g = golden.load(name)
    keys, coefs, ev = run_engine(golden.fixture_workload(g, name))
    golden.check_against(g, keys, coefs, ev)
    if np.isnan(float(g["lower_atol"])):
        assert abs(ev - float(g["exact_energy"])) <= 1e-12


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
def test_engine_matches_oracle_random(seed, basis):
    wl = random_workload(seed, basis)
    ref = oracle.run_port(wl)
    keys, coefs, ev = run_engine(wl)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    a, b = coefs[ia], ref.coefs[ib]
    assert np.all(np.abs(a - b) <= 1e-10 * np.maximum(np.abs(a), np.abs(b)) + 1e-15)
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_reset_and_resident_circuit_with_new_angles():
    wl = W.hubbard6x6()
    L = 500
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    eng.propagate_circuit(circ)
    first = eng.expectation()
    eng.reset()
    eng.propagate_circuit(circ)
    # appends land in a run-dependent order, so the sum may differ in the last bits
    assert abs(eng.expectation() - first) <= 1e-14 * max(1.0, abs(first))
    p2 = wl.params * 1.1
    circ.set_angles(wl.angles(p2)[:L])
    eng.reset()
    eng.propagate_circuit(circ)
    keys, coefs = eng.export()
    ev = eng.expectation()
    circ.close()
    eng.close()
    ref = oracle.run_port(wl, params=p2, n_layers=L)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))


def test_resident_circuit_replays_a_captured_cuda_graph():
    """The 100-qubit circuit's first 1200 gates, resident: the first propagation grows the store, the
    second (no growth) captures the streaming gate range after the shared-memory hand-off, the third
    replays it as one CUDA graph. All three give the reference's store (keys bit-exact, coefficients
    bit-identical per key)."""
    wl = W.ising100()
    L = 1200
    g = golden.load("ising100_L1200")
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    runs = []
    for _ in range(3):
        eng.reset()
        eng.propagate_circuit(circ)
        keys, coefs = eng.export()
        runs.append((keys, coefs, eng.expectation()))
    replays = eng.graph_replay_count()
    circ.close()
    eng.close()
    assert replays == 1
    for keys, coefs, ev in runs:
        golden.check_against(g, keys, coefs, ev)
    (k0, c0, _), (k2, c2, _) = runs[0], runs[2]
    i0, i2 = canonical_order(k0), canonical_order(k2)
    assert np.array_equal(k0[i0], k2[i2]) and np.array_equal(c0[i0], c2[i2])


def test_growth_from_tiny_capacity_matches_presized():
    wl = W.ising50(3)
    k1, c1, e1 = run_engine(wl, capacity_hint=1)
    k2, c2, e2 = run_engine(wl, capacity_hint=1 << 20)
    i1, i2 = canonical_order(k1), canonical_order(k2)
    assert np.array_equal(k1[i1], k2[i2])
    assert np.array_equal(c1[i1], c2[i2])
    assert abs(e1 - e2) <= 1e-12 * max(1.0, abs(e2))
