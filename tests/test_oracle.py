"""The oracle (C restatement in oracle/mp_oracle.c) pinned against the reference.

* against the golden fixtures generated from the unmodified reference engine (tests/golden/), including
  the reference's own exact-energy test fixtures at infinite cutoff (exact energy to 1e-12, the
  reference tests' tolerance: tests/test_infinite_cutoff.py:39-68);
* against the reference engine itself, live, when oracle/_ref/libmpref.so has been built here
  (random Pauli and Majorana circuits exercising lower_atol, upper_atol rescue, odd-weight generators,
  near-zero cosines and the fully-paired exemption);
* on the analytic one-gate truncation cases of the reference's tests/test_coeff_trunc.py:59-96;
* with only_rotate_len_k, with a basis_change and in the Schrodinger picture, against golden fixtures
  and the live reference.
"""

import dataclasses

import numpy as np
import pytest

import oracle
from monoprop_b200 import workloads as W
from monoprop_b200.encoding import canonical_order
from oracle import golden
from oracle.golden import random_workload

SEEDED = {"line20": (W.line20, None), "line20_L200": (W.line20, 200), "hubbard6x6_L400": (W.hubbard6x6, 400),
          "ising100_L600": (W.ising100, 600), "ising50_d2": (lambda: W.ising50(2), None),
          "ising50_d3": (lambda: W.ising50(3), None), "ising100_L1200": (W.ising100, 1200)}


@pytest.mark.parametrize("name", golden.SEEDED)
def test_port_matches_reference_golden(name):
    make, L = SEEDED[name]
    g = golden.load(name)
    r = oracle.run_port(make(), n_layers=L)
    golden.check_against(g, r.keys, r.coefs, r.expectation)


@pytest.mark.parametrize("name", golden.REF_CASES)
def test_port_reproduces_reference_fixture(name):
    g = golden.load(name)
    wl = golden.fixture_workload(g, name)
    r = oracle.run_port(wl)
    golden.check_against(g, r.keys, r.coefs, r.expectation)
    if np.isnan(float(g["lower_atol"])):
        assert abs(r.expectation - float(g["exact_energy"])) <= 1e-12


def test_port_matches_full_depth_hubbard_digest():
    """The full 6x6 Hubbard circuit (2208 gates, 6.4e6 terms) against the reference's full-depth digest."""
    wl = golden.FULL_DEPTH["hubbard6x6"]()
    r = oracle.run_port(wl)
    assert golden.check_digest(golden.load("full_hubbard6x6"), r.keys, r.coefs, r.expectation)


def test_digest_detects_planted_errors():
    """The bucketed digest catches one coefficient off by 1e-8 relative, one key changed, and one term
    missing (mistakes planted in the oracle's own output)."""
    r = oracle.run_port(W.line20())
    g = golden.bucket_digest(r.keys, r.coefs)
    g["expectation"] = np.float64(r.expectation)
    assert golden.check_digest(g, r.keys, r.coefs, r.expectation)
    i = int(np.argsort(np.abs(r.coefs))[r.coefs.size // 2])  # a mid-sized coefficient, not among the largest
    bad = r.coefs.copy()
    bad[i] *= 1 + 1e-8
    with pytest.raises(AssertionError):
        golden.check_digest(g, r.keys, bad, r.expectation)
    keys = r.keys.copy()
    keys[i, 0] ^= np.uint64(1)
    with pytest.raises(AssertionError):
        golden.check_digest(g, keys, r.coefs, r.expectation)
    with pytest.raises(AssertionError):
        golden.check_digest(g, r.keys[1:], r.coefs[1:], r.expectation)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built here")
@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
def test_port_matches_reference_live(seed, basis):
    wl = random_workload(seed, basis)
    a, b = oracle.run_port(wl), oracle.run_ref(wl)
    ia, ib = canonical_order(a.keys), canonical_order(b.keys)
    assert np.array_equal(a.keys[ia], b.keys[ib])
    assert np.array_equal(a.coefs[ia], b.coefs[ib])
    assert a.expectation == b.expectation


@pytest.mark.parametrize("name", sorted(golden.LEN_K))
def test_port_matches_reference_golden_len_k(name):
    """only_rotate_len_k (Scan.h:146-157,376-391): terms longer than k sit out the gate."""
    wl, L = golden.len_k_workload(name)
    r = oracle.run_port(wl, n_layers=L)
    golden.check_against(golden.load(name), r.keys, r.coefs, r.expectation)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built here")
@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
@pytest.mark.parametrize("k", [2, 4, 6])
def test_port_matches_reference_live_len_k(seed, basis, k):
    base = random_workload(seed, basis)
    wl = dataclasses.replace(base, extra={**base.extra, "only_rotate_len_k": k})
    a, b = oracle.run_port(wl), oracle.run_ref(wl)
    ia, ib = canonical_order(a.keys), canonical_order(b.keys)
    assert np.array_equal(a.keys[ia], b.keys[ib])
    assert np.array_equal(a.coefs[ia], b.coefs[ib])
    assert a.expectation == b.expectation


@pytest.mark.parametrize("name", sorted(golden.BASIS_CHANGE))
def test_port_matches_reference_golden_basis_change(name):
    """basis_change: the partner's cutoff is judged on its image (MonomialPropagatorCommon.h:44-62)."""
    wl, L = golden.basis_change_workload(name)
    r = oracle.run_port(wl, n_layers=L)
    golden.check_against(golden.load(name), r.keys, r.coefs, r.expectation)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built here")
@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("kind", ["jw", "perm", "rand"])
def test_port_matches_reference_live_basis_change(seed, kind):
    base = random_workload(seed, "majorana")
    wl = dataclasses.replace(base, extra={**base.extra,
                                          "basis_change": golden.basis_pattern(kind, base.num_modes, 100 + seed)})
    a, b = oracle.run_port(wl), oracle.run_ref(wl)
    ia, ib = canonical_order(a.keys), canonical_order(b.keys)
    assert np.array_equal(a.keys[ia], b.keys[ib])
    assert np.array_equal(a.coefs[ia], b.coefs[ib])
    assert a.expectation == b.expectation


@pytest.mark.parametrize("name", sorted(golden.SCHRODINGER))
def test_port_matches_reference_golden_schrodinger(name):
    """Schrodinger picture: paired-monomial state evolved first to last at the negated angle."""
    wl, L = golden.schrodinger_workload(name)
    r = oracle.run_port(wl, n_layers=L)
    golden.check_against(golden.load(name), r.keys, r.coefs, r.expectation)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built here")
@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("basis", ["pauli", "majorana"])
def test_port_matches_reference_live_schrodinger(seed, basis):
    base = random_workload(seed, basis)
    wl = dataclasses.replace(base, extra={**base.extra, "schrodinger_cutoff": base.cutoff + 1})
    a, b = oracle.run_port(wl), oracle.run_ref(wl)
    ia, ib = canonical_order(a.keys), canonical_order(b.keys)
    assert np.array_equal(a.keys[ia], b.keys[ib])
    assert np.array_equal(a.coefs[ia], b.coefs[ib])
    assert abs(a.expectation - b.expectation) <= 1e-12 * max(1.0, abs(b.expectation))  # summation order


def one_gate(cutoff, upper_atol, lower_atol):
    """exp(i pi/6 m1 m2 m3 m4) on the observable i m0 m1 (tests/test_coeff_trunc.py:59-96)."""
    return W.Workload("one_gate", "majorana", 5, [(1, 2, 3, 4)], np.array([1.0]), np.array([0]),
                      np.array([np.pi / 6]), {(0, 1): 1j}, [], cutoff, "length", lower_atol, upper_atol)


@pytest.mark.parametrize("cutoff, upper_atol, lower_atol, kept", [
    (4, None, None, True), (1, 0.49, None, True), (1, 1.0, None, False), (4, None, 0.9, False),
    (10, None, 0.1, True)])
def test_analytic_one_gate_truncation(cutoff, upper_atol, lower_atol, kept):
    r = oracle.run_port(one_gate(cutoff, upper_atol, lower_atol))
    from monoprop_b200.encoding import words_to_slots
    got = {words_to_slots(k, 5): c for k, c in zip(r.keys, r.coefs)}
    # encoded coefficients: i m0 m1 -> 1 (÷ i^1); cos(pi/3) = 0.5; the sine branch m0 m2 m3 m4 carries
    # -sin(pi/3) after decoding (i^C(4,2) = -1 encoding)
    assert got[(0, 1)] == pytest.approx(0.5, abs=1e-15)
    if kept:
        assert got[(0, 2, 3, 4)] == pytest.approx(0.8660254037844386, abs=1e-15)
    else:
        assert (0, 2, 3, 4) not in got


def test_term_gate_update_count_of_the_line_circuit():
    from monoprop_b200.workloads import TERM_GATE_UPDATES

    r = oracle.run_port(W.line20())
    assert int(r.counts[:, 0].sum()) == TERM_GATE_UPDATES["line20"]
