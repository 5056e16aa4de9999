"""The engine's adjoint gradient (mpx_adjoint_forward / mpx_adjoint_backward) and its torch wrapper.

Checks, all of the gradient of the frozen-structure surrogate (the derivative the reference's
expectation_value_and_gradient returns, MPFunctions.cpp:207-246):

* exact gradients of the reference's own fixtures at infinite cutoff (tests/data/*.msgpack copies);
* the reference's replayed-graph gradient on seeded circuits (tests/golden/grad_*.npz) and its
  parameter-shift gradient on the 20-qubit line circuit (tests/golden/pshift_line20.npz);
* central finite differences (h = 1e-5) of the plain propagation where the truncation structure cannot
  change with the angles (weight cutoff only, no coefficient thresholds): 1e-7 relative;
* segmenting (checkpoint interval) does not change the result; the engine keeps the forward pass's
  evolved operator afterwards; torch autograd returns the same gradient.
"""

import dataclasses

import numpy as np
import pytest
import torch

import oracle
from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from monoprop_b200.autograd import DifferentiablePropagation
from monoprop_b200.encoding import canonical_order
from oracle import golden

pytestmark = pytest.mark.gpu

# Per-angle finite-difference tolerance: |fd - grad| <= 1e-7 |fd| + FD_ATOL. FD_ATOL covers the central
# difference's own error at h = 1e-5 (h^2 |f'''| / 6 + eps |<O>| / h, below 1e-10 for these circuits),
# so an angle whose derivative is near zero is still held to an absolute 1e-9.
FD_RTOL = 1e-7
FD_ATOL = 1e-9


def value_and_grad(wl, theta=None, segment_gates=0):
    dp = DifferentiablePropagation(wl, segment_gates=segment_gates)
    try:
        return dp.value_and_grad(wl.params if theta is None else theta)
    finally:
        dp.close()


def prefix(wl, L):
    P = int(wl.param_map[:L].max()) + 1
    return dataclasses.replace(wl, gate_slots=wl.gate_slots[:L], gen_coeffs=wl.gen_coeffs[:L],
                               param_map=wl.param_map[:L], params=wl.params[:P])


@pytest.mark.parametrize("name", ["ref_rx_rz_ry_rz_exact", "ref_random_exact", "ref_lih_fermionic_spin_exact"])
def test_exact_fixture_gradient(name):
    g = golden.load(name)
    ev, grad = value_and_grad(golden.fixture_workload(g, name))
    assert abs(ev - float(g["exact_energy"])) <= 1e-12
    ref = g["exact_gradient"]
    assert np.max(np.abs(grad - ref)) <= 1e-10 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("name, make, L", [("hubbard6x6_L300", W.hubbard6x6, 300), ("ising100_L600", W.ising100, 600),
                                           ("ising50_d2", lambda: W.ising50(2), None)])
def test_reference_replay_gradient(name, make, L):
    g = golden.load("grad_" + name)
    wl = make()
    wl = prefix(wl, L) if L is not None else wl
    ev, grad = value_and_grad(wl)
    assert abs(ev - float(g["expectation"])) <= 1e-10 * max(1.0, abs(float(g["expectation"])))
    assert np.max(np.abs(grad - g["grad"])) <= 1e-9 * max(1.0, np.max(np.abs(g["grad"])))


def test_parameter_shift_line20():
    g = golden.load("pshift_line20")
    ev, grad = value_and_grad(W.line20())
    assert abs(ev - float(g["expectation"])) <= 1e-10
    assert np.max(np.abs(grad - g["grad"])) <= 1e-9 * max(1.0, np.max(np.abs(g["grad"])))


def expectation(wl, theta):
    eng = _native.engine_for(wl)
    eng.propagate(wl.gen_words(), theta[wl.param_map] * wl.gen_coeffs)
    ev = eng.expectation()
    eng.close()
    return ev


@pytest.mark.parametrize("make", [lambda: W.line20(layers=6), lambda: prefix(W.hubbard6x6(), 400)])
def test_finite_differences_structural_truncation(make):
    wl = dataclasses.replace(make(), lower_atol=None, upper_atol=None)
    theta = wl.params.copy()
    ev, grad = value_and_grad(wl, theta)
    rng = np.random.default_rng(11)
    h = 1e-5
    for p in rng.choice(theta.size, size=min(64, theta.size), replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        fd = (expectation(wl, tp) - expectation(wl, tm)) / (2 * h)
        assert abs(fd - grad[p]) <= FD_RTOL * abs(fd) + FD_ATOL, (p, fd, grad[p])


def test_segments_and_final_state():
    wl = prefix(W.ising100(), 900)
    ev1, g1 = value_and_grad(wl, segment_gates=0)
    dp = DifferentiablePropagation(wl, segment_gates=128)
    ev2, g2 = dp.value_and_grad(wl.params)
    keys, coefs = dp.engine.export()
    ev3 = dp.engine.expectation()
    dp.close()
    # separate runs may append in a different order, so sums can differ in the last bits
    assert ev2 == ev3 and abs(ev1 - ev2) <= 1e-14 * max(1.0, abs(ev1))
    assert np.max(np.abs(g1 - g2)) <= 1e-13 * max(1.0, np.max(np.abs(g1)))
    ref = oracle.run_port(wl)
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert np.array_equal(keys[ia], ref.keys[ib])
    assert np.max(np.abs(coefs[ia] - ref.coefs[ib])) <= 1e-12


def test_torch_autograd():
    wl = prefix(W.hubbard6x6(), 300)
    dp = DifferentiablePropagation(wl)
    theta = torch.tensor(wl.params, dtype=torch.float64, requires_grad=True)
    e = dp(theta)
    e.backward()
    ev, grad = dp.value_and_grad(wl.params)
    dp.close()
    assert abs(float(e) - ev) <= 1e-14 * max(1.0, abs(ev))
    assert np.max(np.abs(theta.grad.numpy() - grad)) <= 1e-13 * max(1.0, np.max(np.abs(grad)))


def test_full_circuit_gradient_finite_differences():
    """The 100-qubit, 5600-angle circuit with checkpoints every 4 circuit layers (1120 gates) against
    central finite differences (h = 1e-5) of the reference's replayed graph on 64 seeded angles
    (tests/golden/fd_ising100.npz): 1e-7 relative per angle."""
    g = golden.load("fd_ising100")
    ev, grad = value_and_grad(W.ising100(), segment_gates=4 * 280)
    assert abs(ev - float(g["expectation"])) <= 1e-10 * max(1.0, abs(float(g["expectation"])))
    fd = g["fd"]
    err = np.abs(grad[g["idx"]] - fd)
    assert np.all(err <= FD_RTOL * np.abs(fd) + FD_ATOL), (g["idx"][np.argmax(err)], float(np.max(err)))


@pytest.mark.parametrize("make, L", [(W.hubbard6x6, 300), (W.ising100, 600)])
def test_pair_log_and_replay_agree(make, L):
    """The forward pass's pair log (backward without the hash resolve), no log (resolve replay) and a log
    too small to hold the pass (overflow: replay) give the same gradient, and graphs built either way
    give the same replayed expectation and gradient at new angles."""
    wl = prefix(make(), L)
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words(), wl.angles())
    out = {}
    for cap in (-1, 0, 1000):
        eng.set_pair_log(cap)
        ev = eng.adjoint_forward(circ, segment_gates=64)
        out[cap] = (ev, eng.adjoint_backward(circ))
    ref_ev, ref_g = out[0]
    for cap in (-1, 1000):
        ev, g = out[cap]
        assert abs(ev - ref_ev) <= 1e-14 * max(1.0, abs(ref_ev))
        assert np.max(np.abs(g - ref_g)) <= 1e-10 * max(1.0, np.max(np.abs(ref_g)))
    theta = wl.params * 1.1 + 0.01
    graphs = {}
    for cap in (-1, 0):
        eng.set_pair_log(cap)
        circ.set_angles(wl.angles())
        eng.graph_build(circ)
        circ.set_angles(wl.angles(theta))
        graphs[cap] = (eng.graph_expectation(circ), *eng.graph_gradient(circ))
    a, b = graphs[-1], graphs[0]
    assert abs(a[0] - b[0]) <= 1e-12 * max(1.0, abs(b[0]))
    assert abs(a[1] - b[1]) <= 1e-12 * max(1.0, abs(b[1]))
    assert np.max(np.abs(a[2] - b[2])) <= 1e-10 * max(1.0, np.max(np.abs(b[2])))
    circ.close()
    eng.close()


def _logged_case(name):
    """(workload, layers, only_rotate_len_k) of a logged-backward case."""
    if name == "ising100_L600":
        return W.ising100(), 600, None
    if name == "hubbard6x6_L300":
        return W.hubbard6x6(), 300, None
    if name == "hubbard6x6_L300_k4":
        return W.hubbard6x6(), 300, 4
    wl = W.line20()  # Schrodinger picture, 200 layers
    return dataclasses.replace(wl, extra={**wl.extra, "schrodinger_cutoff": 4}), 200, None


@pytest.mark.parametrize("name", ["ising100_L600", "hubbard6x6_L300", "hubbard6x6_L300_k4", "line20_L200_s4"])
def test_logged_backward_equals_replayed_backward(name):
    """Once an engine knows a circuit's undo-log size, its next gradient forward pass logs everything the
    reverse sweep needs and the backward pass replays nothing. The gradient is the same as with the segment
    replay (the logged partner values are the ones the forward pass computed: 1e-12 relative), and <O> too;
    without a pair log nothing is logged."""
    wl, L, k = _logged_case(name)
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words()[:L], wl.angles()[:L])
    eng.set_only_rotate_len_k(k)
    ev1 = eng.adjoint_forward(circ, 64)
    assert not eng.adjoint_logged()  # no size known yet: checkpoints and segment replay
    g1 = eng.adjoint_backward(circ)
    ev2 = eng.adjoint_forward(circ, 64)
    assert eng.adjoint_logged()
    g2 = eng.adjoint_backward(circ)
    eng.set_pair_log(0)
    eng.adjoint_forward(circ, 64)
    assert not eng.adjoint_logged()
    g3 = eng.adjoint_backward(circ)
    circ.close()
    eng.close()
    assert abs(ev1 - ev2) <= 1e-13 * max(1.0, abs(ev1))
    scale = max(1.0, float(np.max(np.abs(g1))))
    assert np.max(np.abs(g2 - g1)) <= 1e-12 * scale
    assert np.max(np.abs(g3 - g1)) <= 1e-12 * scale
    assert np.count_nonzero(np.abs(g1) > 1e-9) > 0
