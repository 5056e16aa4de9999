"""The frozen structure ("graph"): mpx_graph_build / mpx_graph_expectation / mpx_graph_gradient.

* at the build's own parameters the frozen replay reproduces the propagation (1e-12 relative);
* at shifted parameters it reproduces the reference's own replay of its graph (expectation 1e-10
  relative, gradient 1e-9 of the largest entry; tests/golden/graph_*.npz);
* its gradient is the exact derivative of the frozen replay: central finite differences (h = 1e-5) of
  mpx_graph_expectation on 48 seeded angles agree to 1e-7 relative, whatever truncation is active;
* segmenting the gradient's checkpoints does not change it.
"""

import dataclasses

import numpy as np
import pytest

from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from oracle import golden

pytestmark = pytest.mark.gpu


def prefix(wl, L):
    P = int(wl.param_map[:L].max()) + 1
    return dataclasses.replace(wl, gate_slots=wl.gate_slots[:L], gen_coeffs=wl.gen_coeffs[:L],
                               param_map=wl.param_map[:L], params=wl.params[:P])


def built(wl, segment_gates=0):
    eng = _native.engine_for(wl)
    circ = eng.upload(wl.gen_words(), wl.angles())
    ev = eng.graph_build(circ, segment_gates)
    return eng, circ, ev


def grad_params(wl, ga):
    g = np.zeros(int(wl.param_map.max()) + 1)
    np.add.at(g, wl.param_map, wl.gen_coeffs * ga)
    return g


@pytest.mark.parametrize("name, make, L", [("hubbard6x6_L300", W.hubbard6x6, 300), ("ising100_L600", W.ising100, 600)])
def test_graph_matches_reference_replay(name, make, L):
    g = golden.load("graph_" + name)
    wl = prefix(make(), L)
    eng, circ, ev_build = built(wl)
    assert abs(ev_build - float(g["expectation_build"])) <= 1e-10 * max(1.0, abs(ev_build))
    assert abs(eng.graph_expectation(circ) - ev_build) <= 1e-12 * max(1.0, abs(ev_build))
    circ.set_angles(g["params"][wl.param_map] * wl.gen_coeffs)
    ev = eng.graph_expectation(circ)
    ev2, ga = eng.graph_gradient(circ, segment_gates=97)
    circ.close()
    eng.close()
    ref = float(g["expectation"])
    assert abs(ev - ref) <= 1e-10 * max(1.0, abs(ref))
    assert abs(ev2 - ref) <= 1e-10 * max(1.0, abs(ref))
    grad = grad_params(wl, ga)
    assert np.max(np.abs(grad - g["grad"])) <= 1e-9 * max(1.0, np.max(np.abs(g["grad"])))


@pytest.mark.parametrize("make", [W.line20, lambda: prefix(W.ising100(), 900)])
def test_graph_gradient_is_the_derivative_of_the_replay(make):
    wl = make()
    eng, circ, _ = built(wl)
    rng = np.random.default_rng(21)
    theta = wl.params + 0.03 * rng.standard_normal(wl.params.size)

    def expval(t):
        circ.set_angles(t[wl.param_map] * wl.gen_coeffs)
        return eng.graph_expectation(circ)

    expval(theta)
    _, ga = eng.graph_gradient(circ)
    grad = grad_params(wl, ga)
    _, ga2 = eng.graph_gradient(circ, segment_gates=64)
    assert np.max(np.abs(ga - ga2)) <= 1e-13 * max(1.0, np.max(np.abs(ga)))
    h = 1e-5
    for p in rng.choice(theta.size, size=min(48, theta.size), replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        fd = (expval(tp) - expval(tm)) / (2 * h)
        # per angle: 1e-7 relative, plus 1e-9 for the central difference's own error at h = 1e-5
        assert abs(fd - grad[p]) <= 1e-7 * abs(fd) + 1e-9, (p, fd, grad[p])
    circ.close()
    eng.close()
