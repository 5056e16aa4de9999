"""Generates the golden fixtures in this directory from the UNMODIFIED reference engine.

Run in a container that has the reference sources (the GPU hosts do not): it builds
``oracle/_ref/libmpref.so`` from them (``oracle/build_ref.sh``) and writes

* ``<workload>.npz`` -- seeded workloads propagated by the reference engine (``partitions=1``), raw FP64
  coefficients exported at the C++ level (not the rounded ``evolved_operator`` dict), keys sorted
  canonically, ``<0|O|0>``; bigger stores keep only a digest: term count, SHA-256 of the sorted keys,
  sum and sum of squares of the coefficients in key order;
* ``grad_<workload>.npz`` -- the reference's gradient of the frozen-structure surrogate (graph built with
  the same parameters, then ``expectation_value_and_gradient``), per parameter;
* ``graph_<workload>.npz`` -- the reference's frozen graph (built at the workload's parameters) replayed
  at shifted parameters: expectation and gradient there (``--graph-len-k``: graphs built with
  ``only_rotate_len_k``; ``--graph-schrodinger``: graphs in the Schrodinger picture, ``graph_*_s<cutoff>``;
  ``--graph-replay``: raw coefficients of a len_k graph replayed at its build parameters,
  ``graph_replay_*``);
* ``pshift_line20.npz`` -- parameter-shift gradient of the 20-qubit line circuit from the reference's
  replayed graph;
* ``<workload>_k<k>.npz`` -- seeded workloads propagated with ``only_rotate_len_k = k``;
* ``<workload>_bc<pattern>.npz`` -- seeded Majorana workloads with a ``basis_change``, and
  ``<workload>_s<cutoff>.npz`` -- seeded workloads in the Schrodinger picture (both written with the
  ``only_rotate_len_k`` fixtures);
* ``ref_<case>.npz`` -- the reference's own exact-energy test fixtures
  (``tests/data/{rx_rz_ry_rz_exact,random_exact,lih_fermionic_spin_exact}.msgpack``), re-expressed as
  engine arrays by this repository's front-end (``Circuit.from_dense_arrays`` + ``expand_monomials``,
  ``MajoranaOperator`` canonicalisation), with the fixture's exact energy and gradient and the reference
  engine's raw output at infinite cutoff (``cutoff = 2 n``).

* ``full_<workload>.npz`` -- the full-depth benchmark circuits (100-qubit kicked Ising, 5600 gates;
  6x6 Hubbard, 2208 gates; two instances of the batched 50-qubit workload at depths 24 and 12), whose
  final stores (up to ~4.4e7 terms) are kept as a bucketed digest (``oracle.golden.bucket_digest``): key
  set SHA-256, per-bucket counts, sums of |c| and of two pseudo-random projections of c, the 4096 largest
  coefficients with their positions, and <0|O|0>.

Usage: ``python tests/golden/make_golden.py [REFERENCE_ROOT] [--fd-full] [--len-k-only] [--full-depth]``
(``--fd-full`` adds the slow finite-difference golden of the full 100-qubit circuit; ``--len-k-only``
writes only the ``only_rotate_len_k`` fixtures; ``--full-depth`` writes only the ``full_*`` digests, a few
minutes on 8 cores). REFERENCE_ROOT defaults to ``$MONOPROP_REFERENCE``.
"""

from __future__ import annotations

import dataclasses
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import golden  # noqa: E402
from monoprop_b200 import workloads as W  # noqa: E402
from monoprop_b200.circuit import Circuit  # noqa: E402
from monoprop_b200.encoding import canonical_order  # noqa: E402
from monoprop_b200.operators import MajoranaOperator  # noqa: E402

FULL_LIMIT = 40_000  # stores up to this many terms are stored in full

SEEDED = [
    ("line20", W.line20, None),
    ("line20_L200", W.line20, 200),
    ("hubbard6x6_L400", W.hubbard6x6, 400),
    ("ising100_L600", W.ising100, 600),
    ("ising50_d2", lambda: W.ising50(2), None),
    ("ising50_d3", lambda: W.ising50(3), None),
    ("ising100_L1200", W.ising100, 1200),
]

# only_rotate_len_k cases: (name, workload, layers, k)
LEN_K = [
    ("line20_k6", W.line20, None, 6),
    ("hubbard6x6_L400_k4", W.hubbard6x6, 400, 4),
    ("ising50_d3_k8", lambda: W.ising50(3), None, 8),
]

REF_CASES = ["rx_rz_ry_rz_exact", "random_exact", "lih_fermionic_spin_exact"]

# Gradients of the frozen-structure surrogate from the reference's graph replay (build_graph seeded
# with the same parameters, then expectation_value_and_gradient): grad_<name>.npz. These circuits keep
# |cos(2 angle)| >= 0.58; the 20-qubit line circuit (angles up to pi) has a gate with |cos| = 1.2e-4,
# where the reference's analytic gradient (which un-scales by 1/cos) loses accuracy, so its golden
# gradient is the parameter shift of the replayed graph instead (pshift_line20.npz).
GRADS = [
    ("hubbard6x6_L300", W.hubbard6x6, 300),
    ("ising100_L600", W.ising100, 600),
    ("ising50_d2", lambda: W.ising50(2), None),
]

GRAPHS = [("hubbard6x6_L300", W.hubbard6x6, 300), ("ising100_L600", W.ising100, 600)]

# The full 100-qubit, 5600-angle circuit: the reference's analytic gradient drifts for the angles it
# reaches last in its reverse sweep (angle 5202: -1.2165 analytic vs 4.6e-5 by finite differences of the
# same replayed graph), so the golden is central finite differences (h = 1e-5) of its replayed graph on
# 64 seeded angles (fd_ising100.npz; about 15 minutes on 8 cores).
FD_FULL = ("ising100", W.ising100, 64, 1e-5, 2024)


def digest(keys: np.ndarray, coefs: np.ndarray) -> dict:
    order = canonical_order(keys)
    k, c = np.ascontiguousarray(keys[order]), coefs[order]
    return {"n": np.int64(k.shape[0]), "sha256": np.bytes_(hashlib.sha256(k.tobytes()).hexdigest()),
            "coef_sum": np.float64(c.sum()), "coef_sumsq": np.float64((c * c).sum())}


def save_result(path: str, keys: np.ndarray, coefs: np.ndarray, ev: float, extra: dict) -> None:
    order = canonical_order(keys)
    payload = {"expectation": np.float64(ev), **digest(keys, coefs), **extra}
    if keys.shape[0] <= FULL_LIMIT:
        payload["keys"] = np.ascontiguousarray(keys[order])
        payload["coefs"] = coefs[order]
    np.savez_compressed(path, **payload)


def fixture_workload(name: str, reference_root: str, lower_atol=None):
    import msgpack

    with open(os.path.join(reference_root, "tests", "data", name + ".msgpack"), "rb") as f:
        d = msgpack.unpackb(f.read())
    n = int(d["num_modes"])
    circ = Circuit.from_dense_arrays([tuple(m) for m in d["majoranas"]], d["gen_coeffs"], d["param_inds"], n,
                                     d["parameters"], d["hartree_fock"])
    ham = d["hamiltonian"]
    op = MajoranaOperator({tuple(k): complex(r, i) for k, r, i in zip(ham["keys"], ham["real"], ham["imag"])}, n)
    wl = W.from_circuit(name, op, circ, cutoff=2 * n, cutoff_type="length", lower_atol=lower_atol)
    return wl, float(d["actual_energy"]), np.asarray(d["actual_gradient"], dtype=np.float64)


def full_depth(names=None) -> None:
    """Digests of the full-depth circuits (all, or ``names``), propagated by the reference with one
    partition (its raw export needs the whole store in one partition)."""
    for name, make in golden.FULL_DEPTH.items():
        if names and name not in names:
            continue
        wl = make()
        r = oracle.run_ref(wl)
        d = golden.bucket_digest(r.keys, r.coefs)
        np.savez_compressed(os.path.join(HERE, f"full_{name}.npz"), expectation=np.float64(r.expectation),
                            n_layers=np.int64(wl.n_layers), seconds=np.float64(r.seconds), **d)
        print("full", name, wl.n_layers, r.keys.shape[0], r.expectation, f"{r.seconds:.1f} s", flush=True)


#: frozen graphs built with only_rotate_len_k: (name, workload, layers, k)
GRAPHS_LEN_K = [("hubbard6x6_L300_k4", W.hubbard6x6, 300, 4), ("ising100_L600_k6", W.ising100, 600, 6)]


def graphs_len_k() -> None:
    """graph_<name>.npz for graphs built with only_rotate_len_k (build_graph's argument, binder.h:102-110):
    the reference's replay at the build parameters and at shifted ones (seed 77, 0.05 N(0, 1)) with its
    gradient there, plus central finite differences (h = 1e-5) of the replay on 32 seeded parameters."""
    for name, make, L, k in GRAPHS_LEN_K:
        wl = make()
        wl = dataclasses.replace(wl, extra={**wl.extra, "only_rotate_len_k": k})
        eng = oracle.RefEngine(wl)
        eng.propagate(n_layers=L, build_graph=True)
        n_params = int(wl.param_map[:L].max()) + 1
        theta = wl.params[:n_params]
        shifted = theta + 0.05 * np.random.default_rng(77).standard_normal(n_params)
        ev, grad, _ = eng.expectation_and_gradient(shifted)
        ev0 = eng.expectation(theta)
        idx = np.sort(np.random.default_rng(5).choice(n_params, size=min(32, n_params), replace=False))
        h = 1e-5
        fd = np.zeros(idx.size)
        for j, p in enumerate(idx):
            tp, tm = shifted.copy(), shifted.copy()
            tp[p] += h
            tm[p] -= h
            fd[j] = (eng.expectation(tp) - eng.expectation(tm)) / (2 * h)
        eng.close()
        np.savez_compressed(os.path.join(HERE, f"graph_{name}.npz"), expectation=np.float64(ev),
                            expectation_build=np.float64(ev0), grad=grad, params=shifted, n_layers=np.int64(L),
                            only_rotate_len_k=np.int64(k), fd_idx=idx, fd=fd)
        print("graph len_k", name, ev0, ev, float(np.abs(grad).max()), float(np.max(np.abs(grad[idx] - fd))))


def graph_replays() -> None:
    """graph_replay_hubbard6x6_L400_k4.npz: the raw coefficients of the reference's graph built with
    only_rotate_len_k = 4, replayed at its build parameters (contract_partially(params, false)), keys sorted.
    Its replay recomputes each layer's cos set with no length filter (MonomialPropagator.inl:872-895), so
    these differ from its own propagation (hubbard6x6_L400_k4.npz) on the terms outside the set and on what
    they rotate into, while <O> agrees."""
    wl = dataclasses.replace(W.hubbard6x6(), extra={**W.hubbard6x6().extra, "only_rotate_len_k": 4})
    L = 400
    eng = oracle.RefEngine(wl)
    eng.propagate(n_layers=L, build_graph=True)
    P = int(wl.param_map[:L].max()) + 1
    ev = eng.expectation(wl.params[:P])
    keys, coefs = eng.export(wl.params[:P])
    eng.close()
    save_result(os.path.join(HERE, "graph_replay_hubbard6x6_L400_k4.npz"), keys, coefs, ev,
                {"n_layers": np.int64(L), "only_rotate_len_k": np.int64(4)})
    print("graph replay hubbard6x6_L400_k4", keys.shape[0], ev)


def _schr_fixture(fixture: str, cutoff: int, sc: int, k=None):
    """The reference's own fermionic test problem ``fixture`` (a ``ref_*`` fixture) in the Schrodinger
    picture with the given cutoffs, as its gradient test builds it (tests/test_infinite_cutoff.py:72-105,
    tests/test_only_rotate_k.py:32)."""
    g = golden.load(fixture)
    wl = golden.fixture_workload(g, fixture)
    extra = {**wl.extra, "schrodinger_cutoff": sc}
    if k is not None:
        extra["only_rotate_len_k"] = k
    return dataclasses.replace(wl, cutoff=cutoff, extra=extra), wl.n_layers


def _schr_line20(L: int):
    wl = W.line20()
    return dataclasses.replace(wl, extra={**wl.extra, "schrodinger_cutoff": 4}), L


#: frozen graphs in the Schrodinger picture: name -> zero-argument builder of (workload, layers)
GRAPHS_SCHR = {
    "ref_lih_fermionic_spin_exact_c4_s6": lambda: _schr_fixture("ref_lih_fermionic_spin_exact", 4, 6),
    "ref_lih_fermionic_spin_exact_c6_s8_k4": lambda: _schr_fixture("ref_lih_fermionic_spin_exact", 6, 8, 4),
    "line20_L200_s4": lambda: _schr_line20(200),
}


def graphs_schrodinger() -> None:
    """graph_<name>.npz for graphs built in the Schrodinger picture (schrodinger_cutoff, the replay from the
    dense reference state, MonomialPropagator.inl:1053-1097): the reference's replay at the build parameters
    and at shifted ones (seed 77, 0.05 N(0, 1)) with its gradient there, plus central finite differences
    (h = 1e-5) of the replay on up to 16 seeded parameters whose gradient is not zero."""
    for name, make in GRAPHS_SCHR.items():
        wl, L = make()
        eng = oracle.RefEngine(wl)
        eng.propagate(n_layers=L, build_graph=True)
        n_params = int(wl.param_map[:L].max()) + 1
        theta = wl.params[:n_params]
        shifted = theta + 0.05 * np.random.default_rng(77).standard_normal(n_params)
        ev, grad, _ = eng.expectation_and_gradient(shifted)
        ev0 = eng.expectation(theta)
        live = np.flatnonzero(np.abs(grad) > 1e-9)
        idx = np.sort(np.random.default_rng(5).choice(live, size=min(16, live.size), replace=False))
        h = 1e-5
        fd = np.zeros(idx.size)
        for j, p in enumerate(idx):
            tp, tm = shifted.copy(), shifted.copy()
            tp[p] += h
            tm[p] -= h
            fd[j] = (eng.expectation(tp) - eng.expectation(tm)) / (2 * h)
        size = eng.size()
        eng.close()
        extra = {}
        if wl.extra.get("only_rotate_len_k") is not None:
            extra["only_rotate_len_k"] = np.int64(wl.extra["only_rotate_len_k"])
        np.savez_compressed(os.path.join(HERE, f"graph_{name}.npz"), expectation=np.float64(ev),
                            expectation_build=np.float64(ev0), grad=grad, params=shifted, n_layers=np.int64(L),
                            schrodinger_cutoff=np.int64(wl.extra["schrodinger_cutoff"]),
                            cutoff=np.int64(wl.cutoff), terms=np.int64(size), fd_idx=idx, fd=fd, **extra)
        print("graph schrodinger", name, size, ev0, ev, f"{live.size}/{grad.size} nonzero",
              float(np.max(np.abs(grad[idx] - fd))) if idx.size else None, flush=True)


def surface(reference_root: str) -> None:
    """The names the reference's nanobind module binds per propagator class and module-wide
    (``src/monoprop/bindings/binder.h``, ``bindings.cpp.in``), and the ``_simulator`` attributes its Python
    front-end uses (``src/monoprop/*.py``): reference_surface.json, read by tests/test_core_surface.py."""
    import json
    import re

    bind = os.path.join(reference_root, "src", "monoprop", "bindings")
    with open(os.path.join(bind, "binder.h")) as f:
        binder = f.read()
    with open(os.path.join(bind, "bindings.cpp.in")) as f:
        module = f.read()
    calls = set()
    src = os.path.join(reference_root, "src", "monoprop")
    for name in sorted(os.listdir(src)):
        if name.endswith(".py"):
            with open(os.path.join(src, name)) as f:
                calls.update(re.findall(r"_simulator\.(\w+)", f.read()))
    out = {"class_members": sorted(set(re.findall(r"cls\.def\w*\(\s*\"(\w+)\"", binder))),
           "module_attributes": sorted(set(re.findall(r"m\.(?:attr|def)\(\s*\"(\w+)\"", module))),
           "frontend_simulator_calls": sorted(calls)}
    with open(os.path.join(HERE, "reference_surface.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("surface", {k: len(v) for k, v in out.items()})


def main(reference_root: str | None = None) -> None:
    reference_root = reference_root or os.environ.get("MONOPROP_REFERENCE")
    if not reference_root:
        raise SystemExit("give the reference source root as an argument or in $MONOPROP_REFERENCE")
    oracle.build(reference_root)
    if not oracle.ref_available():
        raise SystemExit("reference oracle could not be built")
    full = [a for a in sys.argv if a == "--full-depth" or a.startswith("--full-depth=")]
    if full:  # --full-depth (all) or --full-depth=name,name
        full_depth(full[0].split("=", 1)[1].split(",") if "=" in full[0] else None)
        return
    if "--surface" in sys.argv:
        surface(reference_root)
        return
    if "--graph-len-k" in sys.argv:
        graphs_len_k()
        return
    if "--graph-schrodinger" in sys.argv:
        graphs_schrodinger()
        return
    if "--graph-replay" in sys.argv:
        graph_replays()
        return
    for name, make, L, k in LEN_K:
        wl = make()
        wl = dataclasses.replace(wl, extra={**wl.extra, "only_rotate_len_k": k})
        r = oracle.run_ref(wl, n_layers=L)
        save_result(os.path.join(HERE, name + ".npz"), r.keys, r.coefs, r.expectation,
                    {"n_layers": np.int64(wl.n_layers if L is None else L), "only_rotate_len_k": np.int64(k)})
        print(name, r.keys.shape[0], r.expectation)
    for name in golden.SCHRODINGER:
        wl, L = golden.schrodinger_workload(name)
        r = oracle.run_ref(wl, n_layers=L)
        save_result(os.path.join(HERE, name + ".npz"), r.keys, r.coefs, r.expectation,
                    {"n_layers": np.int64(wl.n_layers if L is None else L)})
        print(name, r.keys.shape[0], r.expectation)
    for name in golden.BASIS_CHANGE:
        wl, L = golden.basis_change_workload(name)
        r = oracle.run_ref(wl, n_layers=L)
        save_result(os.path.join(HERE, name + ".npz"), r.keys, r.coefs, r.expectation,
                    {"n_layers": np.int64(wl.n_layers if L is None else L)})
        print(name, r.keys.shape[0], r.expectation)
    if "--len-k-only" in sys.argv:
        return
    for name, make, L in SEEDED:
        wl = make()
        r = oracle.run_ref(wl, n_layers=L)
        save_result(os.path.join(HERE, name + ".npz"), r.keys, r.coefs, r.expectation,
                    {"n_layers": np.int64(wl.n_layers if L is None else L)})
        print(name, r.keys.shape[0], r.expectation)
    for name, make, L in GRADS:
        wl = make()
        n_layers = wl.n_layers if L is None else L
        eng = oracle.RefEngine(wl, partitions=8 if name == "ising100" else 1)
        eng.propagate(n_layers=L, build_graph=True)
        n_params = int(wl.param_map[:n_layers].max()) + 1
        ev, grad, _ = eng.expectation_and_gradient(wl.params[:n_params])
        eng.close()
        np.savez_compressed(os.path.join(HERE, f"grad_{name}.npz"), expectation=np.float64(ev), grad=grad,
                            n_layers=np.int64(n_layers), n_params=np.int64(n_params))
        print("grad", name, ev, float(np.abs(grad).max()))
    if "--fd-full" in sys.argv:
        name, make, count, h, seed = FD_FULL
        wl = make()
        eng = oracle.RefEngine(wl, partitions=8)
        eng.propagate(build_graph=True)
        theta = wl.params.copy()
        idx = np.sort(np.random.default_rng(seed).choice(theta.size, size=count, replace=False))
        fd = np.zeros(count)
        for k, p in enumerate(idx):
            tp, tm = theta.copy(), theta.copy()
            tp[p] += h
            tm[p] -= h
            fd[k] = (eng.expectation(tp) - eng.expectation(tm)) / (2 * h)
        ev0 = eng.expectation(theta)
        eng.close()
        np.savez_compressed(os.path.join(HERE, f"fd_{name}.npz"), expectation=np.float64(ev0), idx=idx, fd=fd,
                            h=np.float64(h))
        print("fd", name, ev0, float(np.abs(fd).max()))
    # Frozen-structure replay at new parameters: the reference's graph built at the workload's parameters,
    # then expectation_value_and_gradient at theta' = theta + 0.05 * N(0, 1) (seed 77): graph_<name>.npz.
    for name, make, L in GRAPHS:
        wl = make()
        n_layers = wl.n_layers if L is None else L
        eng = oracle.RefEngine(wl)
        eng.propagate(n_layers=L, build_graph=True)
        n_params = int(wl.param_map[:n_layers].max()) + 1
        theta = wl.params[:n_params]
        shifted = theta + 0.05 * np.random.default_rng(77).standard_normal(n_params)
        ev, grad, _ = eng.expectation_and_gradient(shifted)
        ev0 = eng.expectation(theta)
        eng.close()
        np.savez_compressed(os.path.join(HERE, f"graph_{name}.npz"), expectation=np.float64(ev),
                            expectation_build=np.float64(ev0), grad=grad, params=shifted, n_layers=np.int64(n_layers))
        print("graph", name, ev0, ev, float(np.abs(grad).max()))
    # Parameter-shift gradient of the 20-qubit line circuit from the reference's replayed graph: each
    # replayed layer is affine in (cos 2 g theta, sin 2 g theta), so E(theta + s e_p) - E(theta - s e_p)
    # with s = pi / (4 |g|) times |g| is the exact derivative of the frozen surrogate (one layer per
    # parameter here).
    wl = W.line20()
    eng = oracle.RefEngine(wl)
    eng.propagate(build_graph=True)
    theta = wl.params.copy()
    ps = np.zeros_like(theta)
    for p in range(theta.size):
        g = abs(float(wl.gen_coeffs[p]))
        s = np.pi / (4 * g)
        tp, tm = theta.copy(), theta.copy()
        tp[p] += s
        tm[p] -= s
        ps[p] = g * (eng.expectation(tp) - eng.expectation(tm))
    ev0 = eng.expectation(theta)
    eng.close()
    np.savez_compressed(os.path.join(HERE, "pshift_line20.npz"), expectation=np.float64(ev0), grad=ps)
    print("pshift line20", ev0, float(np.abs(ps).max()))
    for case in REF_CASES:
        for tag, la in (("", None), ("_atol1e-10", 1e-10)):
            wl, exact, grad = fixture_workload(case, reference_root, la)
            r = oracle.run_ref(wl)
            enc_keys, enc_coefs, core = wl.encoded_observable()
            flat = np.asarray([s for m in wl.gate_slots for s in m], dtype=np.int64)
            off = np.cumsum([0] + [len(m) for m in wl.gate_slots]).astype(np.int64)
            save_result(os.path.join(HERE, f"ref_{case}{tag}.npz"), r.keys, r.coefs, r.expectation,
                        {"exact_energy": np.float64(exact), "exact_gradient": grad,
                         "num_modes": np.int64(wl.num_modes), "gate_slots_flat": flat, "gate_slots_off": off,
                         "gen_coeffs": wl.gen_coeffs, "param_map": wl.param_map, "params": wl.params,
                         "obs_keys": enc_keys, "obs_coefs": enc_coefs, "core": np.float64(core),
                         "state_mask": wl.state_mask(), "initial_state": np.asarray(wl.initial_state, np.int64),
                         "cutoff": np.int64(wl.cutoff),
                         "lower_atol": np.float64(np.nan if la is None else la)})
            print(case + tag, r.keys.shape[0], r.expectation, exact)


if __name__ == "__main__":
    main(*[a for a in sys.argv[1:] if not a.startswith("--")])
