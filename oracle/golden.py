"""Loading the golden fixtures of ``tests/golden/`` (test infrastructure, like the rest of ``oracle``)."""

from __future__ import annotations

import hashlib
import os

import numpy as np

from monoprop_b200.encoding import canonical_order, words_to_slots
from monoprop_b200 import workloads as W
from monoprop_b200.workloads import Workload

GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")

SEEDED = ["line20", "line20_L200", "hubbard6x6_L400", "ising100_L600", "ising50_d2", "ising50_d3", "ising100_L1200"]
#: seeded workloads propagated with only_rotate_len_k: name -> (base workload name, layers, k)
LEN_K = {"line20_k6": ("line20", None, 6), "hubbard6x6_L400_k4": ("hubbard6x6", 400, 4),
         "ising50_d3_k8": ("ising50_d3", None, 8)}
REF_CASES = [f"ref_{c}{t}" for c in ("rx_rz_ry_rz_exact", "random_exact", "lih_fermionic_spin_exact")
             for t in ("", "_atol1e-10")]


#: seeded Majorana workloads with a basis_change: name -> (base workload name, layers, basis pattern)
BASIS_CHANGE = {"hubbard6x6_L400_bcjw": ("hubbard6x6", 400, "jw"),
                "hubbard6x6_L400_bcrand": ("hubbard6x6", 400, "rand")}


def basis_pattern(kind: str, num_modes: int, seed: int = 7) -> list[list[int]]:
    """basis_change rows: "jw" maps slot 2q to {2q} and 2q+1 to {2q, 2q+1}; "perm" is a seeded slot
    permutation; "rand" gives each slot a seeded random monomial of 1 to 3 slots."""
    rng = np.random.default_rng(seed)
    if kind == "jw":
        return [[s] if s % 2 == 0 else [s - 1, s] for s in range(2 * num_modes)]
    if kind == "perm":
        p = rng.permutation(2 * num_modes)
        return [[int(p[s])] for s in range(2 * num_modes)]
    return [sorted(set(int(x) for x in rng.choice(2 * num_modes, size=int(rng.integers(1, 4)), replace=False)))
            for _ in range(2 * num_modes)]


def basis_change_workload(name: str):
    """(workload with basis_change set, layers) of the ``BASIS_CHANGE`` fixture ``name``."""
    import dataclasses

    from monoprop_b200 import workloads as W

    base, L, kind = BASIS_CHANGE[name]
    wl = {"hubbard6x6": W.hubbard6x6}[base]()
    return dataclasses.replace(wl, extra={**wl.extra, "basis_change": basis_pattern(kind, wl.num_modes)}), L


#: seeded workloads in the Schrodinger picture: name -> (base workload name, layers, schrodinger_cutoff)
SCHRODINGER = {"line20_L100_s4": ("line20", 100, 4), "hubbard6x6_L200_s4": ("hubbard6x6", 200, 4)}


def schrodinger_workload(name: str):
    """(workload with schrodinger_cutoff set, layers) of the ``SCHRODINGER`` fixture ``name``."""
    import dataclasses

    from monoprop_b200 import workloads as W

    base, L, sc = SCHRODINGER[name]
    wl = {"line20": W.line20, "hubbard6x6": W.hubbard6x6}[base]()
    return dataclasses.replace(wl, extra={**wl.extra, "schrodinger_cutoff": sc}), L


def len_k_workload(name: str):
    """(workload with only_rotate_len_k set, layers) of the ``LEN_K`` fixture ``name``."""
    import dataclasses

    from monoprop_b200 import workloads as W

    base, L, k = LEN_K[name]
    make = {"line20": W.line20, "hubbard6x6": W.hubbard6x6, "ising50_d3": lambda: W.ising50(3)}[base]
    wl = make()
    return dataclasses.replace(wl, extra={**wl.extra, "only_rotate_len_k": k}), L


def load(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def fixture_workload(g: dict, name: str = "fixture") -> Workload:
    """Majorana workload stored in a ``ref_*`` fixture (engine arrays, infinite cutoff)."""
    n = int(g["num_modes"])
    off, flat = g["gate_slots_off"], g["gate_slots_flat"]
    slots = [tuple(int(s) for s in flat[off[i]:off[i + 1]]) for i in range(len(off) - 1)]
    obs = {}
    for k, c in zip(g["obs_keys"], g["obs_coefs"]):
        mono = words_to_slots(k, n)
        w = len(mono)
        obs[mono] = complex(c) * (1j) ** ((w * (w - 1) // 2) % 4)  # decode back to the operator's coefficient
    if float(g["core"]) != 0.0:
        obs[()] = complex(float(g["core"]))
    la = float(g["lower_atol"])
    return Workload(name, "majorana", n, slots, g["gen_coeffs"], g["param_map"], g["params"], obs,
                    [int(i) for i in g["initial_state"]], int(g["cutoff"]), "length", None if np.isnan(la) else la)


def check_against(g: dict, keys: np.ndarray, coefs: np.ndarray, ev: float, rtol: float = 1e-10) -> None:
    """Asserts that (keys, coefs, ev) equal the golden result: keys bit-exact, coefficients and <O> within rtol."""
    order = canonical_order(keys)
    k, c = np.ascontiguousarray(keys[order]), coefs[order]
    assert k.shape[0] == int(g["n"]), (k.shape[0], int(g["n"]))
    assert hashlib.sha256(k.tobytes()).hexdigest() == g["sha256"].item().decode(), "monomial set differs"
    if "keys" in g:
        assert np.array_equal(k, g["keys"])
        tol = rtol * np.maximum(np.abs(c), np.abs(g["coefs"])) + 1e-15
        assert np.all(np.abs(c - g["coefs"]) <= tol), float(np.max(np.abs(c - g["coefs"])))
    else:
        assert abs(c.sum() - float(g["coef_sum"])) <= rtol * max(1.0, float(np.abs(c).sum()))
        assert abs((c * c).sum() - float(g["coef_sumsq"])) <= rtol * max(1.0, float((c * c).sum()))
    e = float(g["expectation"])
    assert abs(ev - e) <= rtol * max(1.0, abs(e)), (ev, e)


def _batch_instance(depth: int):
    """The first instance of the 256-instance batched workload with ``depth`` layers."""
    return next(wl for wl in W.batch_ising50(256) if wl.extra["depth"] == depth)


def _line20_schrodinger():
    """The full 20-qubit line circuit in the Schrodinger picture, schrodinger_cutoff 4 (6.4e7 final terms)."""
    import dataclasses

    wl = W.line20()
    return dataclasses.replace(wl, extra={**wl.extra, "schrodinger_cutoff": 4})


#: full-depth workloads whose final stores are too large to keep in full (up to ~6.4e7 terms): only a
#: bucketed digest is committed (``full_<name>.npz``). name -> zero-argument workload builder.
FULL_DEPTH = {
    "ising100": W.ising100,
    "hubbard6x6": W.hubbard6x6,
    "ising50_b24": lambda: _batch_instance(24),
    "ising50_b12": lambda: _batch_instance(12),
    "line20_s4": _line20_schrodinger,
}

DIGEST_BUCKETS = 2048
DIGEST_TOP = 4096


def _mix64(x: np.ndarray) -> np.ndarray:
    """The splitmix64 finaliser on a uint64 array (wrapping arithmetic)."""
    x = x.copy()
    x ^= x >> np.uint64(30)
    x *= np.uint64(0xBF58476D1CE4E5B9)
    x ^= x >> np.uint64(27)
    x *= np.uint64(0x94D049BB133111EB)
    x ^= x >> np.uint64(31)
    return x


def key_hashes(keys: np.ndarray) -> np.ndarray:
    """A 64-bit hash of every key row (``uint64[n, W]`` -> ``uint64[n]``)."""
    h = np.zeros(keys.shape[0], dtype=np.uint64)
    with np.errstate(over="ignore"):
        for w in range(keys.shape[1]):
            h ^= _mix64(keys[:, w] + np.uint64(w))
    return h


def _unit(h: np.ndarray) -> np.ndarray:
    """Pseudo-random weights in [-1, 1) from 64-bit hashes."""
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 ** -52) - 1.0


def bucket_digest(keys: np.ndarray, coefs: np.ndarray, buckets: int = DIGEST_BUCKETS, top: int = DIGEST_TOP) -> dict:
    """Size-independent digest of a raw store that still bounds every single coefficient.

    Keys are sorted canonically; the key set is its SHA-256. Each key falls into one of ``buckets``
    buckets by its hash and carries two pseudo-random weights w1, w2 in [-1, 1) from the hash; per
    bucket the digest keeps the term count, sum |c|, sum c*w1 and sum c*w2 (summed in canonical key
    order, so equal inputs give equal bits). If every coefficient agrees to ``rtol`` relative, every
    projected sum agrees to ``rtol * sum |c|`` of its bucket; a single term off by more than that shows
    up in both projections unless its weights vanish. The ``top`` largest coefficients are also kept
    with their canonical positions, for a direct per-term comparison, and the SHA-256 of all coefficient
    bits in key order records whether two stores are bit-identical."""
    order = canonical_order(keys)
    k, c = np.ascontiguousarray(keys[order]), np.ascontiguousarray(coefs[order])
    h = key_hashes(k)
    b = (h % np.uint64(buckets)).astype(np.int64)
    with np.errstate(over="ignore"):
        w1, w2 = _unit(h), _unit(_mix64(h ^ np.uint64(0x9E3779B97F4A7C15)))
    a = np.abs(c)
    t = min(top, c.shape[0])
    pos = np.sort(np.argpartition(-a, t - 1)[:t]) if t > 0 else np.zeros(0, dtype=np.int64)
    return {"n": np.int64(k.shape[0]), "sha256": np.bytes_(hashlib.sha256(k.tobytes()).hexdigest()),
            "coef_sha256": np.bytes_(hashlib.sha256(c.tobytes()).hexdigest()),
            "b_count": np.bincount(b, minlength=buckets).astype(np.int64),
            "b_abs": np.bincount(b, weights=a, minlength=buckets),
            "b_w1": np.bincount(b, weights=c * w1, minlength=buckets),
            "b_w2": np.bincount(b, weights=c * w2, minlength=buckets),
            "top_pos": pos.astype(np.int64), "top_keys": k[pos], "top_coefs": c[pos]}


def check_digest(g: dict, keys: np.ndarray, coefs: np.ndarray, ev: float, rtol: float = 1e-10) -> bool:
    """Asserts (keys, coefs, ev) against a :func:`bucket_digest` fixture: key set bit-exact, per-bucket
    projections within ``rtol`` of the bucket's sum |c|, the largest coefficients within ``rtol`` relative,
    <O> within ``rtol`` relative. Returns whether the coefficients are bit-identical to the fixture's."""
    d = bucket_digest(keys, coefs, buckets=int(g["b_count"].shape[0]), top=0)
    assert int(d["n"]) == int(g["n"]), (int(d["n"]), int(g["n"]))
    assert d["sha256"].item() == g["sha256"].item(), "monomial set differs"
    assert np.array_equal(d["b_count"], g["b_count"])
    bound = rtol * np.maximum(d["b_abs"], g["b_abs"]) + 1e-300
    for name in ("b_w1", "b_w2"):
        err = np.abs(d[name] - g[name])
        assert np.all(err <= bound), (name, float(np.max(err / bound)))
    order = canonical_order(keys)
    pos = g["top_pos"]
    k = keys[order[pos]]
    c = coefs[order[pos]]
    assert np.array_equal(k, g["top_keys"])
    tc = g["top_coefs"]
    assert np.all(np.abs(c - tc) <= rtol * np.maximum(np.abs(c), np.abs(tc)) + 1e-300)
    e = float(g["expectation"])
    assert abs(ev - e) <= rtol * max(1.0, abs(e)), (ev, e)
    return d["coef_sha256"].item() == g["coef_sha256"].item()


def random_workload(seed: int, basis: str) -> Workload:
    """Random circuit on few modes with truncation active (small cutoffs, both atols)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(3, 7))
    L = int(rng.integers(10, 60))
    slots = []
    for _ in range(L):
        w = int(rng.integers(1, 5))
        slots.append(tuple(sorted(rng.choice(2 * n, size=w, replace=False).tolist())))
    g = rng.choice([-1.0, -0.5, 0.5, 1.0], size=L)
    params = rng.uniform(-np.pi, np.pi, size=L)
    j = int(rng.integers(0, L))
    params[j] = np.pi / 4 / abs(g[j])  # cos(2 angle) ~ 6e-17: the partner value stored/cos is ill-conditioned
    obs = {tuple(sorted(rng.choice(2 * n, size=2, replace=False).tolist())): 1.0 + 0j for _ in range(3)}
    if basis == "pauli":
        return Workload(f"rand_pauli_{seed}", "pauli", n, slots, g, np.arange(L), params,
                          {k: complex(abs(v)) for k, v in obs.items()}, [0] if n > 1 else [], int(rng.integers(1, 3)),
                          "support", float(rng.choice([1e-3, 1e-2])), float(rng.choice([0.05, 0.2])))
    obs = {k: (1j if len(k) % 4 in (2, 3) else 1.0) for k in obs}
    return Workload(f"rand_maj_{seed}", "majorana", n, slots, g, np.arange(L), params, obs,
                      list(range(0, n, 2)), int(rng.integers(2, 5)), str(rng.choice(["length", "support"])),
                      float(rng.choice([1e-3, 1e-2])), float(rng.choice([0.05, 0.2])))
