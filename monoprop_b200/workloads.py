"""Seeded synthetic circuits for the benchmark and parity workloads.

Each builder returns a :class:`Workload`: the engine-level per-monomial arrays that the reference's
``expand_monomials`` (``src/monoprop/circuit.py:573-605``) produces, plus the observable, the reference
state and the truncation settings. Angles come from ``numpy.random.default_rng(seed)`` in gate order.

Qiskit-convention rotations ``RZZ(t)`` / ``RX(t)`` are ``exp(-i t P / 2)``, i.e. the ``exp(+i t g P)``
gate with ``g = -0.5`` (``src/monoprop/qiskit_conversion.py``).

Workloads (sizes, value distributions and truncation as specified for the hot path):

* ``line20``   -- 20-qubit line, 10 layers of RZZ on the 19 nearest-neighbour pairs then RX on every
  qubit (390 gates), theta ~ U[0, pi); observable Z_10; Pauli weight <= 8, lower_atol 1e-4.
* ``ising100`` -- 10x10 kicked Ising, 20 layers of RZZ on the 180 lattice edges (the 90 horizontal edges
  row-major, then the 90 vertical edges) then RX on the 100 sites (5600 gates), theta ~ U[0, 0.3 pi);
  observable (1/100) sum_i Z_i; Pauli weight <= 10, lower_atol 1e-5.
* ``hubbard6x6`` -- spinful Fermi-Hubbard on a 6x6 open lattice (72 modes, mode ``2s + spin``), 8 Trotter
  steps; per step and per bond (a, b) and spin, one gate of the two hopping monomials ``{2a, 2b+1}``
  (g=+1) and ``{2a+1, 2b}`` (g=-1) sharing an angle ~ N(0.1, 0.02); then 36 on-site weight-4 gates
  ``{4s..4s+3}`` (g=+1) with angles ~ N(0.4, 0.05); observable (1 + i m0 m1)/2; Majorana length <= 8,
  lower_atol 1e-5; reference state one electron per site, spin alternating (mode ``2s + s % 2``).
* ``ising50(depth)`` -- 5x10 kicked Ising (85 edges, 50 sites), ``depth`` layers, theta ~ U[0, 0.3 pi);
  observable Z_i; Pauli weight <= 8, lower_atol 1e-5 (one instance of the batched workload).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .encoding import encode_many, state_mask_words, words_for


@dataclass
class Workload:
    """Engine-level arrays for one propagation problem (circuit order, Heisenberg applies last first)."""

    name: str
    basis: str  # "pauli" | "majorana"
    num_modes: int  # qubits for Pauli, fermionic modes for Majorana
    gate_slots: list[tuple[int, ...]]  # one monomial per layer
    gen_coeffs: np.ndarray  # float64[L]
    param_map: np.ndarray  # int64[L]
    params: np.ndarray  # float64[P]
    observable: dict[tuple[int, ...], complex]  # slot tuple -> coefficient (engine encoding)
    initial_state: list[int]
    cutoff: int
    cutoff_type: str  # "support" | "length"
    lower_atol: float | None
    upper_atol: float | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n_layers(self) -> int:
        return len(self.gate_slots)

    @property
    def words(self) -> int:
        return words_for(self.num_modes)

    def gen_words(self) -> np.ndarray:
        return encode_many(self.gate_slots, self.num_modes)

    def angles(self, params: np.ndarray | None = None) -> np.ndarray:
        """Per-layer mapped angle ``theta[map[l]] * g[l]`` (``MPFunctions.cpp:57-69``)."""
        p = self.params if params is None else np.asarray(params, dtype=np.float64)
        return p[self.param_map] * self.gen_coeffs

    def encoded_observable(self) -> tuple[np.ndarray, np.ndarray, float]:
        """(keys uint64[n, W], encoded real coefficients float64[n], core term).

        Terms are ordered by their slot tuples, the iteration order of the reference's
        ``std::map`` initial operator (``MonomialPropagator.inl:147-160``).
        """
        keys, coefs, core = [], [], 0.0
        for slots in sorted(self.observable):
            c = complex(self.observable[slots])
            enc = encode_coefficient(self.basis, slots, c)
            if len(slots) == 0:
                core = enc
                continue
            keys.append(slots)
            coefs.append(enc)
        return encode_many(keys, self.num_modes), np.asarray(coefs, dtype=np.float64), core

    def state_mask(self) -> np.ndarray:
        return state_mask_words(self.initial_state, self.num_modes)


def encode_coefficient(basis: str, slots: tuple[int, ...], coeff: complex) -> float:
    """Real engine coefficient of an observable term.

    Pauli: the real part; a non-negligible imaginary part is rejected
    (``algebra/PauliAlgebra.h:150-155``). Majorana: ``coeff / i^{C(|M|,2)}`` must be real
    (``algebra/MajoranaAlgebra.h:162-171``).
    """
    if basis == "pauli":
        if abs(coeff.imag) > 1e-10:
            raise RuntimeError("Non-real Pauli coeffs detected")
        return float(coeff.real)
    w = len(slots)
    enc = coeff / (1j ** ((w * (w - 1) // 2) % 4))
    if abs(enc.imag) > 1e-10:
        raise RuntimeError("Non-Hermitian coeffs detected")
    return float(enc.real)


def _zz(a: int, b: int) -> tuple[int, ...]:
    return tuple(sorted((2 * a, 2 * a + 1, 2 * b, 2 * b + 1)))


def _x(q: int) -> tuple[int, ...]:
    return (2 * q,)


def kicked_ising(nx: int, ny: int, layers: int, seed: int, theta_max: float,
                 edges: list[tuple[int, int]] | None = None) -> tuple[list, np.ndarray, np.ndarray, np.ndarray]:
    """RZZ on every edge, then RX on every site, per layer; one independent angle per gate."""
    n = nx * ny
    if edges is None:
        edges = [(r * nx + c, r * nx + c + 1) for r in range(ny) for c in range(nx - 1)]
        edges += [(r * nx + c, (r + 1) * nx + c) for r in range(ny - 1) for c in range(nx)]
    slots: list[tuple[int, ...]] = []
    for _ in range(layers):
        slots += [_zz(a, b) for a, b in edges]
        slots += [_x(q) for q in range(n)]
    rng = np.random.default_rng(seed)
    params = rng.uniform(0.0, theta_max, size=len(slots))
    g = np.full(len(slots), -0.5)
    pmap = np.arange(len(slots), dtype=np.int64)
    return slots, g, pmap, params


def _per_layer(edges_n: int, sites: int) -> dict:
    return {"gates_per_layer": edges_n + sites}


def line20(seed: int = 1234, layers: int = 10) -> Workload:
    n = 20
    edges = [(i, i + 1) for i in range(n - 1)]
    slots, g, pmap, params = kicked_ising(n, 1, layers, seed, np.pi, edges)
    return Workload("line20", "pauli", n, slots, g, pmap, params, {(20, 21): 1.0 + 0j}, [], 8, "support", 1e-4,
                    extra=_per_layer(n - 1, n))


def ising100(seed: int = 1234, layers: int = 20) -> Workload:
    slots, g, pmap, params = kicked_ising(10, 10, layers, seed, 0.3 * np.pi)
    obs = {(2 * i, 2 * i + 1): 0.01 + 0j for i in range(100)}
    return Workload("ising100", "pauli", 100, slots, g, pmap, params, obs, [], 10, "support", 1e-5,
                    extra=_per_layer(180, 100))


def ising50(depth: int, seed: int = 99, observable_qubit: int | None = None) -> Workload:
    slots, g, pmap, params = kicked_ising(10, 5, depth, seed, 0.3 * np.pi)
    q = observable_qubit if observable_qubit is not None else int(np.random.default_rng(seed + 1).integers(0, 50))
    obs = {(2 * q, 2 * q + 1): 1.0 + 0j}
    return Workload(f"ising50_d{depth}", "pauli", 50, slots, g, pmap, params, obs, [], 8, "support", 1e-5,
                    extra={"observable_qubit": q, "depth": depth, **_per_layer(85, 50)})


def hubbard6x6(seed: int = 7, steps: int = 8, lx: int = 6, ly: int = 6) -> Workload:
    sites = lx * ly
    bonds = [(y * lx + x, y * lx + x + 1) for y in range(ly) for x in range(lx - 1)]
    bonds += [(y * lx + x, (y + 1) * lx + x) for y in range(ly - 1) for x in range(lx)]
    rng = np.random.default_rng(seed)
    slots: list[tuple[int, ...]] = []
    g: list[float] = []
    pmap: list[int] = []
    params: list[float] = []
    for _ in range(steps):
        for a_site, b_site in bonds:
            for spin in (0, 1):
                a, b = 2 * a_site + spin, 2 * b_site + spin
                p = len(params)
                params.append(float(rng.normal(0.1, 0.02)))
                slots += [tuple(sorted((2 * a, 2 * b + 1))), tuple(sorted((2 * a + 1, 2 * b)))]
                g += [1.0, -1.0]
                pmap += [p, p]
        for s in range(sites):
            p = len(params)
            params.append(float(rng.normal(0.4, 0.05)))
            slots.append((4 * s, 4 * s + 1, 4 * s + 2, 4 * s + 3))
            g.append(1.0)
            pmap.append(p)
    obs = {(): 0.5 + 0j, (0, 1): 0.5j}
    state = [2 * s + (s % 2) for s in range(sites)]
    return Workload("hubbard6x6", "majorana", 2 * sites, slots, np.asarray(g), np.asarray(pmap, dtype=np.int64),
                    np.asarray(params), obs, state, 8, "length", 1e-5,
                    extra={"gates_per_layer": 2 * 2 * len(bonds) + sites})


def batch_ising50(n_instances: int = 256, seed: int = 99, min_depth: int = 4, max_depth: int = 24) -> list[Workload]:
    """The batched workload: independent 5x10 kicked-Ising instances of seeded uneven depth."""
    rng = np.random.default_rng(seed)
    depths = rng.integers(min_depth, max_depth + 1, size=n_instances)
    qubits = rng.integers(0, 50, size=n_instances)
    return [ising50(int(d), seed=seed * 1000 + i, observable_qubit=int(q)) for i, (d, q) in enumerate(zip(depths, qubits))]


BY_NAME = {"line20": line20, "ising100": ising100, "hubbard6x6": hubbard6x6}

#: sum over gates of the terms present when the gate is applied (term-gate updates) for the default
#: seeds, as counted by the oracle and the reference engine; the GPU engine's per-gate counters must sum
#: to the same numbers (tests/test_gpu_parity.py). The reference's timing arm divides by these.
TERM_GATE_UPDATES = {"line20": 694_230, "hubbard6x6": 3_416_554_382, "ising100": 107_553_458_845}


def from_circuit(name: str, operator, circuit, *, cutoff: int, cutoff_type: str = "length",
                 lower_atol: float | None = None, upper_atol: float | None = None) -> Workload:
    """Workload of a front-end circuit and observable (``PauliOperator`` or ``MajoranaOperator``).

    The gate expansion is :func:`monoprop_b200.circuit.expand_monomials` (the reference's
    ``expand_monomials``); a ``PauliOperator`` observable is taken in the native Pauli slot encoding.
    """
    from .circuit import expand_monomials
    from .operators import PauliOperator

    if isinstance(operator, PauliOperator):
        basis, terms, n = "pauli", operator.get_local_operator().terms, operator.num_qubits
    else:
        basis, terms, n = "majorana", operator.get_majorana_operator().terms, operator.num_modes
    monos, g, pmap, _ = expand_monomials(circuit.gates, circuit.resolved_mapping, n)
    params = np.asarray(circuit.parameters, dtype=np.float64)
    return Workload(name, basis, n, [tuple(m) for m in monos], np.asarray(g, dtype=np.float64),
                    np.asarray(pmap, dtype=np.int64), params, dict(terms), list(circuit.initial_state), cutoff,
                    cutoff_type, lower_atol, upper_atol)
