"""Circuits of exponential gates and their expansion into the engine's per-monomial arrays.

Public surface and conventions of the reference's ``src/monoprop/circuit.py``:

* ``ExpGate(generator, index=None, atol=1e-8)`` applies ``exp(+i theta H)`` for a Hermitian generator
  ``H`` (a ``PauliOperator`` or ``MajoranaOperator``); terms with ``|c| <= atol`` are dropped and the
  remaining terms must pairwise commute (``circuit.py:71-127``).
* ``Circuit(gates, system_size, parameters=(), initial_state=None)``: with no gate ``index`` set, gate i
  drives angle i; otherwise every gate sets an index and the indices are contiguous ``0..n-1``
  (``circuit.py:208-347``).
* ``expand_monomials`` flattens gates to ``(monomials, gen_coeffs, mapping, gate_indices)``
  (``circuit.py:573-605``): a Pauli term keeps its real coefficient on its native slots; a Majorana
  term's coefficient is divided by ``i^{C(w,2)}`` and negated (``circuit.py:525-534``) unless the gate
  came from the dense wire format, whose coefficients already are the engine's ``g``.
"""

from __future__ import annotations

from collections.abc import Sequence

from .operators import MajoranaOperator, PauliOperator

_HERMITICITY_ATOL = 1e-9


def _real_coefficient(mono, value) -> float:
    value = complex(value)
    if abs(value.imag) > _HERMITICITY_ATOL:
        raise ValueError(f"Gate generator is not Hermitian: monomial {tuple(mono)} yields the structural generator "
                         f"coefficient {value}, whose imaginary part is not negligible.")
    return float(value.real)


class ExpGate:
    """``exp(+i theta H)`` for a Hermitian generator ``H``; ``index`` selects the driving angle."""

    __slots__ = ("_atol", "_structural", "family", "generator", "index")

    def __init__(self, generator, index: int | None = None, *, atol: float = 1e-8, _structural: bool = False):
        if isinstance(generator, PauliOperator):
            family = "pauli"
            gen = PauliOperator({p: c for p, c in generator.terms.items() if abs(c) > atol}, generator.num_qubits)
        elif isinstance(generator, MajoranaOperator) or hasattr(generator, "get_majorana_operator"):
            generator = generator.get_majorana_operator()
            family = "majorana"
            gen = MajoranaOperator({m: c for m, c in generator.terms.items() if abs(c) > atol}, generator.num_modes)
        else:
            raise TypeError("ExpGate generator must be a MajoranaOperator, PauliOperator, or FermiOperator "
                            f"(an operator object carrying its mode/qubit count), not a bare term; got "
                            f"{type(generator).__name__}.")
        if not gen.all_pairwise_commute():
            raise ValueError("The provided generator must be composed of commuting terms.")
        self.generator = gen
        self.index = None if index is None else int(index)
        self.family = family
        self._atol = atol
        self._structural = _structural

    @property
    def system_size(self) -> int:
        g = self.generator
        return g.num_qubits if isinstance(g, PauliOperator) else g.num_modes

    def layers(self) -> list[tuple[tuple[int, ...], float]]:
        """(engine monomial, engine generator coefficient g) per term, in application order."""
        g = self.generator
        if isinstance(g, PauliOperator):
            for p in g.terms:
                if p.qubits and p.qubits[-1] >= g.num_qubits:
                    raise ValueError(f"Gate generator term {p} acts on a qubit index >= the system's "
                                     f"num_qubits={g.num_qubits}.")
            return [(p.slots(), _real_coefficient(p.slots(), c)) for p, c in g.terms.items()]
        if self._structural:
            return [(m, _real_coefficient(m, c)) for m, c in g.terms.items()]
        out = []
        for m, c in g.terms.items():
            w = len(m)
            out.append((m, _real_coefficient(m, -complex(c) / (1j) ** ((w * (w - 1) // 2) % 4))))
        return out

    def __eq__(self, other) -> bool:
        if not isinstance(other, ExpGate):
            return NotImplemented
        return (self.generator == other.generator and self.index == other.index and self.family == other.family
                and self._structural == other._structural)

    __hash__ = None

    def __repr__(self) -> str:
        return f"ExpGate({self.generator}, index={self.index})"


def _identity(gate: ExpGate) -> bool:
    return len(gate.generator.terms) == 0


class Circuit:
    """An ordered sequence of :class:`ExpGate` with optional bound angles and a reference state."""

    def __init__(self, gates: Sequence[ExpGate], system_size: int, parameters: Sequence[float] = (),
                 initial_state: Sequence[int] | None = None) -> None:
        gates = tuple(gates)
        parameters = tuple(float(v) for v in parameters)
        self._state_given = initial_state is not None
        initial_state = tuple(int(i) for i in initial_state or ())
        if isinstance(system_size, bool) or not isinstance(system_size, int) or system_size < 0:
            raise ValueError(f"system_size must be a non-negative integer; got {system_size!r}.")
        if len(set(initial_state)) != len(initial_state):
            raise ValueError("Duplicate indices in initial state")
        if any(i < 0 or i >= system_size for i in initial_state):
            raise ValueError(f"initial_state entries must be in 0..{system_size - 1}; got {list(initial_state)}.")
        for g in gates:
            if not isinstance(g, ExpGate):
                raise TypeError(f"Circuit gates must be ExpGate; got {type(g).__name__}.")
            if g.system_size != system_size:
                raise ValueError(f"Gate generator width {g.system_size} does not match circuit "
                                 f"system_size={system_size}.")
        if all(g.index is None for g in gates) and any(_identity(g) for g in gates):
            if parameters and len(parameters) != len(gates):
                raise ValueError(f"parameters has {len(parameters)} values but the circuit has {len(gates)} gates.")
            kept = [i for i, g in enumerate(gates) if not _identity(g)]
            parameters = tuple(parameters[i] for i in kept) if parameters else ()
            gates = tuple(gates[i] for i in kept)
        self.gates = gates
        self.parameters = parameters
        self.initial_state = initial_state
        self.system_size = system_size
        fams = {g.family for g in gates}
        if len(fams) > 1:
            raise TypeError("A circuit cannot mix qubit and Majorana/fermionic gates; build separate circuits per "
                            "family.")
        self.family = fams.pop() if fams else "empty"
        _ = self.resolved_mapping
        if self.parameters and len(self.parameters) != self.n_parameters:
            raise ValueError(f"parameters has {len(self.parameters)} values but the circuit has {self.n_parameters} "
                             "parameters.")

    @property
    def resolved_mapping(self) -> tuple[int, ...]:
        idx = [g.index for g in self.gates]
        if all(i is None for i in idx):
            return tuple(range(len(self.gates)))
        if any(i is None for i in idx):
            raise ValueError("Either every gate must set `index`, or none of them must (mixing an explicit index "
                             "with the default would be ambiguous).")
        mapping = tuple(int(i) for i in idx)
        validate_parameter_mapping(mapping, len(self.gates), "gates")
        return mapping

    @property
    def n_parameters(self) -> int:
        m = self.resolved_mapping
        return max(m) + 1 if m else 0

    def __len__(self) -> int:
        return len(self.gates)

    def __iter__(self):
        return iter(self.gates)

    def __add__(self, other: Circuit) -> Circuit:
        if not isinstance(other, Circuit):
            return NotImplemented
        if other.system_size != self.system_size:
            raise ValueError("Cannot concatenate circuits of different system_size.")
        if (self.parameters == ()) != (other.parameters == ()) and len(self) and len(other):
            raise ValueError("Cannot concatenate a bound circuit with an unbound one.")
        shift = self.n_parameters
        gates = [ExpGate(g.generator, m, atol=g._atol, _structural=g._structural)
                 for g, m in zip(self.gates, self.resolved_mapping)]
        gates += [ExpGate(g.generator, m + shift, atol=g._atol, _structural=g._structural)
                  for g, m in zip(other.gates, other.resolved_mapping)]
        state = self.initial_state if self._state_given else (other.initial_state if other._state_given else None)
        return Circuit(gates, self.system_size, self.parameters + other.parameters, state)

    @classmethod
    def from_dense_arrays(cls, majoranas: Sequence[Sequence[int]], gen_coeffs: Sequence[float],
                          param_inds: Sequence[int], system_size: int, parameters: Sequence[float] = (),
                          initial_state: Sequence[int] | None = None) -> Circuit:
        """Majorana circuit from the flat wire format: consecutive monomials sharing a parameter index form
        one gate whose coefficients are already the engine's ``g`` (``circuit.py:407-478``)."""
        gates: list[ExpGate] = []
        run: list[tuple[int, ...]] = []
        coeffs: list[complex] = []
        cur = None
        for mono, c, p in zip(majoranas, gen_coeffs, param_inds, strict=True):
            p = int(p)
            if run and p != cur:
                gates.append(ExpGate(MajoranaOperator._from_terms(run, coeffs, system_size), cur, _structural=True))
                run, coeffs = [], []
            cur = p
            m = tuple(int(i) for i in mono)
            if any(i < 0 for i in m):
                raise ValueError(f"Majorana indices must be non-negative; got {m}.")
            if m and max(m) >= 2 * system_size:
                raise ValueError(f"Majorana term {m} acts on an index >= 2*system_size={2 * system_size}.")
            run.append(m)
            coeffs.append(complex(float(c)))
        if run:
            gates.append(ExpGate(MajoranaOperator._from_terms(run, coeffs, system_size), cur, _structural=True))
        return cls(tuple(gates), system_size, tuple(float(v) for v in parameters),
                   tuple(int(i) for i in initial_state or ()))


def validate_parameter_mapping(mapping: Sequence[int], expected_len: int, unit: str = "gates") -> None:
    if len(mapping) != expected_len:
        raise ValueError(f"parameter_mapping has {len(mapping)} entries but there are {expected_len} {unit}.")
    if mapping and set(mapping) != set(range(max(mapping) + 1)):
        raise ValueError(f"parameter_mapping indices must be contiguous 0..n-1 with no gaps; got {sorted(set(mapping))}.")


def expand_monomials(gates: Sequence[ExpGate], mapping: Sequence[int],
                     num_qubits: int) -> tuple[list[tuple[int, ...]], list[float], list[int], list[int]]:
    """Per-monomial ``(monomials, gen_coeffs, parameter_mapping, gate_indices)``; an all-dropped gate
    becomes the identity layer ``((), 0.0)`` so gate and parameter indices stay contiguous."""
    monos: list[tuple[int, ...]] = []
    coeffs: list[float] = []
    per: list[int] = []
    gidx: list[int] = []
    for gi, (gate, p) in enumerate(zip(gates, mapping, strict=True)):
        for mono, g in gate.layers() or [((), 0.0)]:
            monos.append(tuple(mono))
            coeffs.append(g)
            per.append(int(p))
            gidx.append(gi)
    return monos, coeffs, per, gidx
