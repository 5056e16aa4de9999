"""Observable and generator operators of the front-end: Majorana and Pauli sums.

Same public surface and normalisation rules as the reference's ``src/monoprop/majorana.py`` and
``src/monoprop/pauli.py``:

* a Majorana monomial is a sorted tuple of distinct indices; an unsorted product is brought to that
  form with the sign of the reordering (Majoranas anticommute) and repeated indices cancel in pairs
  (``m_i m_i = 1``) -- ``Majorana.from_unsorted`` (``majorana.py:76-95``, ``conversion_utils.py:115-145``);
* a Pauli term is letters on qubits, identities dropped and sorted by qubit (``pauli.py:56-95``); the
  engine's native Pauli encoding puts ``X_q`` on slot ``2q``, ``Y_q`` on ``2q+1`` and ``Z_q`` on both
  (``conversion_utils.py:66-114``).
"""

from __future__ import annotations

from collections import defaultdict
from collections.abc import Mapping, Sequence

import numpy as np

_PAULI_LETTERS = frozenset("IXYZ")


def _check_size(value, name: str) -> int:
    if isinstance(value, bool) or not isinstance(value, (int, np.integer)):
        raise TypeError(f"{name} must be an integer; got {type(value).__name__}.")
    if value < 0:
        raise ValueError(f"{name} must be non-negative; got {value}.")
    return int(value)


def reorder_sign(indices: Sequence[int]) -> int:
    """(-1)^(number of strictly inverted pairs): the sign of sorting anticommuting Majoranas."""
    inv = 0
    for i, x in enumerate(indices):
        for y in indices[i + 1:]:
            inv += x > y
    return -1 if inv & 1 else 1


def cancel_pairs(sorted_indices: Sequence[int]) -> tuple[int, ...]:
    """Drop equal neighbours two at a time from a sorted index sequence (``m_i^2 = 1``)."""
    out: list[int] = []
    for x in sorted_indices:
        if out and out[-1] == x:
            out.pop()
        else:
            out.append(x)
    return tuple(out)


class Majorana:
    """A Majorana monomial ``m_{i1} ... m_{iw}`` with sorted, distinct, non-negative indices."""

    __slots__ = ("indices",)

    def __init__(self, *indices: int) -> None:
        if any(i < 0 for i in indices):
            raise ValueError(f"Majorana indices must be non-negative; got {indices}.")
        if any(a >= b for a, b in zip(indices, indices[1:])):
            raise ValueError(f"Majorana indices must be distinct and sorted; got {indices}.")
        self.indices = tuple(int(i) for i in indices)

    @classmethod
    def from_unsorted(cls, *indices: int) -> tuple[Majorana, float]:
        if any(i < 0 for i in indices):
            raise ValueError(f"Majorana indices must be non-negative; got {indices}.")
        return cls(*cancel_pairs(sorted(indices))), float(reorder_sign(indices))

    def __eq__(self, other) -> bool:
        return isinstance(other, Majorana) and self.indices == other.indices

    def __hash__(self) -> int:
        return hash(self.indices)

    def __repr__(self) -> str:
        return f"Majorana({', '.join(map(str, self.indices))})"


class MajoranaOperator:
    """A weighted sum of Majorana monomials; ``terms`` maps sorted index tuples to complex weights."""

    def __init__(self, terms: Mapping, num_modes: int) -> None:
        keys = [k.indices if isinstance(k, Majorana) else tuple(int(i) for i in k) for k in terms]
        for k in keys:
            Majorana.from_unsorted(*k)  # index validation
        self.num_modes = _check_size(num_modes, "num_modes")
        for k in keys:
            if k and max(k) >= 2 * self.num_modes:
                raise ValueError(f"Majorana term {k} acts on an index >= num_modes={self.num_modes}.")
        self.terms = self._accumulate(keys, list(terms.values()))

    @classmethod
    def _from_terms(cls, monomials: Sequence[Sequence[int]], coefficients: Sequence[complex],
                    num_modes: int) -> MajoranaOperator:
        obj = cls.__new__(cls)
        obj.num_modes = _check_size(num_modes, "num_modes")
        obj.terms = cls._accumulate(monomials, coefficients)
        return obj

    @staticmethod
    def _accumulate(monomials, coefficients) -> dict[tuple[int, ...], complex]:
        acc: dict[tuple[int, ...], complex] = defaultdict(complex)
        for mono, c in zip(monomials, coefficients, strict=True):
            canon, sign = Majorana.from_unsorted(*mono)
            acc[canon.indices] += complex(c) * sign
        return dict(acc)

    def get_majorana_operator(self) -> MajoranaOperator:
        return self

    def all_pairwise_commute(self) -> bool:
        """Monomials with supports S1, S2 commute iff |S1||S2| - |S1 & S2| is even."""
        sets = [set(k) for k in self.terms]
        for i, a in enumerate(sets):
            for b in sets[i + 1:]:
                if (len(a) * len(b) - len(a & b)) % 2:
                    return False
        return True

    def isclose(self, other, rtol: float = 1e-5, atol: float = 1e-8) -> bool:
        if not isinstance(other, MajoranaOperator):
            raise TypeError(f"Cannot compare MajoranaOperator with {type(other).__name__}.")
        if self.num_modes != other.num_modes:
            return False
        return all(np.isclose(self.terms.get(k, 0), other.terms.get(k, 0), rtol=rtol, atol=atol)
                   for k in self.terms | other.terms)

    def __len__(self) -> int:
        return len(self.terms)

    def __eq__(self, other) -> bool:
        if not isinstance(other, MajoranaOperator):
            return NotImplemented
        return self.num_modes == other.num_modes and self.terms == other.terms

    __hash__ = None

    def __repr__(self) -> str:
        return f"MajoranaOperator({len(self)} terms, {self.num_modes} modes)"


class Pauli:
    """Pauli letters on qubits; identities dropped, sorted by qubit."""

    __slots__ = ("qubits", "string")

    def __init__(self, string: str, qubits: int | Sequence[int] | None = None) -> None:
        if qubits is None:
            qubits = range(len(string))
        elif isinstance(qubits, (int, np.integer)):
            qubits = (int(qubits),)
        qs = tuple(int(q) for q in qubits)
        bad = set(string) - _PAULI_LETTERS
        if bad:
            raise ValueError(f"Invalid characters in Pauli string: {bad}. Only I, X, Y, Z are allowed.")
        if len(string) != len(qs):
            raise ValueError(f"Pauli string {string!r} and qubits {qs} must have the same length.")
        if len(set(qs)) != len(qs):
            raise ValueError(f"Duplicate qubit indices in Pauli term: {qs}.")
        if any(q < 0 for q in qs):
            raise ValueError(f"Pauli qubit indices must be non-negative; got {qs}.")
        pairs = sorted((q, p) for q, p in zip(qs, string) if p != "I")
        self.qubits = tuple(q for q, _ in pairs)
        self.string = "".join(p for _, p in pairs)

    def slots(self) -> tuple[int, ...]:
        """Native engine slots: X_q -> {2q}, Y_q -> {2q+1}, Z_q -> {2q, 2q+1}."""
        out: list[int] = []
        for p, q in zip(self.string, self.qubits):
            if p == "X":
                out.append(2 * q)
            elif p == "Y":
                out.append(2 * q + 1)
            else:
                out += [2 * q, 2 * q + 1]
        return tuple(sorted(out))

    @classmethod
    def from_slots(cls, slots: Sequence[int]) -> Pauli:
        """Inverse of :meth:`slots`: (2q only) X, (2q+1 only) Y, (both) Z."""
        present = set(int(s) for s in slots)
        letters, qubits = [], []
        for q in sorted({s // 2 for s in present}):
            u, v = 2 * q in present, 2 * q + 1 in present
            letters.append("X" if u and not v else ("Y" if v and not u else "Z"))
            qubits.append(q)
        return cls("".join(letters), tuple(qubits))

    def __eq__(self, other) -> bool:
        return isinstance(other, Pauli) and (self.string, self.qubits) == (other.string, other.qubits)

    def __hash__(self) -> int:
        return hash((self.string, self.qubits))

    def __repr__(self) -> str:
        return f"Pauli({self.string!r}, {self.qubits})"


class PauliOperator:
    """A real-weighted sum of Pauli terms on ``num_qubits`` qubits."""

    def __init__(self, terms: Mapping, num_qubits: int) -> None:
        acc: dict[Pauli, float] = defaultdict(float)
        for key, c in terms.items():
            p = key if isinstance(key, Pauli) else Pauli(key)
            v = np.real_if_close(c)
            if np.iscomplexobj(v):
                raise ValueError("Operator has complex terms")
            acc[p] += float(v)
        self.terms: dict[Pauli, float] = dict(acc)
        self.num_qubits = _check_size(num_qubits, "num_qubits")
        for p in self.terms:
            if p.qubits and p.qubits[-1] >= self.num_qubits:
                raise ValueError(f"Pauli term {p} acts on a qubit index >= num_qubits={self.num_qubits}.")

    def get_local_operator(self) -> MajoranaOperator:
        """The operator in the engine's native Pauli slot encoding (a container of slot tuples)."""
        return MajoranaOperator._from_terms([p.slots() for p in self.terms], list(self.terms.values()),
                                            self.num_qubits)

    def all_pairwise_commute(self) -> bool:
        items = list(self.terms)
        for i, a in enumerate(items):
            da = dict(zip(a.qubits, a.string))
            for b in items[i + 1:]:
                anti = sum(1 for q, p in zip(b.qubits, b.string) if q in da and da[q] != p)
                if anti & 1:
                    return False
        return True

    def isclose(self, other, rtol: float = 1e-5, atol: float = 1e-8) -> bool:
        if not isinstance(other, PauliOperator):
            raise TypeError(f"Cannot compare PauliOperator with {type(other).__name__}.")
        if self.num_qubits != other.num_qubits:
            return False
        return all(np.isclose(self.terms.get(k, 0.0), other.terms.get(k, 0.0), rtol=rtol, atol=atol)
                   for k in self.terms | other.terms)

    def __len__(self) -> int:
        return len(self.terms)

    def __eq__(self, other) -> bool:
        if not isinstance(other, PauliOperator):
            return NotImplemented
        return self.num_qubits == other.num_qubits and self.terms == other.terms

    __hash__ = None

    def __repr__(self) -> str:
        return f"PauliOperator({len(self)} terms, {self.num_qubits} qubits)"
