"""Monomial key encoding shared by the host engine, the Python front-end and the tests.

A monomial over ``n`` logical modes (qubits, in the Pauli basis) lives in a storage tier of
``T = ceil(n / 32) * 32`` modes: ``2T`` bits packed into ``W = T / 32`` little-endian ``uint64`` words.
Slot ``s`` (a Majorana index, or a Pauli symplectic slot) is bit ``2T - 1 - s`` ("MSb0"), exactly the
reference's layout (``cpp/monoprop/algebra/AlgebraCommon.h:45-65``, tiers from
``tools/_binding_layout.py``), so exported keys compare word for word with the reference engine.

Pauli slots follow ``src/monoprop/conversion_utils.py:66-114``: ``X_q -> {2q}``, ``Y_q -> {2q+1}``,
``Z_q -> {2q, 2q+1}``.
"""

from __future__ import annotations

from collections.abc import Iterable, Sequence

import numpy as np

MAX_NUM_MODES = 256


def storage_tier(num_modes: int) -> int:
    """Storage tier (a multiple of 32 modes) holding ``num_modes`` logical modes."""
    if num_modes < 1 or num_modes > MAX_NUM_MODES:
        raise ValueError(f"num_modes must be in [1, {MAX_NUM_MODES}]; got {num_modes}")
    return ((num_modes + 31) // 32) * 32


def words_for(num_modes: int) -> int:
    """Number of uint64 words in one monomial key for ``num_modes`` logical modes."""
    return storage_tier(num_modes) // 32


def slots_to_words(slots: Iterable[int], num_modes: int) -> np.ndarray:
    """Encode one slot tuple as its key words (``uint64[W]``)."""
    tier = storage_tier(num_modes)
    out = np.zeros(tier // 32, dtype=np.uint64)
    top = 2 * tier - 1
    for s in slots:
        s = int(s)
        if s < 0 or s >= 2 * num_modes:
            raise ValueError(f"Majorana/Pauli index {s} is out of range; must be less than {2 * num_modes}.")
        b = top - s
        out[b // 64] ^= np.uint64(1) << np.uint64(b % 64)
    return out


def encode_many(monomials: Sequence[Sequence[int]], num_modes: int) -> np.ndarray:
    """Encode a list of slot tuples as a ``uint64[n, W]`` key array."""
    w = words_for(num_modes)
    out = np.zeros((len(monomials), w), dtype=np.uint64)
    for i, m in enumerate(monomials):
        out[i] = slots_to_words(m, num_modes)
    return out


def basis_rows(basis_change: Sequence[Sequence[int]], num_modes: int) -> np.ndarray:
    """``uint64[2T, W]``: row s is the monomial slot s maps to under ``basis_change`` (its listed slots set,
    as ``indices_to_bitset_checked``, ``AlgebraCommon.h:44-63``); rows of slots >= 2 * num_modes are zero."""
    if len(basis_change) != 2 * num_modes:
        raise ValueError(f"basis_change must have exactly 2*logical_num_modes ({2 * num_modes}) rows; "
                         f"got {len(basis_change)}.")
    tier = storage_tier(num_modes)
    out = np.zeros((2 * tier, tier // 32), dtype=np.uint64)
    for s, row in enumerate(basis_change):
        out[s] = slots_to_words(sorted(set(int(x) for x in row)), num_modes)
    return out


def words_to_slots(words: np.ndarray, num_modes: int) -> tuple[int, ...]:
    """Decode one key (``uint64[W]``) into its ascending slot tuple."""
    tier = storage_tier(num_modes)
    top = 2 * tier - 1
    slots = []
    for wi, word in enumerate(np.asarray(words, dtype=np.uint64).tolist()):
        while word:
            low = word & -word
            bit = low.bit_length() - 1
            slots.append(top - (wi * 64 + bit))
            word ^= low
    return tuple(sorted(slots))


def state_mask_words(initial_state: Iterable[int], num_modes: int) -> np.ndarray:
    """Key words with slot ``2*m`` set for every occupied mode ``m``.

    This is the mask the ``<0|O|0>`` phase is scored against
    (``cpp/monoprop/algebra/AlgebraCommon.h:114-122``).
    """
    return slots_to_words([2 * int(m) for m in initial_state], num_modes)


def sort_key(words_row: np.ndarray) -> tuple[int, ...]:
    """Total order on keys used to compare term sets independently of storage order."""
    return tuple(int(x) for x in words_row[::-1])


def canonical_order(keys: np.ndarray) -> np.ndarray:
    """Permutation sorting ``keys`` (``uint64[n, W]``) lexicographically, most significant word first."""
    if keys.shape[0] == 0:
        return np.zeros(0, dtype=np.int64)
    cols = [keys[:, w] for w in range(keys.shape[1])]
    return np.lexsort(cols)
