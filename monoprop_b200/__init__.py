"""B200-native Pauli and Majorana propagation (Heisenberg picture) with monoprop's public API.

The package's public names resolve lazily, so the build helpers and the ctypes layer import without
the compiled ``_core`` module present.
"""

_EXPORTS = {
    "PauliPropagator": "propagators", "MajoranaPropagator": "propagators", "MonomialPropagator": "propagators",
    "Circuit": "circuit", "ExpGate": "circuit", "expand_monomials": "circuit",
    "Pauli": "operators", "PauliOperator": "operators", "Majorana": "operators", "MajoranaOperator": "operators",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name in _EXPORTS:
        import importlib

        return getattr(importlib.import_module(f".{_EXPORTS[name]}", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
