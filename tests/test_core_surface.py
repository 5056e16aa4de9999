"""The `_core` module offers every name the reference's nanobind module binds (no GPU needed).

tests/golden/reference_surface.json lists, as read from the reference sources by
``tests/golden/make_golden.py --surface``: the members the reference binds on each
``MonomialPropagatorNNN`` class (src/monoprop/bindings/binder.h), its module attributes
(bindings.cpp.in) and every ``_simulator.<name>`` its Python front-end uses
(src/monoprop/monomial_propagator.py, pauli_propagator.py, majorana_propagator.py). A front-end that
dispatches to this `_core` must find all of them, on every storage tier.
"""

import json
import os

import pytest

from monoprop_b200 import _core

HERE = os.path.dirname(os.path.abspath(__file__))
SURFACE = json.load(open(os.path.join(HERE, "golden", "reference_surface.json")))
TIERS = [32, 64, 96, 128, 160, 192, 224, 256]


@pytest.mark.parametrize("tier", TIERS)
def test_every_bound_member_exists(tier):
    cls = getattr(_core, f"MonomialPropagator{tier:03d}")
    missing = [name for name in SURFACE["class_members"] if not hasattr(cls, name)]
    assert not missing, missing
    assert cls.storage_num_modes == tier


def test_front_end_calls_are_covered():
    assert set(SURFACE["frontend_simulator_calls"]) <= set(SURFACE["class_members"])
    cls = _core.MonomialPropagator032
    assert all(hasattr(cls, name) for name in SURFACE["frontend_simulator_calls"])


def test_module_attributes():
    missing = [name for name in SURFACE["module_attributes"] if not hasattr(_core, name)]
    assert not missing, missing
    assert _core.MAX_NUM_MODES == 256 and _core.has_mpi is False
    assert _core.is_antihermitian([0, 1]) and not _core.is_antihermitian([0, 1, 2, 3])


def test_read_write_properties():
    """Properties the front-end assigns (cutoff, lower_atol, upper_atol, cutoff_type, parameter_mapping,
    basis_change) have setters; num_modes, schrodinger and basis are read-only as in the reference."""
    cls = _core.MonomialPropagator064
    for name in ("cutoff", "lower_atol", "upper_atol", "cutoff_type", "parameter_mapping", "basis_change"):
        assert getattr(cls, name).fset is not None, name
    for name in ("num_modes", "schrodinger", "basis"):
        assert getattr(cls, name).fset is None, name
