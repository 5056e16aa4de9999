"""The C-ABI library loads here (no GPU) and exports every entry point include/mpx.h declares."""

import os
import re

from monoprop_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "mpx.h")).read()
    return sorted(set(re.findall(r"MPX_API\s+[\w\s\*]*?\b(mpx_\w+)\s*\(", text)))


def test_header_lists_match_binding():
    assert declared_entry_points() == sorted(_native.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    for name in declared_entry_points():
        assert hasattr(lib, name), name


def test_create_without_device_fails_loudly():
    # No CUDA device in the CPU container: the engine must refuse rather than fall back to the CPU.
    import torch

    if torch.cuda.is_available():
        return
    import numpy as np
    import pytest

    with pytest.raises(_native.MpxError) as ei:
        _native.Engine(basis="pauli", cutoff_type="support", cutoff=4, num_modes=4,
                       keys=np.zeros((1, 1), np.uint64), coefs=np.ones(1), core=0.0,
                       state_mask=np.zeros(1, np.uint64))
    assert ei.value.status == 6
