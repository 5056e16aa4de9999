"""The allocation-free <0|O|0> entry point (mpx_expectation_noalloc) against the engine's own.

mpx_expectation_noalloc serves callers that cannot call cudaMalloc while they run (a host runtime that
owns all device memory and lends this library pre-sized buffers, or one that cannot take the device-wide
synchronisation an allocation implies): it reads a device-resident term store and writes <O> to a device
buffer, keeping its scratch in a fixed array inside the library. This file is collected last, so a run
that stops at the first failure has run every other test first; it also passes alone in a fresh process.

Two calls in a row must each agree with mpx_expectation on the same store to 1e-10 relative (the
tolerance of the other GPU parity tests): the second call sees the first call's leftovers in the shared
scratch array.
"""

import ctypes as C

import numpy as np
import pytest

from monoprop_b200 import _native
from monoprop_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _noalloc(lib, eng, basis_code, mask, core, out_ptr, stream):
    keys, coefs, n = C.c_void_p(), C.c_void_p(), C.c_uint64(0)
    eng._check(lib.mpx_device_view(eng.h, C.byref(keys), C.byref(coefs), C.byref(n)))
    err = C.create_string_buffer(512)
    m = np.ascontiguousarray(mask, dtype=np.uint64)
    rc = lib.mpx_expectation_noalloc(basis_code, eng.words, keys, coefs, n.value, m.ctypes.data_as(C.c_void_p),
                                     float(core), C.c_void_p(out_ptr), C.c_void_p(stream), err, 512)
    assert rc == 0, err.value.decode()


# key widths 1 (20 qubits), 3 (72 modes), 2 (50 qubits) and 4 (100 qubits)
@pytest.mark.parametrize("make, n_layers", [(W.line20, None), (W.hubbard6x6, 700), (lambda: W.ising50(3), None),
                                            (W.ising100, 900)])
def test_noalloc_expectation_matches_engine(make, n_layers):
    import torch

    wl = make()
    lib = _native.load()
    eng = _native.engine_for(wl)
    L = wl.n_layers if n_layers is None else n_layers
    eng.propagate(wl.gen_words()[:L], wl.angles()[:L])
    expected = eng.expectation()
    _, _, core = wl.encoded_observable()
    basis_code = 1 if wl.basis == "pauli" else 0
    stream = eng.stream()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for k in range(2):
        _noalloc(lib, eng, basis_code, wl.state_mask(), core, out.data_ptr() + 8 * k, stream)
    torch.cuda.ExternalStream(stream).synchronize()
    got = out.cpu().numpy()
    eng.close()
    for v in got:
        assert abs(v - expected) <= RTOL * max(1.0, abs(expected)), (v, expected)


def test_noalloc_rejects_oversized_store():
    lib = _native.load()
    err = C.create_string_buffer(512)
    rc = lib.mpx_expectation_noalloc(1, 1, C.c_void_p(16), C.c_void_p(16), (1 << 28) + 1, None, 0.0,
                                     C.c_void_p(16), None, err, 512)
    assert rc == 4 and b"268435456" in err.value
