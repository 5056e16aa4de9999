"""Test oracle for the propagation hot path -- test infrastructure, never product code.

Two CPU engines sit behind one interface:

* ``PortOracle`` -- ``oracle/mp_oracle.c``, this repository's plain-C restatement of the reference's
  Heisenberg per-gate sweep (built to ``oracle/libmporacle.so`` by :func:`build`). It travels to the
  GPU box and is what the GPU parity tests compare against.
* ``RefOracle`` -- the unmodified reference engine (monoprop's ``MonomialPropagator<N>``) compiled from
  its own sources by ``oracle/build_ref.sh`` into ``oracle/_ref/libmpref.so``. It pins the port:
  ``tests/test_oracle.py`` checks the port against it, and the golden fixtures under ``tests/golden/``
  were generated from it.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs import this
package.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "libmporacle.so")
REF_LIB = os.path.join(HERE, "_ref", "libmpref.so")


def build(reference_root: str | None = None) -> None:
    """Compile the C restatement, and the reference oracle when its sources are present.

    ``reference_root`` (else ``$MONOPROP_REFERENCE``, else the default of ``oracle/build_ref.sh``) is the
    reference source tree; without it the prebuilt ``oracle/_ref`` is kept as it is."""
    src = os.path.join(HERE, "mp_oracle.c")
    if not os.path.exists(PORT_LIB) or os.path.getmtime(src) > os.path.getmtime(PORT_LIB):
        # -ffp-contract=fast on an FMA target mirrors how the reference's own -O3 build contracts
        # c += s*phi*v into one fused multiply-add (checked bit-for-bit in tests/test_oracle.py).
        subprocess.check_call(["gcc", "-O2", "-march=x86-64-v3", "-ffp-contract=fast", "-shared", "-fPIC",
                               src, "-o", PORT_LIB, "-lm"])
    reference_root = reference_root or os.environ.get("MONOPROP_REFERENCE")
    subprocess.check_call([os.path.join(HERE, "build_ref.sh"), *([reference_root] if reference_root else [])])


class _PortCfg(C.Structure):
    _fields_ = [("basis", C.c_int32), ("cutoff_type", C.c_int32), ("cutoff", C.c_uint32),
                ("has_lower", C.c_int32), ("lower", C.c_double), ("has_upper", C.c_int32),
                ("upper", C.c_double), ("words", C.c_int32), ("has_len_k", C.c_int32), ("len_k", C.c_uint32),
                ("basis_rows", C.c_void_p), ("schrodinger", C.c_int32), ("logical_modes", C.c_int32)]


class _RefCfg(C.Structure):
    _fields_ = [("basis", C.c_int32), ("cutoff_type", C.c_int32), ("cutoff", C.c_uint32),
                ("has_lower", C.c_int32), ("lower", C.c_double), ("has_upper", C.c_int32),
                ("upper", C.c_double), ("partitions", C.c_int32), ("logical_num_modes", C.c_int32),
                ("len_k", C.c_int32), ("schrodinger_cutoff", C.c_int32)]


_P = np.ctypeslib.ndpointer


def _ptr(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class Result:
    keys: np.ndarray  # uint64[n, W]
    coefs: np.ndarray  # float64[n]
    expectation: float
    seconds: float
    counts: np.ndarray | None = None  # uint64[L, 4]: n_g, a_g, e_g, m_g per applied gate


_port = None
_ref = None


def _load_port() -> C.CDLL:
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build()
        lib = C.CDLL(PORT_LIB)
        lib.mpo_create.restype = C.c_void_p
        lib.mpo_create.argtypes = [C.POINTER(_PortCfg), C.c_size_t, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]
        lib.mpo_propagate.restype = C.c_int
        lib.mpo_propagate.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.mpo_size.restype = C.c_size_t
        lib.mpo_size.argtypes = [C.c_void_p]
        lib.mpo_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.mpo_expectation.restype = C.c_double
        lib.mpo_expectation.argtypes = [C.c_void_p]
        lib.mpo_destroy.argtypes = [C.c_void_p]
        _port = lib
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


#: builds of the reference by instruction set (oracle/build_ref.sh), most specific first, with the host CPU
#: flags each needs
REF_BUILDS = {
    "spr": (os.path.join(HERE, "_ref", "libmpref_spr.so"),
            ("avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd", "avx512_fp16", "avx512_bf16", "amx_tile",
             "avx512_vpopcntdq", "avx512_bitalg", "avx512vbmi", "avx512_vbmi2", "avx512_vnni", "gfni", "vaes")),
    "v4": (os.path.join(HERE, "_ref", "libmpref_v4.so"), ("avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd")),
    "v3": (REF_LIB, ("avx2", "fma", "bmi2")),
}


def _host_flags() -> set[str]:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def native_ref_build() -> str:
    """The reference build matching this host's CPU, as the reference's own default -march=native build
    would (``cmake/compiler_flags/CXXFlags.cmake``): the most specific one whose instruction-set extensions
    the host has and whose library was built, checked by a short run in a child process (an illegal
    instruction there cannot take this process down)."""
    import subprocess
    import sys

    flags = _host_flags()
    for name, (path, need) in REF_BUILDS.items():
        if name == "v3" or not os.path.exists(path) or not all(f in flags for f in need):
            continue
        probe = ("import sys; sys.path.insert(0, %r); import oracle; from monoprop_b200 import workloads as W; "
                 "oracle.RefEngine(W.line20(), build=%r).propagate(n_layers=40)") % (os.path.dirname(HERE), name)
        if subprocess.run([sys.executable, "-c", probe], capture_output=True, timeout=120).returncode == 0:
            return name
    return "v3"


def _load_ref(build: str = "v3") -> C.CDLL:
    global _ref
    if _ref is None:
        _ref = {}
    if build not in _ref:
        lib = C.CDLL(REF_BUILDS[build][0])
        lib.mpref_create.restype = C.c_void_p
        lib.mpref_create.argtypes = [C.POINTER(_RefCfg), C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p,
                                     C.c_size_t]
        lib.mpref_propagate.restype = C.c_int
        lib.mpref_propagate.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_size_t, C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_char_p,
                                        C.c_size_t]
        lib.mpref_expectation.restype = C.c_int
        lib.mpref_expectation.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.POINTER(C.c_double), C.c_char_p,
                                          C.c_size_t]
        lib.mpref_expectation_and_gradient.restype = C.c_int
        lib.mpref_expectation_and_gradient.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.POINTER(C.c_double),
                                                       C.c_void_p, C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
        lib.mpref_size.restype = C.c_size_t
        lib.mpref_size.argtypes = [C.c_void_p]
        lib.mpref_words.restype = C.c_size_t
        lib.mpref_words.argtypes = [C.c_void_p]
        lib.mpref_core.restype = C.c_double
        lib.mpref_core.argtypes = [C.c_void_p]
        lib.mpref_export.restype = C.c_int64
        lib.mpref_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t]
        lib.mpref_export_at.restype = C.c_int64
        lib.mpref_export_at.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_char_p, C.c_size_t]
        lib.mpref_destroy.argtypes = [C.c_void_p]
        _ref[build] = lib
    return _ref[build]


def _basis_code(basis: str) -> int:
    return 1 if basis == "pauli" else 0


def _cutoff_code(ct: str) -> int:
    return 1 if ct == "support" else 0


def run_port(wl, params: np.ndarray | None = None, n_layers: int | None = None) -> Result:
    """Propagate workload ``wl`` through the C restatement (optionally only its first ``n_layers``)."""
    lib = _load_port()
    keys, coefs, core = wl.encoded_observable()
    W = wl.words
    len_k = wl.extra.get("only_rotate_len_k")
    rows = None
    if wl.extra.get("basis_change") is not None:
        from monoprop_b200.encoding import basis_rows

        rows = np.ascontiguousarray(basis_rows(wl.extra["basis_change"], wl.num_modes))
    cfg = _PortCfg(_basis_code(wl.basis), _cutoff_code(wl.cutoff_type), wl.cutoff,
                   int(wl.lower_atol is not None), float(wl.lower_atol or 0.0),
                   int(wl.upper_atol is not None), float(wl.upper_atol or 0.0), W,
                   int(len_k is not None), int(len_k or 0), None if rows is None else rows.ctypes.data,
                   int(wl.extra["schrodinger_cutoff"]) if wl.extra.get("schrodinger_cutoff") is not None else -1,
                   int(wl.num_modes))
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    coefs = np.ascontiguousarray(coefs, dtype=np.float64)
    mask = np.ascontiguousarray(wl.state_mask(), dtype=np.uint64)
    h = lib.mpo_create(C.byref(cfg), keys.shape[0], _ptr(keys), _ptr(coefs), core, _ptr(mask))
    if not h:
        raise RuntimeError("oracle create failed")
    try:
        L = wl.n_layers if n_layers is None else n_layers
        gw = np.ascontiguousarray(wl.gen_words()[:L], dtype=np.uint64)
        ang = np.ascontiguousarray(wl.angles(params)[:L], dtype=np.float64)
        counts = np.zeros((L, 4), dtype=np.uint64)
        t0 = time.perf_counter()
        rc = lib.mpo_propagate(h, L, _ptr(gw), _ptr(ang), _ptr(counts))
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError("oracle propagate failed")
        n = lib.mpo_size(h)
        ok = np.zeros((n, W), dtype=np.uint64)
        oc = np.zeros(n, dtype=np.float64)
        lib.mpo_export(h, _ptr(ok), _ptr(oc))
        ev = lib.mpo_expectation(h)
    finally:
        lib.mpo_destroy(h)
    return Result(ok, oc, ev, dt, counts)


def _flat_slots(monos) -> tuple[np.ndarray, np.ndarray]:
    off = np.zeros(len(monos) + 1, dtype=np.int64)
    flat: list[int] = []
    for i, m in enumerate(monos):
        flat.extend(int(s) for s in m)
        off[i + 1] = len(flat)
    return off, np.asarray(flat if flat else [0], dtype=np.int64)


class RefEngine:
    """The unmodified reference ``MonomialPropagator<N>`` through the C-ABI driver."""

    def __init__(self, wl, partitions: int = 1, build: str = "v3"):
        self.lib = _load_ref(build)
        self.wl = wl
        obs = sorted(wl.observable.items())
        off, flat = _flat_slots([k for k, _ in obs])
        re = np.asarray([complex(v).real for _, v in obs], dtype=np.float64)
        im = np.asarray([complex(v).imag for _, v in obs], dtype=np.float64)
        st = np.asarray(list(wl.initial_state) or [0], dtype=np.int64)
        cfg = _RefCfg(_basis_code(wl.basis), _cutoff_code(wl.cutoff_type), wl.cutoff,
                      int(wl.lower_atol is not None), float(wl.lower_atol or 0.0),
                      int(wl.upper_atol is not None), float(wl.upper_atol or 0.0), partitions, wl.num_modes,
                      int(wl.extra.get("only_rotate_len_k") or 0),
                      int(wl.extra["schrodinger_cutoff"]) if wl.extra.get("schrodinger_cutoff") is not None else -1)
        err = C.create_string_buffer(1024)
        self._keep = (off, flat, re, im, st)
        bc = wl.extra.get("basis_change")
        boff, bflat = _flat_slots(bc) if bc is not None else (np.zeros(1, np.int64), np.zeros(1, np.int64))
        self._keep = (off, flat, re, im, st, boff, bflat)
        self.h = self.lib.mpref_create(C.byref(cfg), len(obs), _ptr(off), _ptr(flat), _ptr(re), _ptr(im),
                                       len(wl.initial_state), _ptr(st), 0 if bc is None else len(bc), _ptr(boff),
                                       _ptr(bflat), err, 1024)
        if not self.h:
            raise RuntimeError(err.value.decode())

    def _gates(self, n_layers):
        L = self.wl.n_layers if n_layers is None else n_layers
        off, flat = _flat_slots(self.wl.gate_slots[:L])
        g = np.ascontiguousarray(self.wl.gen_coeffs[:L], dtype=np.float64)
        pm = np.ascontiguousarray(self.wl.param_map[:L], dtype=np.int64)
        return L, off, flat, g, pm

    def propagate(self, params=None, n_layers=None, build_graph=False) -> float:
        L, off, flat, g, pm = self._gates(n_layers)
        p = np.ascontiguousarray(self.wl.params if params is None else params, dtype=np.float64)
        p = np.ascontiguousarray(p[: int(pm.max()) + 1]) if L else p
        secs = C.c_double(0.0)
        err = C.create_string_buffer(1024)
        rc = self.lib.mpref_propagate(self.h, L, _ptr(off), _ptr(flat), _ptr(g), _ptr(pm), p.size, _ptr(p),
                                      int(build_graph), C.byref(secs), err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return secs.value

    def expectation(self, params=()) -> float:
        p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
        out = C.c_double(0.0)
        err = C.create_string_buffer(1024)
        pp = p if p.size else np.zeros(1)
        if self.lib.mpref_expectation(self.h, p.size, _ptr(pp), C.byref(out), err, 1024) != 0:
            raise RuntimeError(err.value.decode())
        return out.value

    def expectation_and_gradient(self, params) -> tuple[float, np.ndarray, float]:
        p = np.ascontiguousarray(params, dtype=np.float64)
        g = np.zeros(p.size, dtype=np.float64)
        out = C.c_double(0.0)
        secs = C.c_double(0.0)
        err = C.create_string_buffer(1024)
        if self.lib.mpref_expectation_and_gradient(self.h, p.size, _ptr(p), C.byref(out), _ptr(g), C.byref(secs),
                                                   err, 1024) != 0:
            raise RuntimeError(err.value.decode())
        return out.value, g, secs.value

    def size(self) -> int:
        return int(self.lib.mpref_size(self.h))

    def export(self, params=None) -> tuple[np.ndarray, np.ndarray]:
        """Raw keys and coefficients of the current operator, or of the stored graph replayed at ``params``."""
        n = self.size()
        W = int(self.lib.mpref_words(self.h))
        keys = np.zeros((max(n, 1), W), dtype=np.uint64)
        coefs = np.zeros(max(n, 1), dtype=np.float64)
        err = C.create_string_buffer(1024)
        if params is None:
            got = self.lib.mpref_export(self.h, _ptr(keys), _ptr(coefs), n, err, 1024)
        else:
            p = np.ascontiguousarray(params, dtype=np.float64)
            got = self.lib.mpref_export_at(self.h, p.size, _ptr(p), _ptr(keys), _ptr(coefs), n, err, 1024)
        if got < 0:
            raise RuntimeError(err.value.decode())
        return keys[:got], coefs[:got]

    def close(self):
        if self.h:
            self.lib.mpref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_ref(wl, params=None, partitions: int = 1, n_layers: int | None = None) -> Result:
    """Propagate ``wl`` through the unmodified reference; keys/coefs exported raw (partitions must be 1)."""
    eng = RefEngine(wl, partitions=partitions)
    try:
        secs = eng.propagate(params, n_layers)
        ev = eng.expectation()
        if partitions == 1:
            keys, coefs = eng.export()
        else:
            keys, coefs = np.zeros((0, wl.words), np.uint64), np.zeros(0)
    finally:
        eng.close()
    return Result(keys, coefs, ev, secs)
