"""ctypes binding of the engine's C ABI (``include/mpx.h``, ``monoprop_b200/libmpx.so``).

This is the thin host layer every Python caller goes through. There is no CPU fallback: if the library
is missing or no sm_100a device is visible, constructing an :class:`Engine` raises.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmpx.so")

MPX_OK = 0
_STATUS = {1: "MPX_ERR_INVALID", 2: "MPX_ERR_CUDA", 3: "MPX_ERR_NOMEM", 4: "MPX_ERR_CAPACITY", 5: "MPX_ERR_STATE",
           6: "MPX_ERR_NO_DEVICE"}

#: Every entry point declared in include/mpx.h.
EXPORTED = ("mpx_create", "mpx_propagate", "mpx_circuit_upload", "mpx_circuit_set_angles", "mpx_propagate_circuit",
            "mpx_circuit_destroy", "mpx_expectation", "mpx_size", "mpx_words", "mpx_export", "mpx_gate_stats",
            "mpx_reset", "mpx_set_cutoff", "mpx_set_lower_atol", "mpx_set_upper_atol",
            "mpx_set_only_rotate_len_k", "mpx_set_basis_change", "mpx_device_view",
            "mpx_stream", "mpx_launch_count", "mpx_adjoint_forward", "mpx_adjoint_backward", "mpx_graph_build", "mpx_graph_expectation",
            "mpx_graph_gradient", "mpx_set_pair_log", "mpx_set_profiling", "mpx_kernel_times",
            "mpx_trim_device_memory", "mpx_last_error",
            "mpx_destroy", "mpx_expectation_noalloc", "mpx_batch_run", "mpx_update_initial_operator", "mpx_memory",
            "mpx_graph_info", "mpx_clone", "mpx_current_device", "mpx_graph_pare", "mpx_set_cutoff_type",
            "mpx_graph_replay_count", "mpx_adjoint_logged")


class MpxError(RuntimeError):
    """An engine call failed; ``status`` is the mpx_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class MpxInvalid(MpxError, ValueError):
    """MPX_ERR_INVALID: the reference raises ValueError for these."""


class Config(C.Structure):
    _fields_ = [("basis", C.c_int32), ("cutoff_type", C.c_int32), ("cutoff", C.c_uint32),
                ("has_lower_atol", C.c_int32), ("lower_atol", C.c_double), ("has_upper_atol", C.c_int32),
                ("upper_atol", C.c_double), ("num_modes", C.c_int32), ("device", C.c_int32),
                ("capacity_hint", C.c_uint64), ("blocks_per_sm", C.c_int32), ("table_shift", C.c_int32),
                ("has_schrodinger", C.c_int32), ("schrodinger_cutoff", C.c_int32), ("logical_num_modes", C.c_int32)]


class MemoryInfo(C.Structure):
    """``mpx_memory_info``: device bytes the engine holds, by part."""

    _fields_ = [("terms", C.c_uint64), ("capacity", C.c_uint64), ("words", C.c_uint32), ("key_bytes", C.c_uint64),
                ("coef_bytes", C.c_uint64), ("table_bytes", C.c_uint64), ("column_bytes", C.c_uint64),
                ("scratch_bytes", C.c_uint64), ("initial_bytes", C.c_uint64), ("graph_layers", C.c_uint64),
                ("graph_pairs", C.c_uint64), ("graph_bytes", C.c_uint64)]


_lib = None


def load() -> C.CDLL:
    """Load libmpx.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m monoprop_b200.build` "
                              "(the engine has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        vp, u64, st = C.c_void_p, C.c_uint64, C.c_int
        sig = {
            "mpx_create": (st, [C.POINTER(Config), vp, vp, u64, C.c_double, vp, C.POINTER(vp)]),
            "mpx_propagate": (st, [vp, vp, vp, u64]),
            "mpx_circuit_upload": (st, [vp, vp, vp, u64, C.POINTER(vp)]),
            "mpx_circuit_set_angles": (st, [vp, vp, vp]),
            "mpx_propagate_circuit": (st, [vp, vp]),
            "mpx_circuit_destroy": (None, [vp]),
            "mpx_expectation": (st, [vp, C.POINTER(C.c_double)]),
            "mpx_size": (st, [vp, C.POINTER(u64)]),
            "mpx_words": (st, [vp, C.POINTER(C.c_uint32)]),
            "mpx_export": (st, [vp, vp, vp, u64, C.POINTER(u64)]),
            "mpx_gate_stats": (st, [vp, vp, u64, C.POINTER(u64)]),
            "mpx_reset": (st, [vp]),
            "mpx_set_cutoff": (st, [vp, C.c_uint32]),
            "mpx_set_lower_atol": (st, [vp, C.c_int32, C.c_double]),
            "mpx_set_upper_atol": (st, [vp, C.c_int32, C.c_double]),
            "mpx_set_only_rotate_len_k": (st, [vp, C.c_int64]),
            "mpx_set_basis_change": (st, [vp, vp, C.c_uint32]),
            "mpx_device_view": (st, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(u64)]),
            "mpx_stream": (st, [vp, C.POINTER(vp)]),
            "mpx_launch_count": (st, [vp, C.POINTER(u64)]),
            "mpx_adjoint_forward": (st, [vp, vp, u64, C.POINTER(C.c_double)]),
            "mpx_adjoint_backward": (st, [vp, vp, vp]),
            "mpx_graph_build": (st, [vp, vp, u64, C.POINTER(C.c_double)]),
            "mpx_graph_expectation": (st, [vp, vp, C.POINTER(C.c_double)]),
            "mpx_graph_gradient": (st, [vp, vp, u64, C.POINTER(C.c_double), vp]),
            "mpx_set_pair_log": (st, [vp, C.c_int64]),
            "mpx_set_profiling": (st, [vp, C.c_int32]),
            "mpx_kernel_times": (st, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(u64)]),
            "mpx_trim_device_memory": (st, [C.c_int32]),
            "mpx_last_error": (C.c_char_p, [vp]),
            "mpx_destroy": (None, [vp]),
            "mpx_expectation_noalloc": (st, [C.c_int32, C.c_uint32, vp, vp, u64, vp, C.c_double, vp, vp, C.c_char_p,
                                             C.c_size_t]),
            "mpx_batch_run": (st, [C.POINTER(Config), vp, u64, vp, C.c_char_p, C.c_size_t]),
            "mpx_update_initial_operator": (st, [vp, vp, vp, u64, C.c_int32, C.c_double, C.POINTER(u64)]),
            "mpx_memory": (st, [vp, C.POINTER(MemoryInfo)]),
            "mpx_graph_info": (st, [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64)]),
            "mpx_clone": (st, [vp, vp, C.POINTER(vp), C.POINTER(vp)]),
            "mpx_current_device": (st, [C.POINTER(C.c_int32)]),
            "mpx_graph_pare": (st, [vp, vp, C.c_double]),
            "mpx_set_cutoff_type": (st, [vp, C.c_int32]),
            "mpx_graph_replay_count": (st, [vp, C.POINTER(u64)]),
            "mpx_adjoint_logged": (st, [vp, C.POINTER(C.c_int32)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class GateStats:
    """Per applied gate (application order): terms before, anticommuting, emitted, appended."""

    n: np.ndarray
    anti: np.ndarray
    emitted: np.ndarray
    appended: np.ndarray

    @property
    def term_gate_updates(self) -> int:
        return int(self.n.sum())


class Circuit:
    """A circuit resident in device memory (``mpx_circuit``)."""

    def __init__(self, engine: Engine, gen_words: np.ndarray, angles: np.ndarray):
        self.engine = engine
        gw = np.ascontiguousarray(gen_words, dtype=np.uint64)
        an = np.ascontiguousarray(angles, dtype=np.float64)
        if gw.ndim != 2 or gw.shape[0] != an.shape[0] or gw.shape[1] != engine.words:
            raise ValueError("gen_words must be [n_layers, W] and angles [n_layers]")
        self.n_layers = gw.shape[0]
        h = C.c_void_p()
        engine._check(engine.lib.mpx_circuit_upload(engine.h, _p(gw), _p(an), self.n_layers, C.byref(h)))
        self.h = h

    def set_angles(self, angles: np.ndarray) -> None:
        an = np.ascontiguousarray(angles, dtype=np.float64)
        if an.shape != (self.n_layers,):
            raise ValueError("angles must have one entry per layer")
        self.engine._check(self.engine.lib.mpx_circuit_set_angles(self.engine.h, self.h, _p(an)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.engine.lib.mpx_circuit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """One device-resident Heisenberg term store (``mpx_engine``)."""

    def __init__(self, *, basis: str, cutoff_type: str, cutoff: int, num_modes: int,
                 keys: np.ndarray, coefs: np.ndarray, core: float, state_mask: np.ndarray,
                 lower_atol: float | None = None, upper_atol: float | None = None, device: int = 0,
                 capacity_hint: int = 0, blocks_per_sm: int = 0, table_shift: int = 0,
                 schrodinger_cutoff: int | None = None):
        """``schrodinger_cutoff`` (slots): the Schrodinger picture -- the store starts as the paired
        reference-state monomials and ``keys``/``coefs`` is the observable dotted into the evolved state."""
        self.lib = load()
        cfg = Config(1 if basis == "pauli" else 0, 1 if cutoff_type == "support" else 0, int(cutoff),
                     int(lower_atol is not None), float(lower_atol or 0.0), int(upper_atol is not None),
                     float(upper_atol or 0.0), int(num_modes), int(device), int(capacity_hint),
                     int(blocks_per_sm), int(table_shift), int(schrodinger_cutoff is not None),
                     int(schrodinger_cutoff or 0), int(num_modes))
        self.words = (int(num_modes) + 31) // 32
        self.num_modes = int(num_modes)
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1, self.words)
        c = np.ascontiguousarray(coefs, dtype=np.float64).reshape(-1)
        m = np.ascontiguousarray(state_mask, dtype=np.uint64).reshape(-1)
        if k.shape[0] != c.shape[0]:
            raise ValueError("keys and coefs disagree in length")
        if m.shape[0] < self.words:
            m = np.concatenate([m, np.zeros(self.words - m.shape[0], np.uint64)])
        h = C.c_void_p()
        rc = self.lib.mpx_create(C.byref(cfg), _p(k) if k.size else None, _p(c) if c.size else None, k.shape[0],
                                 float(core), _p(m), C.byref(h))
        if rc != MPX_OK:
            msg = self.lib.mpx_last_error(None).decode()
            raise (MpxInvalid if rc == 1 else MpxError)(rc, msg)
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != MPX_OK:
            msg = self.lib.mpx_last_error(self.h).decode()
            raise (MpxInvalid if rc == 1 else MpxError)(rc, msg)

    def propagate(self, gen_words: np.ndarray, angles: np.ndarray) -> None:
        gw = np.ascontiguousarray(gen_words, dtype=np.uint64).reshape(-1, self.words)
        an = np.ascontiguousarray(angles, dtype=np.float64).reshape(-1)
        if gw.shape[0] != an.shape[0]:
            raise ValueError("one angle per generator is required")
        self._check(self.lib.mpx_propagate(self.h, _p(gw), _p(an), gw.shape[0]))

    def upload(self, gen_words: np.ndarray, angles: np.ndarray) -> Circuit:
        return Circuit(self, gen_words, angles)

    def propagate_circuit(self, circuit: Circuit) -> None:
        self._check(self.lib.mpx_propagate_circuit(self.h, circuit.h))

    def expectation(self) -> float:
        out = C.c_double(0.0)
        self._check(self.lib.mpx_expectation(self.h, C.byref(out)))
        return out.value

    def size(self) -> int:
        out = C.c_uint64(0)
        self._check(self.lib.mpx_size(self.h, C.byref(out)))
        return int(out.value)

    def export(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.size()
        keys = np.zeros((max(n, 1), self.words), dtype=np.uint64)
        coefs = np.zeros(max(n, 1), dtype=np.float64)
        got = C.c_uint64(0)
        self._check(self.lib.mpx_export(self.h, _p(keys), _p(coefs), n, C.byref(got)))
        return keys[:n], coefs[:n]

    def gate_stats(self) -> GateStats:
        n = C.c_uint64(0)
        self._check(self.lib.mpx_gate_stats(self.h, None, 0, C.byref(n)))
        out = np.zeros((max(int(n.value), 1), 4), dtype=np.uint64)
        self._check(self.lib.mpx_gate_stats(self.h, _p(out), int(n.value), C.byref(n)))
        out = out[: int(n.value)]
        return GateStats(out[:, 0].copy(), out[:, 1].copy(), out[:, 2].copy(), out[:, 3].copy())

    def reset(self) -> None:
        self._check(self.lib.mpx_reset(self.h))

    def set_cutoff(self, cutoff: int) -> None:
        self._check(self.lib.mpx_set_cutoff(self.h, int(cutoff)))

    def set_lower_atol(self, value: float | None) -> None:
        self._check(self.lib.mpx_set_lower_atol(self.h, int(value is not None), float(value or 0.0)))

    def set_upper_atol(self, value: float | None) -> None:
        self._check(self.lib.mpx_set_upper_atol(self.h, int(value is not None), float(value or 0.0)))

    def set_only_rotate_len_k(self, k: int | None) -> None:
        """only_rotate_len_k of the next propagate calls (None clears it)."""
        self._check(self.lib.mpx_set_only_rotate_len_k(self.h, 0 if k is None else int(k)))

    def set_basis_change(self, basis_change) -> None:
        """basis_change rows (one slot list per slot, 2 * num_modes of them), or None to clear."""
        if basis_change is None:
            self._check(self.lib.mpx_set_basis_change(self.h, None, 0))
            return
        from .encoding import basis_rows

        rows = np.ascontiguousarray(basis_rows(basis_change, self.num_modes)[: 2 * self.num_modes])
        self._check(self.lib.mpx_set_basis_change(self.h, _p(rows), rows.shape[0]))

    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self.lib.mpx_stream(self.h, C.byref(s)))
        return int(s.value or 0)

    def launch_count(self) -> int:
        out = C.c_uint64(0)
        self._check(self.lib.mpx_launch_count(self.h, C.byref(out)))
        return int(out.value)

    def graph_replay_count(self) -> int:
        """Propagations of a resident circuit that ran their streaming gates as one replayed CUDA graph."""
        out = C.c_uint64(0)
        self._check(self.lib.mpx_graph_replay_count(self.h, C.byref(out)))
        return int(out.value)

    def adjoint_logged(self) -> bool:
        """Whether the last adjoint_forward logged everything the reverse sweep needs (no segment replay)."""
        out = C.c_int32(0)
        self._check(self.lib.mpx_adjoint_logged(self.h, C.byref(out)))
        return bool(out.value)

    def adjoint_forward(self, circuit: Circuit, segment_gates: int = 0) -> float:
        """Reset, propagate ``circuit`` saving coefficient checkpoints every ``segment_gates`` gates; <O>."""
        out = C.c_double(0.0)
        self._check(self.lib.mpx_adjoint_forward(self.h, circuit.h, int(segment_gates), C.byref(out)))
        return out.value

    def adjoint_backward(self, circuit: Circuit) -> np.ndarray:
        """d<O>/d(angle_l) for every layer l of ``circuit`` (after :meth:`adjoint_forward`)."""
        out = np.zeros(max(circuit.n_layers, 1), dtype=np.float64)
        self._check(self.lib.mpx_adjoint_backward(self.h, circuit.h, _p(out)))
        return out[: circuit.n_layers]

    def graph_build(self, circuit: Circuit, segment_gates: int = 0) -> float:
        """Propagate ``circuit`` and keep its truncation structure (the frozen graph); <O>."""
        out = C.c_double(0.0)
        self._check(self.lib.mpx_graph_build(self.h, circuit.h, int(segment_gates), C.byref(out)))
        return out.value

    def graph_expectation(self, circuit: Circuit) -> float:
        """<O> of the frozen graph at ``circuit``'s current angles."""
        out = C.c_double(0.0)
        self._check(self.lib.mpx_graph_expectation(self.h, circuit.h, C.byref(out)))
        return out.value

    def graph_gradient(self, circuit: Circuit, segment_gates: int = 0) -> tuple[float, np.ndarray]:
        """<O> and d<O>/d(angle_l) of the frozen graph at ``circuit``'s current angles."""
        out = C.c_double(0.0)
        g = np.zeros(max(circuit.n_layers, 1), dtype=np.float64)
        self._check(self.lib.mpx_graph_gradient(self.h, circuit.h, int(segment_gates), C.byref(out), _p(g)))
        return out.value, g[: circuit.n_layers]

    def set_pair_log(self, capacity: int) -> None:
        """Pair log of the gradient forward pass: < 0 automatic, 0 off, > 0 that many records."""
        self._check(self.lib.mpx_set_pair_log(self.h, int(capacity)))

    def set_profiling(self, on: bool) -> None:
        self._check(self.lib.mpx_set_profiling(self.h, int(bool(on))))

    def kernel_times(self) -> tuple[float, float, float, int]:
        """(summed sweep, resolve and column-append ms, gates) of the last propagate call (profiling on)."""
        a, b, c, n = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0), C.c_uint64(0)
        self._check(self.lib.mpx_kernel_times(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(n)))
        return a.value, b.value, c.value, int(n.value)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mpx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def engine_for(wl, **kw) -> Engine:
    """Engine holding workload ``wl``'s observable (see :mod:`monoprop_b200.workloads`)."""
    keys, coefs, core = wl.encoded_observable()
    if wl.extra.get("schrodinger_cutoff") is not None:
        kw.setdefault("schrodinger_cutoff", int(wl.extra["schrodinger_cutoff"]))
    eng = Engine(basis=wl.basis, cutoff_type=wl.cutoff_type, cutoff=wl.cutoff, num_modes=wl.num_modes,
                 keys=keys, coefs=coefs, core=core, state_mask=wl.state_mask(), lower_atol=wl.lower_atol,
                 upper_atol=wl.upper_atol, **kw)
    if wl.extra.get("basis_change") is not None:  # a constructor argument of the reference propagator
        try:
            eng.set_basis_change(wl.extra["basis_change"])
        except Exception:
            eng.close()
            raise
    return eng
