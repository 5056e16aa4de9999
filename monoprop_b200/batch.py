"""Batches of independent propagation problems on one GPU (``mpx_batch_run``) and their autotuner.

A batch is a list of :class:`~monoprop_b200.workloads.Workload` sharing the basis, key width and
truncation settings (observables, angles and depths may all differ). :func:`run_batch` hands the whole
batch to the engine in one call; the engine spreads it over ``workers`` concurrent instances (host
threads, each with its own CUDA stream), deepest first, with memory admission.

:class:`Autotuner` picks the batch knobs by measurement: concurrency (``workers``), the per-gate kernel
grid (``blocks_per_sm``) and the hash-table load factor (``table_shift``). It times each candidate on a
calibration sample of the batch and caches the winner per (device, workload signature) in a JSON file.
"""

from __future__ import annotations

import ctypes as C
import itertools
import json
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _native


class _Item(C.Structure):
    _fields_ = [("obs_words", C.c_void_p), ("obs_coef", C.c_void_p), ("n_obs", C.c_uint64), ("core", C.c_double),
                ("state_mask", C.c_void_p), ("gen_words", C.c_void_p), ("angles", C.c_void_p),
                ("n_layers", C.c_uint64), ("expectation", C.c_void_p), ("grad_angles", C.c_void_p),
                ("final_terms", C.c_void_p), ("export_words", C.c_void_p), ("export_coefs", C.c_void_p),
                ("export_cap", C.c_uint64), ("export_n", C.c_void_p)]


class _Options(C.Structure):
    _fields_ = [("workers", C.c_int32), ("gradient", C.c_int32), ("segment_gates", C.c_uint64)]


@dataclass
class BatchConfig:
    workers: int = 8
    blocks_per_sm: int = 0  # 0 = engine default (4)
    table_shift: int = 0  # 0 = engine default (1: load factor <= 1/2)

    def as_dict(self) -> dict:
        return {"workers": self.workers, "blocks_per_sm": self.blocks_per_sm, "table_shift": self.table_shift}


@dataclass
class BatchResult:
    expectations: np.ndarray
    grads: list[np.ndarray] | None  # d<O>/d(angle_l) per instance (gradient runs)
    final_terms: np.ndarray
    seconds: float
    exports: list[tuple[np.ndarray, np.ndarray]] | None = None  # raw (keys, coefs) per instance, on request


def run_batch(workloads, config: BatchConfig | None = None, gradient: bool = False, segment_gates: int = 0,
              device: int = 0, export_caps=None) -> BatchResult:
    """Propagate every workload (and its adjoint gradient when ``gradient``) in one engine call.

    ``export_caps``: per instance, the number of terms of room for a raw export of its evolved store
    (keys and coefficients in storage order); the result's ``exports`` then holds them."""
    config = config or BatchConfig()
    lib = _native.load()
    if not workloads:
        return BatchResult(np.zeros(0), [] if gradient else None, np.zeros(0, np.uint64), 0.0)
    w0 = workloads[0]
    for wl in workloads:
        if (wl.basis, wl.words, wl.cutoff, wl.cutoff_type, wl.lower_atol, wl.upper_atol) != \
                (w0.basis, w0.words, w0.cutoff, w0.cutoff_type, w0.lower_atol, w0.upper_atol):
            raise ValueError("batch workloads must share basis, key width and truncation settings")
    cfg = _native.Config(1 if w0.basis == "pauli" else 0, 1 if w0.cutoff_type == "support" else 0, int(w0.cutoff),
                         int(w0.lower_atol is not None), float(w0.lower_atol or 0.0), int(w0.upper_atol is not None),
                         float(w0.upper_atol or 0.0), int(w0.num_modes), int(device), 0, int(config.blocks_per_sm),
                         int(config.table_shift))
    n = len(workloads)
    items = (_Item * n)()
    keep = []
    ev = np.zeros(n, dtype=np.float64)
    terms = np.zeros(n, dtype=np.uint64)
    grads = [np.zeros(wl.n_layers, dtype=np.float64) for wl in workloads] if gradient else None
    exp_bufs = None
    if export_caps is not None:
        exp_bufs = [(np.zeros((max(int(c), 1), w0.words), np.uint64), np.zeros(max(int(c), 1)), np.zeros(1, np.uint64))
                    for c in export_caps]
    for i, wl in enumerate(workloads):
        keys, coefs, core = wl.encoded_observable()
        arrs = (np.ascontiguousarray(keys, np.uint64), np.ascontiguousarray(coefs, np.float64),
                np.ascontiguousarray(wl.state_mask(), np.uint64), np.ascontiguousarray(wl.gen_words(), np.uint64),
                np.ascontiguousarray(wl.angles(), np.float64))
        keep.append(arrs)
        it = items[i]
        it.obs_words, it.obs_coef = arrs[0].ctypes.data, arrs[1].ctypes.data
        it.n_obs, it.core = arrs[0].shape[0], float(core)
        it.state_mask, it.gen_words, it.angles = arrs[2].ctypes.data, arrs[3].ctypes.data, arrs[4].ctypes.data
        it.n_layers = wl.n_layers
        it.expectation = ev.ctypes.data + 8 * i
        it.final_terms = terms.ctypes.data + 8 * i
        it.grad_angles = grads[i].ctypes.data if gradient and wl.n_layers else None
        if exp_bufs is not None:
            kb, cb, nb = exp_bufs[i]
            it.export_words, it.export_coefs, it.export_n = kb.ctypes.data, cb.ctypes.data, nb.ctypes.data
            it.export_cap = int(export_caps[i])
    opt = _Options(int(config.workers), int(gradient), int(segment_gates))
    err = C.create_string_buffer(1024)
    t0 = time.perf_counter()
    rc = lib.mpx_batch_run(C.byref(cfg), C.cast(items, C.c_void_p), n, C.byref(opt), err, 1024)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise _native.MpxError(rc, err.value.decode())
    exports = None
    if exp_bufs is not None:
        exports = []
        for (kb, cb, nb), cap in zip(exp_bufs, export_caps):
            k = min(int(nb[0]), int(cap))
            exports.append((kb[:k], cb[:k]))
    return BatchResult(ev, grads, terms, dt, exports)


def shard_instances(workloads, rank: int, world: int) -> list[int]:
    """Indices of the instances rank ``rank`` of ``world`` propagates when a batch is split over GPUs (no
    data-path collective: instances are independent). Instances are dealt deepest first, round robin, so
    every rank gets a near-equal number of gates: the ranks' totals differ by at most one instance depth."""
    order = sorted(range(len(workloads)), key=lambda i: (-workloads[i].n_layers, i))
    return order[rank::world]


def signature(workloads) -> str:
    """Workload family key for the tuning cache: basis, key width, truncation, size of the batch."""
    w0 = workloads[0]
    depths = sorted(wl.n_layers for wl in workloads)
    return (f"{w0.basis}-W{w0.words}-c{w0.cutoff}-{w0.cutoff_type}-l{w0.lower_atol}-u{w0.upper_atol}-"
            f"n{len(workloads)}-L{depths[0]}..{depths[-1]}")


class Autotuner:
    """Measures batch knob combinations on a calibration sample, then re-times the fastest few and the
    defaults on a larger sample, and keeps the fastest there.

    The second stage exists because a small sample under-rewards concurrency: with about as many instances
    as workers, the batch's pipelined steady state never forms (measured on 256 instances of the batched
    50-qubit workload: 4 workers were fastest on 24 sampled instances, 86.8 s on the whole batch against
    71.9 s for the defaults' 8)."""

    WORKERS = (1, 4, 8, 16)
    BLOCKS_PER_SM = (2, 4)
    TABLE_SHIFT = (1, 2)
    FINALISTS = 3

    def __init__(self, cache_path: str | None = None, sample: int = 24, seed: int = 0, validate: int = 64):
        self.cache_path = cache_path or os.path.join(os.path.expanduser("~"), ".cache", "monoprop_b200",
                                                     "autotune.json")
        self.sample = sample
        self.validate = validate
        self.seed = seed

    def _load(self) -> dict:
        try:
            with open(self.cache_path) as f:
                return json.load(f)
        except (OSError, ValueError):
            return {}

    def _store(self, cache: dict) -> None:
        os.makedirs(os.path.dirname(self.cache_path), exist_ok=True)
        with open(self.cache_path, "w") as f:
            json.dump(cache, f, indent=1)

    def calibration_sample(self, workloads, size: int | None = None) -> list:
        """A depth-stratified sample of ``size`` instances (default: the first stage's): the batch sorted by
        depth, every k-th instance."""
        size = self.sample if size is None else size
        order = sorted(range(len(workloads)), key=lambda i: workloads[i].n_layers)
        k = max(1, len(order) // size)
        return [workloads[i] for i in order[::k][:size]]

    def tune(self, workloads, gradient: bool = False, segment_gates: int = 0, device: int = 0,
             use_cache: bool = True) -> tuple[BatchConfig, dict]:
        """Best configuration for this batch family and the timing table it was chosen from."""
        key = f"dev{device}:{signature(workloads)}:grad{int(gradient)}"
        cache = self._load() if use_cache else {}
        if key in cache:
            return BatchConfig(**cache[key]["best"]), cache[key]
        sample = self.calibration_sample(workloads)
        run_batch(sample[:2], BatchConfig(), gradient, segment_gates, device)  # warm the engine and the pool
        table = []
        for workers, bps, shift in itertools.product(self.WORKERS, self.BLOCKS_PER_SM, self.TABLE_SHIFT):
            cfg = BatchConfig(workers, bps, shift)
            r = run_batch(sample, cfg, gradient, segment_gates, device)
            table.append({**cfg.as_dict(), "seconds": r.seconds})
        best = min(table, key=lambda row: row["seconds"])
        validation = []
        vsample = self.calibration_sample(workloads, self.validate)
        if len(vsample) > len(sample):
            keys = ("workers", "blocks_per_sm", "table_shift")
            finalists = [BatchConfig(**{k: row[k] for k in keys})
                         for row in sorted(table, key=lambda row: row["seconds"])[: self.FINALISTS]]
            if BatchConfig() not in finalists:
                finalists.append(BatchConfig())
            for cfg in finalists:
                r = run_batch(vsample, cfg, gradient, segment_gates, device)
                validation.append({**cfg.as_dict(), "seconds": r.seconds})
            best = min(validation, key=lambda row: row["seconds"])
        entry = {"best": {k: best[k] for k in ("workers", "blocks_per_sm", "table_shift")}, "table": table,
                 "sample": len(sample), "validation": validation, "validation_sample": len(vsample)}
        cache[key] = entry
        if use_cache:
            self._store(cache)
        return BatchConfig(**entry["best"]), entry
