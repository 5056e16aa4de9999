"""Host-side logic that needs no GPU: the bench's max-over-ranks timing on two gloo ranks, the batch
API's argument checks and the autotuner's sampling."""

import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from monoprop_b200 import _native
from monoprop_b200 import workloads as W
from monoprop_b200.batch import Autotuner, signature


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    out[rank] = bench.max_over_ranks(10.0 + rank, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert out[0] == out[1] == 11.0


def _shard_main(rank, world, port, out):
    import torch.distributed as dist

    from monoprop_b200.batch import shard_instances

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    full = W.batch_ising50(40, seed=4)
    mine = shard_instances(full, rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_batch_instance_split_two_gloo_ranks():
    """The multi-GPU batch split (bench.py --workload batch under torchrun): two ranks take disjoint
    shares that cover every instance once, with gate totals within one instance depth of each other."""
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    shares = out[0]
    assert out[1] == shares
    full = W.batch_ising50(40, seed=4)
    assert sorted(shares[0] + shares[1]) == list(range(40)) and not set(shares[0]) & set(shares[1])
    gates = [sum(full[i].n_layers for i in s) for s in shares]
    assert abs(gates[0] - gates[1]) <= max(wl.n_layers for wl in full)


def test_batch_run_rejects_null_buffers_without_touching_a_device():
    lib = _native.load()
    cfg = _native.Config(1, 1, 4, 0, 0.0, 0, 0.0, 8, 0, 0, 0, 0)
    err = C.create_string_buffer(256)
    rc = lib.mpx_batch_run(C.byref(cfg), None, 3, None, err, 256)
    assert rc == 1 and b"NULL" in err.value


def test_batch_run_rejects_a_device_it_cannot_use():
    """An out-of-range device ordinal (or no device at all) is a non-OK status with a message, never a
    silent MPX_OK with unwritten results."""
    from monoprop_b200.batch import _Item, _Options

    lib = _native.load()
    cfg = _native.Config(1, 1, 4, 0, 0.0, 0, 0.0, 8, 999, 0, 0, 0)
    ev = np.full(1, np.nan)
    gw = np.zeros((1, 1), np.uint64)
    an = np.zeros(1)
    items = (_Item * 1)()
    items[0].expectation, items[0].gen_words, items[0].angles, items[0].n_layers = (ev.ctypes.data, gw.ctypes.data,
                                                                                   an.ctypes.data, 1)
    opt = _Options(2, 0, 0)
    err = C.create_string_buffer(256)
    rc = lib.mpx_batch_run(C.byref(cfg), C.cast(items, C.c_void_p), 1, C.byref(opt), err, 256)
    assert rc in (1, 6) and err.value  # MPX_ERR_INVALID (ordinal out of range) or MPX_ERR_NO_DEVICE
    assert np.isnan(ev[0])


def test_autotuner_sample_is_depth_stratified():
    batch = W.batch_ising50(40, seed=4)
    sample = Autotuner(cache_path="/nonexistent/x.json", sample=8).calibration_sample(batch)
    depths = sorted(wl.n_layers for wl in batch)
    got = sorted(wl.n_layers for wl in sample)
    assert len(sample) == 8 and got[0] == depths[0] and got[-1] >= depths[len(depths) * 3 // 4]
    assert signature(batch).startswith("pauli-W2-c8-support")


def test_autotuner_second_stage_overrules_the_small_sample(tmp_path, monkeypatch):
    """The tuner's choice comes from the second stage: the three fastest configurations of the small sample
    and the defaults, re-timed on the larger one. Here a fake batch runner makes few workers win on the
    small sample and lose on the large one (as measured on the 256-instance batched workload), so the
    defaults must be chosen; the choice is cached."""
    from monoprop_b200 import batch as B

    calls = []

    class _R:
        def __init__(self, seconds):
            self.seconds = seconds

    def fake_run(sample, cfg, gradient=False, segment_gates=0, device=0):
        calls.append((len(sample), cfg))
        if len(sample) <= 6:  # small sample: fewer workers look faster
            return _R(1.0 + 0.1 * cfg.workers + 0.01 * cfg.blocks_per_sm + 0.001 * cfg.table_shift)
        return _R(10.0 / max(cfg.workers, 1))  # large sample: concurrency pays

    monkeypatch.setattr(B, "run_batch", fake_run)
    batch = W.batch_ising50(40, seed=4)
    tuner = B.Autotuner(cache_path=str(tmp_path / "t.json"), sample=6, validate=24)
    best, entry = tuner.tune(batch)
    assert len(entry["table"]) == len(B.Autotuner.WORKERS) * len(B.Autotuner.BLOCKS_PER_SM) * len(B.Autotuner.TABLE_SHIFT)
    finalists = [(r["workers"], r["blocks_per_sm"], r["table_shift"]) for r in entry["validation"]]
    assert finalists[:3] == [(1, 2, 1), (1, 2, 2), (1, 4, 1)] and (8, 0, 0) in finalists
    assert entry["validation_sample"] == 24 and best == B.BatchConfig()
    n_calls = len(calls)
    again, _ = tuner.tune(batch)  # from the cache: nothing re-timed
    assert again == best and len(calls) == n_calls


def test_basis_rows_encoding():
    """basis_change rows: one row per slot, listed slots set once (indices_to_bitset_checked), zero rows
    above 2 * num_modes, the reference's row-count message."""
    import numpy as np
    import pytest

    from monoprop_b200.encoding import basis_rows, slots_to_words

    n = 6
    rows = basis_rows([[s] if s % 2 == 0 else [s - 1, s, s] for s in range(2 * n)], n)
    assert rows.shape == (64, 1)
    assert np.array_equal(rows[3], slots_to_words([2, 3], n))  # the duplicate 3 is set, not cancelled
    assert not rows[2 * n:].any()
    with pytest.raises(ValueError, match="basis_change must have exactly 2\\*logical_num_modes \\(12\\) rows"):
        basis_rows([[0]] * 5, n)


def test_reference_arm_json_line():
    """bench.py --impl reference: one JSON line on the bench's metric, with the reference-arm keys
    (impl, cpu_baseline describing the run, e2e with no host-device bytes)."""
    import json
    import os
    import subprocess
    import sys

    import pytest

    import oracle

    if not oracle.ref_available():
        pytest.skip("reference oracle not built here")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--workload",
                          "line20", "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1])
    assert d["impl"] == "reference" and d["metric"] == "term-gate updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
