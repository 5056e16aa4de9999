"""Batches of independent problems (mpx_batch_run) and the batch autotuner.

Every instance of a batch must give what it gives alone: <O> against the oracle (1e-10 relative), its
evolved store against the oracle's (keys bit-exact, coefficients 1e-10 relative), and with gradients the
single-instance adjoint's gradient, whatever the concurrency and tuning knobs. The depth-12 and depth-24
instances of the 256-instance batched workload are checked at full depth in test_gpu_full_depth.py.
"""

import numpy as np
import pytest

import oracle
from monoprop_b200 import workloads as W
from monoprop_b200.encoding import canonical_order
from monoprop_b200.autograd import DifferentiablePropagation
from monoprop_b200.batch import Autotuner, BatchConfig, run_batch

pytestmark = pytest.mark.gpu


def small_batch(n=12, seed=3):
    rng = np.random.default_rng(seed)
    return [W.ising50(int(d), seed=100 + i, observable_qubit=int(q))
            for i, (d, q) in enumerate(zip(rng.integers(1, 4, size=n), rng.integers(0, 50, size=n)))]


def _same_store(keys, coefs, ref):
    """Keys bit-exact and coefficients within 1e-10 relative of the oracle's, whatever the storage order."""
    ia, ib = canonical_order(keys), canonical_order(ref.keys)
    assert keys.shape == ref.keys.shape and np.array_equal(keys[ia], ref.keys[ib]), "monomial sets differ"
    a, b = coefs[ia], ref.coefs[ib]
    assert np.all(np.abs(a - b) <= 1e-10 * np.maximum(np.abs(a), np.abs(b)) + 1e-15)


@pytest.mark.parametrize("cfg", [BatchConfig(1, 0, 0), BatchConfig(8, 2, 2), BatchConfig(16, 4, 1)])
def test_batch_matches_single_instances(cfg):
    batch = small_batch()
    refs = [oracle.run_port(wl) for wl in batch]
    r = run_batch(batch, cfg, export_caps=[ref.keys.shape[0] + 8 for ref in refs])
    for ref, ev, n, (keys, coefs) in zip(refs, r.expectations, r.final_terms, r.exports):
        assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))
        assert int(n) == ref.keys.shape[0]
        _same_store(keys, coefs, ref)


def test_batch_of_uneven_depths_4_to_6_matches_oracle():
    """Instances of the batched workload's family at depths 4..6 (2.6e5 to ~5e6 terms each): every
    instance's evolved store against the oracle's, key for key."""
    rng = np.random.default_rng(21)
    batch = [W.ising50(int(d), seed=500 + i, observable_qubit=int(q))
             for i, (d, q) in enumerate(zip(rng.integers(4, 7, size=5), rng.integers(0, 50, size=5)))]
    refs = [oracle.run_port(wl) for wl in batch]
    r = run_batch(batch, BatchConfig(4), export_caps=[ref.keys.shape[0] + 8 for ref in refs])
    for ref, ev, (keys, coefs) in zip(refs, r.expectations, r.exports):
        assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))
        _same_store(keys, coefs, ref)


def test_batch_gradients_match_single_instance():
    batch = small_batch(6, seed=9)
    r = run_batch(batch, BatchConfig(4), gradient=True, segment_gates=135)
    for wl, ev, g in zip(batch, r.expectations, r.grads):
        dp = DifferentiablePropagation(wl, segment_gates=135)
        ev1 = dp.forward_value(wl.params)
        ga = dp.engine.adjoint_backward(dp.circuit)
        dp.close()
        assert abs(ev - ev1) <= 1e-13 * max(1.0, abs(ev1))
        assert np.max(np.abs(g - ga)) <= 1e-12 * max(1.0, np.max(np.abs(ga)))


def test_autotuner_picks_a_measured_configuration(tmp_path):
    batch = small_batch(16, seed=5)
    tuner = Autotuner(cache_path=str(tmp_path / "tune.json"), sample=6, validate=12)
    best, entry = tuner.tune(batch)
    assert len(entry["table"]) == len(Autotuner.WORKERS) * len(Autotuner.BLOCKS_PER_SM) * len(Autotuner.TABLE_SHIFT)
    # second stage: the three fastest of the first and the defaults, re-timed on 12 instances
    keys = ("workers", "blocks_per_sm", "table_shift")
    val = entry["validation"]
    assert entry["validation_sample"] == 12 and BatchConfig().as_dict() in [{k: r[k] for k in keys} for r in val]
    top = sorted(entry["table"], key=lambda row: row["seconds"])[: Autotuner.FINALISTS]
    assert all({k: r[k] for k in keys} in [{k: v[k] for k in keys} for v in val] for r in top)
    fastest = min(val, key=lambda row: row["seconds"])
    assert best == BatchConfig(**{k: fastest[k] for k in keys})
    again, _ = tuner.tune(batch)  # served from the cache
    assert again == best
    r = run_batch(batch, best)
    for wl, ev in zip(batch, r.expectations):
        ref = oracle.run_port(wl)
        assert abs(ev - ref.expectation) <= 1e-10 * max(1.0, abs(ref.expectation))
