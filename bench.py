"""Benchmark of the Heisenberg propagation hot path on B200: term-gate updates per second.

Workload (one "step"): the 10x10 kicked-Ising circuit (100 qubits, 20 layers of RZZ on the 180 lattice
edges then RX on the 100 sites = 5600 gates, angles U[0, 0.3 pi) from seed 1234), observable
(1/100) sum_i Z_i, Pauli weight <= 10, lower_atol 1e-5, FP64, propagated in full from the initial
observable. A term-gate update is one term present in the store when one gate is applied; the rate is
sum_g n_g / time.

* ``value``: device time (CUDA events on the engine's stream) of ``mpx_propagate_circuit`` with the circuit
  and the initial store already resident in HBM; the store is reset (untimed) before every step and L2 is
  flushed (a 256 MiB write) between steps.
* ``e2e``: the same rate through the public C ABI with host buffers, per step: ``mpx_create`` from the host
  observable, ``mpx_propagate`` from the host circuit arrays (host-to-device copy inside), ``mpx_expectation``
  (device-to-host read of <O>), ``mpx_destroy``.
* ``roofline``: the sweep kernel (the per-gate anticommutation scan over every stored term). Its
  algorithmic bytes per launch are what the bit-column scan must move: ``(f_g + 1) n_g / 8`` (the f_g
  fold columns read, the leader-emitted bitmap written) ``+ 16 a_g`` (read+write of every anticommuting
  coefficient) ``+ (8W + 13) e_g`` (key rows of the emitted terms, the query records written), over its
  event-timed duration, against the measured HBM copy bandwidth. ``path_frac`` is the whole path against
  the row-store formula ``sum_g 8W n_g + 16 a_g + (8W + 8) m_g`` over the device step time; the column
  index lets the path move fewer bytes than that formula, so ``path_frac`` can exceed 1.
* ``cpu_baseline``: the unmodified reference engine (compiled from its own sources into
  ``oracle/_ref/libmpref.so``) propagating the same circuit on the host cores.
* ``gradient``: <O> and the gradient of all 5600 angles per second, two ways: the engine's adjoint of the
  propagation (``mpx_adjoint_forward`` / ``_backward``) and, under ``graph``, the frozen structure of the
  reference's variational loop (``mpx_graph_build`` once, then ``mpx_graph_gradient`` per call, what
  ``_core.expectation_value_and_gradient`` runs); ``cpu_reference`` is the reference's own build_graph +
  expectation_value_and_gradient on the host cores.

``--impl reference`` times that reference engine alone on the same workload and prints its own line.
Multi-GPU (``--gpus N`` under torchrun): N independent replicas of the workload, one per GPU (the
single-operator path has no partitioned form yet); value = all ranks' updates / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def _peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"mpx_clocks_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import datetime

    import torch.distributed as dist

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    return rank, ws, local, dist


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's ``value`` (timings are reported as the slowest rank's); every rank
    takes part in the same collective."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


_REF_BUILD = None


def ref_build() -> str:
    """The reference build this host's CPU runs as the reference's stock -march=native build would
    (oracle.native_ref_build), chosen once per process."""
    global _REF_BUILD
    if _REF_BUILD is None:
        import oracle

        _REF_BUILD = oracle.native_ref_build()
    return _REF_BUILD


def time_reference(wl, steps: int, warmup: int, partitions: int) -> dict:
    """The unmodified reference engine on the host cores: per step, one full propagate of ``wl``.

    Partition count: all host threads, or 1 when that is faster (small workloads, where the partition
    exchange costs more than it saves; decided on full runs during warm-up when one takes < 1 s)."""
    import oracle

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libmpref.so is missing (build it with oracle/build_ref.sh)")
    build = ref_build()

    def run(p, n_layers=None):
        eng = oracle.RefEngine(wl, partitions=p, build=build)
        t = eng.propagate(n_layers=n_layers)
        eng.close()
        return t

    # Warm-up: a 400-gate prefix per warm-up step (pages the library and allocator in; CPU code has no JIT).
    for _ in range(warmup):
        run(partitions, min(400, wl.n_layers))
    chosen = partitions
    if partitions > 1 and run(partitions) < 1.0 and run(1) < run(partitions):
        chosen = 1
    secs = [run(chosen) for _ in range(steps)]
    return {"seconds": secs, "partitions": chosen, "build": build}


def time_reference_gradient(wl, partitions: int, evals: int = 1) -> dict:
    """The reference's <O> + full gradient: build_graph once at the workload's parameters
    (MonomialPropagator.inl:620-690), then ``evals`` calls of expectation_value_and_gradient
    (MPFunctions.cpp:207-246) on all host threads."""
    import oracle

    build = ref_build()
    eng = oracle.RefEngine(wl, partitions=partitions, build=build)
    try:
        t_build = eng.propagate(build_graph=True)
        secs = [eng.expectation_and_gradient(wl.params)[2] for _ in range(evals)]
    finally:
        eng.close()
    return {"value": len(secs) / sum(secs), "unit": "gradients/s", "seconds_per_eval": sum(secs) / len(secs),
            "build_graph_seconds": t_build, "cores": partitions, "kind": "reference", "build": build,
            "sample": f"build_graph once, then {evals} expectation_value_and_gradient call(s), partitions={partitions}"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mpx", choices=["mpx", "reference"])
    ap.add_argument("--workload", default="ising100", choices=["ising100", "line20", "hubbard6x6", "batch"])
    ap.add_argument("--batch-instances", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-partitions", type=int, default=0, help="reference partitions (0: all host threads)")
    ap.add_argument("--kernel-case", type=int, default=0,
                    help="profiling case instead of the benchmark: a store of this many random 100-qubit terms of "
                         "Pauli weight <= 10, then the last --case-gates gates of the 10x10 circuit")
    ap.add_argument("--case-gates", type=int, default=4)
    ap.add_argument("--regime-case", type=int, default=0,
                    help="profiling case in the benchmark's own regime: the 10x10 circuit propagated until the store "
                         "holds this many terms, then --case-gates more gates inside the NVTX range mpx_profile")
    ap.add_argument("--profile-kernels", action="store_true",
                    help="profiling case for the other kernels (shared-memory path, expectation, columns, table "
                         "build, frozen replay and adjoint), each inside an NVTX range named after it")
    ap.add_argument("--no-gradient", action="store_true", help="skip the <O> + full-gradient measurement")
    ap.add_argument("--no-sub-results", action="store_true",
                    help="skip the compact measurements of the 20-qubit line and 6x6 Hubbard circuits")
    ap.add_argument("--segment-layers", type=int, default=4,
                    help="gradient checkpoint interval in circuit layers (the circuit repeats one layer of gates)")
    args = ap.parse_args()
    if args.kernel_case:
        kernel_case(args.kernel_case, args.case_gates)
        return
    if args.regime_case:
        regime_case(args.regime_case, args.case_gates)
        return
    if args.profile_kernels:
        profile_kernels()
        return
    if args.workload == "batch":
        batch_bench(args)
        return
    if args.warmup < 3:
        args.warmup = 3

    from monoprop_b200 import workloads as WL

    if args.workload == "batch" and args.impl == "reference":
        batch_reference(args)
        return
    wl = WL.BY_NAME[args.workload]()
    rank, world, local, dist = _dist()
    cores = args.cpu_partitions or _cpu_threads()
    config = {"workload": f"{wl.name}: {wl.num_modes} modes, {wl.n_layers} gates, {wl.basis}, cutoff {wl.cutoff}, "
                          f"lower_atol {wl.lower_atol}", "n_gates": wl.n_layers, "words": wl.words,
              "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
              "kernel_times": "separate event-bracketed steps after the timed ones"}

    if args.impl == "reference":
        if rank != 0:
            return
        t = time_reference(wl, args.steps, args.warmup, cores)
        updates = _updates(wl)
        secs = t["seconds"]
        v = updates * len(secs) / sum(secs)
        line = {"metric": "term-gate updates/s", "value": v, "unit": "updates/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded circuit)", "config": config, "impl": "reference",
                "cpu_baseline": {"value": v, "unit": "updates/s", "cores": cores, "kind": "reference",
                                 "build": t["build"],
                                 "sample": f"full {wl.name} propagate per step, partitions={t['partitions']}, "
                                           f"reference built for the host CPU ({t['build']})"},
                "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if not args.no_gradient:
            line["gradient"] = time_reference_gradient(wl, cores)
        print(json.dumps(line), flush=True)
        return

    import torch

    from monoprop_b200 import _native

    torch.cuda.set_device(local)
    if dist is not None:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    gw = wl.gen_words()
    ang = wl.angles()
    keys, coefs, core = wl.encoded_observable()

    eng = _native.engine_for(wl, device=local)
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)
    circ = eng.upload(gw, ang)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def one_step(profile: bool):
        eng.reset()
        with torch.cuda.stream(stream):
            flush.fill_(1)
        eng.set_profiling(profile)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.propagate_circuit(circ)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    for _ in range(args.warmup):
        one_step(False)
    stats = eng.gate_stats()
    updates = stats.term_gate_updates
    n, anti, app = stats.n.astype(np.float64), stats.anti.astype(np.float64), stats.appended.astype(np.float64)
    emitted = stats.emitted.astype(np.float64)
    W = wl.words
    gpop = np.array([sum(bin(int(x)).count("1") for x in row) for row in gw], dtype=np.float64)
    fold = gpop + ((gpop % 2 == 1) if wl.basis == "majorana" else 0)  # + the |M|-parity column
    fold = fold[::-1]  # gates are applied last to first; stats are in application order
    sweep_bytes = float(((fold + 1) * n / 8 + 16 * anti + (8 * W + 13) * emitted).sum())
    path_bytes = float((8 * W * n + 16 * anti + (8 * W + 8) * app).sum())

    launches0 = eng.launch_count()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms = []
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("bench_step")  # what a kernel profiler selects for the launch list
        for _ in range(args.steps):
            ms.append(one_step(False))
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = eng.launch_count() - launches0
    graph_replays = eng.graph_replay_count()
    # Per-kernel device times from the same number of steps again, each kernel launch bracketed by CUDA
    # events on the engine stream (the events themselves cost time, so these steps are not the value).
    sweep_ms, resolve_ms = [], []
    for _ in range(args.steps):
        one_step(True)
        s_ms, r_ms, _, _ = eng.kernel_times()
        sweep_ms.append(s_ms)
        resolve_ms.append(r_ms)
    total_ms = max_over_ranks(sum(ms), dist, dev)
    ms_per_step = total_ms / args.steps
    value = updates * world / (ms_per_step * 1e-3)
    ev_dev = eng.expectation()

    # <O> + full gradient per second: forward with coefficient checkpoints every --segment-layers circuit
    # layers, then the adjoint sweep (same engine, circuit resident), against the plain forward above.
    # The first calls grow the tape and replay buffers (measured 560-720 ms backward against ~280 ms once
    # they are sized), so the gradient gets the same untimed warm-up calls as the propagate steps.
    grad_line = None
    if not args.no_gradient:
        seg = args.segment_layers * wl.extra.get("gates_per_layer", wl.n_layers)
        eng.set_profiling(False)
        g_ms = []
        g_warm = max(1, args.warmup)
        for i in range(g_warm + args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ev_g = eng.adjoint_forward(circ, seg)
            grad = eng.adjoint_backward(circ)
            b.record(stream)
            b.synchronize()
            if i >= g_warm:
                g_ms.append(a.elapsed_time(b))
        g_total = max_over_ranks(sum(g_ms), dist, dev)
        g_per = g_total / len(g_ms)
        grad_line = {"metric": "<O>+full-gradient/s", "value": world * 1e3 / g_per, "unit": "gradients/s",
                     "ms_per_eval": g_per, "forward_ms": ms_per_step, "cost_vs_forward": g_per / ms_per_step,
                     "warmup": g_warm, "segment_gates": seg, "n_angles": int(wl.n_layers), "expectation": ev_g,
                     "grad_abs_max": float(np.max(np.abs(grad)))}
        # The variational loop as the reference runs it (its gradient leg below times the same two calls):
        # build the frozen structure once, then <O> + gradient of the replayed structure per call (what
        # _core.expectation_value_and_gradient runs).
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.graph_build(circ)
        b.record(stream)
        b.synchronize()
        build_ms = max_over_ranks(a.elapsed_time(b), dist, dev)
        gg_ms = []
        for i in range(g_warm + args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ev_gg, _ = eng.graph_gradient(circ)
            b.record(stream)
            b.synchronize()
            if i >= g_warm:
                gg_ms.append(a.elapsed_time(b))
        gg_per = max_over_ranks(sum(gg_ms), dist, dev) / len(gg_ms)
        grad_line["graph"] = {"value": world * 1e3 / gg_per, "unit": "gradients/s", "ms_per_eval": gg_per,
                              "build_graph_ms": build_ms, "cost_vs_forward": gg_per / ms_per_step,
                              "expectation": ev_gg}

    # The other two circuits of the task (the 20-qubit line and the 6x6 Hubbard circuit), measured the same
    # way on this GPU (one rank only: no collective takes part).
    sub_results = []
    if world == 1 and not args.no_sub_results:
        for name in ("line20", "hubbard6x6"):
            sub_results.append(measure_compact(WL.BY_NAME[name](), max(args.steps, 5), args.warmup, local, flush))

    # End to end through the C ABI with host buffers (create + propagate + expectation + destroy).
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2 = _native.engine_for(wl, device=local)
        e2.propagate(gw, ang)
        ev2 = e2.expectation()
        e2.close()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_ms.append(dt * 1e3)
    e2e_total = max_over_ranks(sum(e2e_ms), dist, dev)
    e2e = updates * world / (e2e_total / args.steps * 1e-3)
    h2d = int(gw.nbytes + ang.nbytes + keys.nbytes + coefs.nbytes)

    peak, peak_kind = _peaks()
    sweep_avg_s = statistics.mean(sweep_ms) * 1e-3
    achieved = sweep_bytes / sweep_avg_s / 1e9
    roofline = {"bound": "hbm", "kernel": "k_sweep", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                "traffic": None, "algorithmic_bytes_per_launch": sweep_bytes / wl.n_layers,
                "avg_launch_us": sweep_avg_s / wl.n_layers * 1e6,
                "kernel_ms_per_step": {"k_sweep": statistics.mean(sweep_ms), "k_resolve": statistics.mean(resolve_ms)},
                "path_bytes_per_step": path_bytes,
                # the sweep's binding resource: random 32-byte DRAM sectors (each anticommuting coefficient is
                # read and written once, each emitted term's key row read), per second of sweep time
                "random_sectors_per_s": float((2 * anti + np.ceil(W / 4) * emitted).sum()) / (statistics.mean(sweep_ms) * 1e-3),
                # per step: anticommuting terms (cos-scaled), emitted sine branches, appended partners
                "anticommuting_per_step": int(anti.sum()), "emitted_per_step": int(emitted.sum()),
                "appended_per_step": int(app.sum()),
                "path_frac": path_bytes / (ms_per_step * 1e-3) / 1e9 / peak}
    # DRAM bytes per launch: the ncu-measured traffic/algorithmic ratio of the sweep (captured on this
    # circuit itself at 8.0e6 terms, `--regime-case`), scaled to the average launch's algorithmic bytes.
    traffic_file = os.path.join(ROOT, "profiles", "k_sweep_traffic.json")
    if os.path.exists(traffic_file):
        with open(traffic_file) as f:
            ratio = json.load(f)["traffic_over_algorithmic"]
        roofline["traffic"] = ratio * sweep_bytes / wl.n_layers
        roofline["traffic_source"] = "ncu ratio from profiles/k_sweep_traffic.json x algorithmic bytes"

    if dist is not None:
        dist.barrier()
    if rank != 0:
        eng.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle

        if oracle.ref_available():
            t = time_reference(wl, 1, 0, cores)
            secs = t["seconds"]
            cpu = {"value": updates / secs[0], "unit": "updates/s", "cores": cores, "kind": "reference",
                   "build": t["build"],
                   "sample": f"one full {wl.name} propagate (all {wl.n_layers} gates), "
                             f"partitions={t['partitions']}, reference built for the host CPU ({t['build']})",
                   "seconds": secs[0]}
            if grad_line is not None:
                grad_line["cpu_reference"] = time_reference_gradient(wl, cores)
            if not args.no_sub_results:
                for sub in sub_results:
                    st = time_reference(WL.BY_NAME[sub["workload"]](), 3, 1, cores)
                    sub["cpu_baseline"] = {"value": _updates(WL.BY_NAME[sub["workload"]]()) * 3 / sum(st["seconds"]),
                                           "unit": "updates/s", "cores": cores, "kind": "reference",
                                           "build": st["build"], "partitions": st["partitions"],
                                           "sample": "3 full propagates"}
        else:
            cpu = {"value": None, "unit": "updates/s", "cores": 0, "kind": "reference",
                   "sample": "oracle/_ref/libmpref.so not built"}

    line = {"metric": "term-gate updates/s", "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded circuit)",
            "config": config, "term_gate_updates_per_step": updates, "final_terms": int(stats.n[-1] + stats.appended[-1]),
            "expectation": ev_dev, "expectation_e2e": ev2,
            "e2e": {"value": e2e, "unit": "updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8,
                    "ms_per_step": e2e_total / args.steps},
            "gpu_launches": launches, "graph_replays": graph_replays, "roofline": roofline, "cpu_baseline": cpu,
            "clocks": clk.summary(), "gradient": grad_line, "sub_results": sub_results}
    print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.destroy_process_group()


def measure_compact(wl, steps: int, warmup: int, device: int, flush) -> dict:
    """Device rate of one resident circuit (store reset untimed, L2 flushed, CUDA events on the engine's
    stream) and its end-to-end rate through the C ABI from host buffers, as for the main workload."""
    import torch

    from monoprop_b200 import _native

    dev = torch.device("cuda", device)
    gw, ang = wl.gen_words(), wl.angles()
    eng = _native.engine_for(wl, device=device)
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)
    circ = eng.upload(gw, ang)
    ms = []
    for i in range(warmup + steps):
        eng.reset()
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.propagate_circuit(circ)
        b.record(stream)
        b.synchronize()
        if i >= warmup:
            ms.append(a.elapsed_time(b))
    updates = eng.gate_stats().term_gate_updates
    ev = eng.expectation()
    circ.close()
    eng.close()
    e2e_ms = []
    for i in range(warmup + steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2 = _native.engine_for(wl, device=device)
        e2.propagate(gw, ang)
        e2.expectation()
        e2.close()
        if i >= warmup:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
    keys, coefs, _ = wl.encoded_observable()
    return {"workload": wl.name, "config": f"{wl.num_modes} modes, {wl.n_layers} gates, {wl.basis}, cutoff {wl.cutoff}, "
                                          f"lower_atol {wl.lower_atol}",
            "metric": "term-gate updates/s", "value": updates * len(ms) / (sum(ms) * 1e-3), "unit": "updates/s",
            "ms_per_step": sum(ms) / len(ms), "steps": len(ms), "expectation": ev,
            "e2e": {"value": updates * len(e2e_ms) / (sum(e2e_ms) * 1e-3), "unit": "updates/s",
                    "ms_per_step": sum(e2e_ms) / len(e2e_ms),
                    "h2d_bytes_per_step": int(gw.nbytes + ang.nbytes + keys.nbytes + coefs.nbytes),
                    "d2h_bytes_per_step": 8}}


def batch_bench(args) -> None:
    """The batched workload: independent 5x10 kicked-Ising instances (50 qubits) of depth U{4..24},
    angles U[0, 0.3 pi), one Z_i observable each (i from the seed), Pauli weight <= 8, lower_atol 1e-5;
    <O> and the full gradient of every instance in one engine call, with the autotuned knobs against
    the defaults. Gradient checkpoints every 4 circuit layers (540 gates)."""
    import torch

    from monoprop_b200 import workloads as WL
    from monoprop_b200.batch import Autotuner, BatchConfig, run_batch, shard_instances

    rank, world, local, dist = _dist()
    torch.cuda.set_device(local)
    if dist is not None:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    full = WL.batch_ising50(args.batch_instances)
    # instances are independent: rank r takes its deepest-first round-robin share (no data-path collective)
    batch = [full[i] for i in shard_instances(full, rank, world)]
    seg = 4 * 135
    run_batch(batch[-4:], BatchConfig(), gradient=True, segment_gates=seg, device=local)  # warm-up
    tuner = Autotuner(cache_path=os.path.join(tempfile.gettempdir(), f"mpx_autotune_{os.getpid()}.json"))
    t0 = time.perf_counter()
    best, entry = tuner.tune(batch, gradient=True, segment_gates=seg, device=local, use_cache=False)
    tune_s = time.perf_counter() - t0
    tuned, default = [], []
    for _ in range(max(1, args.steps)):
        tuned.append(run_batch(batch, best, gradient=True, segment_gates=seg, device=local))
        default.append(run_batch(batch, BatchConfig(), gradient=True, segment_gates=seg, device=local))
    fwd = run_batch(batch, best, gradient=False, device=local)
    dev = torch.device("cuda", local)
    t_tuned = max_over_ranks(min(r.seconds for r in tuned), dist, dev)
    t_default = max_over_ranks(min(r.seconds for r in default), dist, dev)
    t_fwd = max_over_ranks(fwd.seconds, dist, dev)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    n = len(full)
    batch = full
    depths = [wl.n_layers // 135 for wl in batch]
    line = {"metric": "<O>+full-gradient/s", "value": n / t_tuned, "unit": "gradients/s", "n_gpus": world,
            "steps": len(tuned), "warmup": 1, "ms_per_step": 1e3 * t_tuned, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded circuits)",
            "config": {"workload": f"batch of {n} 5x10 kicked-Ising instances, depth {min(depths)}..{max(depths)}, "
                                   "Pauli weight <= 8, lower_atol 1e-5, gradient checkpoints every 540 gates",
                       "parallelism": f"instances split over {world} GPU(s), no collective on the data path",
                       "angles": int(sum(wl.n_layers for wl in batch)),
                       "final_terms_max": int(max(int(x) for x in tuned[0].final_terms))},
            "autotuned": {**best.as_dict(), "seconds": t_tuned, "tuning_seconds": tune_s,
                          "candidates": entry["table"], "validation": entry.get("validation"),
                          "validation_sample": entry.get("validation_sample")},
            "default": {**BatchConfig().as_dict(), "seconds": t_default},
            "forward_only": {"value": n / t_fwd, "unit": "expectations/s", "seconds": t_fwd},
            "e2e": {"value": n / t_tuned, "unit": "gradients/s",
                    "h2d_bytes_per_step": int(sum(wl.gen_words().nbytes + wl.angles().nbytes for wl in batch)),
                    "d2h_bytes_per_step": int(sum(8 * (wl.n_layers + 1) for wl in batch))}}
    print(json.dumps(line), flush=True)


def batch_reference(args) -> None:
    """The reference engine on a bounded, depth-stratified sample of the batch (forward propagate of each
    sampled instance on all host threads); the rate is instances per second."""
    import oracle

    from monoprop_b200 import workloads as WL

    rank, world, _, _ = _dist()
    if rank != 0:
        return
    full = WL.batch_ising50(args.batch_instances)
    order = sorted(range(len(full)), key=lambda i: full[i].n_layers)
    sample = [full[i] for i in order[:: max(1, len(order) // 4)][:4]]
    cores = args.cpu_partitions or _cpu_threads()
    secs = [time_reference(wl, 1, 0, cores)["seconds"][0] for wl in sample]
    v = len(sample) / sum(secs)
    line = {"metric": "<O>/s (forward)", "value": v, "unit": "expectations/s", "n_gpus": args.gpus, "steps": 1,
            "warmup": 0, "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded circuits)",
            "config": {"workload": f"batch of {len(full)} 5x10 kicked-Ising instances (depth-stratified sample of "
                                   f"{len(sample)}: depths {[wl.n_layers // 135 for wl in sample]})"},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "expectations/s", "cores": cores, "kind": "reference",
                             "sample": f"{len(sample)} instances, one forward propagate each"},
            "e2e": {"value": v, "unit": "expectations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_case(n_terms: int, n_gates: int) -> None:
    """A large store built in one upload (few launches before the profiled ones), then a few gates."""
    from monoprop_b200 import _native
    from monoprop_b200 import workloads as WL

    wl = WL.ising100()
    rng = np.random.default_rng(5)
    tier, W = 128, 4
    keys = np.zeros((n_terms, W), dtype=np.uint64)
    qubits = rng.integers(0, 100, size=(n_terms, 10))
    kinds = rng.integers(1, 4, size=(n_terms, 10))  # 1: X (slot 2q), 2: Y (2q+1), 3: Z (both)
    for j in range(10):
        for slot_off, sel in ((0, kinds[:, j] != 2), (1, kinds[:, j] != 1)):
            bit = (2 * tier - 1) - (2 * qubits[:, j] + slot_off)
            word, pos = bit // 64, (bit % 64).astype(np.uint64)
            for w in range(W):
                m = sel & (word == w)
                keys[m, w] |= np.uint64(1) << pos[m]
    keys = np.unique(keys, axis=0)
    coefs = rng.uniform(-1e-2, 1e-2, size=keys.shape[0])
    eng = _native.Engine(basis="pauli", cutoff_type="support", cutoff=wl.cutoff, num_modes=100, keys=keys,
                         coefs=coefs, core=0.0, state_mask=wl.state_mask(), lower_atol=wl.lower_atol)
    eng.propagate(wl.gen_words()[-n_gates:], wl.angles()[-n_gates:])
    st = eng.gate_stats()
    print(json.dumps({"kernel_case_terms": int(keys.shape[0]), "n_g": st.n.tolist(), "a_g": st.anti.tolist(),
                      "e_g": st.emitted.tolist(), "m_g": st.appended.tolist()}), flush=True)
    eng.close()


def regime_case(n_terms: int, n_gates: int) -> None:
    """The 100-qubit benchmark circuit in its own regime: propagated (gates last to first) until the store
    holds about ``n_terms`` terms, then ``n_gates`` more gates inside the NVTX range ``mpx_profile`` (what a
    kernel profiler selects)."""
    import torch

    from monoprop_b200 import _native
    from monoprop_b200 import workloads as WL

    wl = WL.ising100()
    gw, ang = wl.gen_words(), wl.angles()
    L = wl.n_layers
    eng = _native.engine_for(wl)
    eng.propagate(gw, ang)
    n = eng.gate_stats().n
    eng.close()
    _native.load().mpx_trim_device_memory(0)  # hand the full-size store back before the profiled case
    steps = int(np.searchsorted(n, n_terms))  # applied steps before the profiled gates
    steps = min(steps, L - n_gates)
    eng = _native.engine_for(wl)
    eng.propagate(gw[L - steps:], ang[L - steps:])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("mpx_profile")
    eng.propagate(gw[L - steps - n_gates:L - steps], ang[L - steps - n_gates:L - steps])
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    st = eng.gate_stats()
    print(json.dumps({"regime_case_steps_before": steps, "n_g": st.n.tolist(), "a_g": st.anti.tolist(),
                      "e_g": st.emitted.tolist(), "m_g": st.appended.tolist()}), flush=True)
    eng.close()


def profile_kernels() -> None:
    """Small cases for the kernels the benchmark step does not profile: the shared-memory path (the
    20-qubit line circuit), the expectation reduction, the column and table builds (the 100-qubit circuit's
    first 1200 gates, with a reset), and the frozen replay and adjoint kernels (its gradient with
    checkpoints every 280 gates), each inside an NVTX range named after the work."""
    import torch

    from monoprop_b200 import _native
    from monoprop_b200 import workloads as WL

    nvtx = torch.cuda.nvtx
    wl = WL.line20()
    eng = _native.engine_for(wl)
    torch.cuda.synchronize()
    nvtx.range_push("small_path")
    eng.propagate(wl.gen_words(), wl.angles())
    torch.cuda.synchronize()
    nvtx.range_pop()
    eng.close()
    wl = WL.ising100()
    L = 1200
    gw, ang = wl.gen_words()[:L], wl.angles()[:L]
    eng = _native.engine_for(wl)
    circ = eng.upload(gw, ang)
    eng.propagate_circuit(circ)
    torch.cuda.synchronize()
    nvtx.range_push("expectation")
    eng.expectation()
    torch.cuda.synchronize()
    nvtx.range_pop()
    nvtx.range_push("reset_build")
    eng.reset()
    torch.cuda.synchronize()
    nvtx.range_pop()
    ev = eng.adjoint_forward(circ, 280)
    torch.cuda.synchronize()
    nvtx.range_push("adjoint_backward")
    g = eng.adjoint_backward(circ)
    torch.cuda.synchronize()
    nvtx.range_pop()
    eng.graph_build(circ)
    torch.cuda.synchronize()
    nvtx.range_push("frozen_replay")
    eng.graph_expectation(circ)
    torch.cuda.synchronize()
    nvtx.range_pop()
    print(json.dumps({"profile_kernels": "ok", "terms": eng.size(), "expectation": ev,
                      "grad_abs_max": float(np.max(np.abs(g)))}), flush=True)
    circ.close()
    eng.close()


def _updates(wl) -> int:
    """sum_g n_g of ``wl`` (the oracle's count, equal to the engine's per-gate counters)."""
    from monoprop_b200.workloads import TERM_GATE_UPDATES

    return TERM_GATE_UPDATES[wl.name]


if __name__ == "__main__":
    main()
