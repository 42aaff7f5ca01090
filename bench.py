#!/usr/bin/env python3
"""Benchmark: query Mbp/s of the seed-and-extend search on the medium workload.

Workload (seeded synthetic data with the shapes of the reference's medium
configuration): a 100 Mbp target in 200 contigs (log-normal lengths, median
300 kbp, 10 % of bases in 500 repeat families at 85-99 % identity, 0.1 % N
runs) and 1,000,000 reads of 150 bp (2 % substitutions, 0.5 % indels, half
reverse strand, 5 % random decoys), reference default settings (l 15,
stride 5, repeat 20, width 100, gap 8, global, cut-off 10, tRAM/qRAM 64,
tVRAM 64, qVRAM 2 MBase).  One step = the whole job: index every target window
of both target RAM loads, map all five query RAM loads, and return the hits
in the reference's output order.

  value  -- inputs already in HBM (device tensors), CUDA events around K steps
  e2e    -- the same job through the C ABI from pinned host buffers, host-to-
            device copies and the result download inside the timed region

--impl reference times the reference's own CPU implementation (its sources
built for the host CPU, oracle/_ref/clast_ref) on this box's cores.

Multi-GPU (torchrun): each rank maps its own 1M reads (seed + rank) against a
replicated target index; no data-path collective (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from clast_b200 import api, synth  # noqa: E402

METRIC = "query Mbp/s (bit-exact hits)"
# DRAM bytes (read + write) per looked-up l-mer of k_seed_fused, from an ncu
# capture on the half-size medium workload (profiles/k_seed_fused_medium_half.md)
SEED_DRAM_BYTES_PER_KMER = 12.2
T_RAM, Q_RAM, T_VRAM, Q_VRAM = 64e6, 64e6, 64e6, 2e6  # common.hpp:12-15, x 1e6 (CHostSetting.cu:133-136)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="medium")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=0xC1A57)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-sample-reads", type=int, default=40000)
    return ap.parse_args()


def workload_config(args, t, q):
    return {
        "workload": "%s: %d bp target in %d contigs, %d reads of %s bp" % (
            args.workload, int(t.offsets[-1]), len(t), len(q),
            "150" if args.workload != "uneven" else "50-10000"),
        "target_bp": int(t.offsets[-1]), "contigs": len(t), "reads": len(q),
        "query_bp": int(q.offsets[-1]),
        "settings": "reference defaults: lMer 15, stride 5, repeat 20, width 100, gap 8, global, cutOff 10, "
                    "tRAM/qRAM/tVRAM 64, qVRAM 2 MBase",
        "l2": "inputs larger than L2 (target + reads + indexes >> 126 MB); no flush",
        "seed": args.seed,
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baselines (the reference built for the CPU, else the oracle port)
# ---------------------------------------------------------------------------
def cpu_reference_rate(t, q, n_sample, threads=None):
    """Reference CPU throughput on this host, extrapolated to the full job.

    Two runs on the full target: with 1 read (the fixed cost: FASTA parsing and
    the index builds of both target RAM loads) and with the first n_sample
    reads.  The full job needs one pair of index builds per query RAM load, so
    T_full = loads_full * T_fixed + (reads_full / n_sample) * (T_sample - T_fixed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kind = "reference" if O.ref_available() else "port"
    exe = O.REF if kind == "reference" else O.CLI
    if kind == "port" and not os.path.exists(exe):
        O.build()
    threads = threads or os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    with tempfile.TemporaryDirectory() as d:
        tp = os.path.join(d, "t.fa")
        t.to_fasta(tp)
        times = {}
        for n in (1, n_sample):
            qs = synth.SeqSet(q.labels[:n], q.bases[:q.offsets[n]], q.offsets[:n + 1])
            qp = os.path.join(d, "q%d.fa" % n)
            qs.to_fasta(qp)
            t0 = time.perf_counter()
            r = subprocess.run([exe, "-t", tp, "-q", qp, "-o", os.path.join(d, "o.tsv")], env=env,
                               capture_output=True, text=True)
            times[n] = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError("CPU baseline failed: %s" % (r.stdout + r.stderr)[-500:])
    q_loads = len(api.ram_loads(np.diff(q.offsets), int(Q_RAM / 2))[1])
    per_read = max(times[n_sample] - times[1], 1e-9) / n_sample
    t_full = q_loads * times[1] + len(q) * per_read
    mbp = q.offsets[-1] / 1e6
    return {
        "value": mbp / t_full, "unit": "Mbp/s", "cores": threads, "kind": kind,
        "sample": "full target; a 1-read run (%.1f s: FASTA + index builds) and a %d-read run (%.1f s), "
                  "extrapolated to %d query RAM loads and %d reads (%.0f s)" % (
                      times[1], n_sample, times[n_sample], q_loads, len(q), t_full),
    }


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    # data: same target on every rank, reads seeded by rank
    t, q0 = synth.workload(args.workload, seed=args.seed, scale=args.scale)
    q = q0 if rank == 0 else synth.workload(args.workload, seed=args.seed + 1000 * rank, scale=args.scale)[1]
    s = api.Setting(total_db=float(t.offsets[-1]))  # synthetic FASTA: every non-'>' line is bases
    t_keep, t_loads = api.ram_loads(np.diff(t.offsets), int(T_RAM))
    q_keep, q_loads = api.ram_loads(np.diff(q.offsets), int(Q_RAM / 2))
    assert t_keep.all() and q_keep.all()
    eng = api.Engine(local)
    int32_peak = eng.int32_peak()  # tera-ops/s, measured on this GPU
    # pinned host buffers (e2e) and device-resident copies (value)
    t_pin = torch.from_numpy(t.bases).pin_memory()
    q_pin = torch.from_numpy(q.bases).pin_memory()
    t_dev = t_pin.to("cuda", non_blocking=False)
    q_dev = q_pin.to("cuda", non_blocking=False)
    torch.cuda.synchronize()

    host = {"targets": [], "map": [], "close": [], "ctypes": [], "inside": [], "map_device": []}

    def step(tb, qb):
        c0 = time.perf_counter()
        T = eng.targets(s, tb, t.offsets, t_loads, int(T_VRAM))
        c1 = time.perf_counter()
        res = eng.map(s, T, qb, q.offsets, q_loads, int(Q_VRAM))
        c2 = time.perf_counter()
        T.close()
        c3 = time.perf_counter()
        host["targets"].append((c1 - c0) * 1e3)
        host["map"].append((c2 - c1) * 1e3)
        host["close"].append((c3 - c2) * 1e3)
        host["ctypes"].append(eng.last_map_py_ms[1])
        sm = eng.stats()
        host["inside"].append(sm["map_call_ms"])
        host["map_device"].append(sm["map_ms"] + sm["map_upload_ms"])
        return res

    def timed(tb, qb, sampler=None):
        # warm-up in the timed loop's own pattern: the previous step's result is
        # still held while the next one is mapped (two result buffers in use)
        res = None
        for _ in range(args.warmup):
            res = step(tb, qb)
        del res
        for v in host.values():
            v.clear()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        e0.record()
        for _ in range(args.steps):
            res = step(tb, qb)
            st = eng.stats()
            launches += st["index_launches"] + st["map_launches"]
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            x = torch.tensor([ms], device="cuda")
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            ms = float(x.item())
        # host wall time of the API calls per step: median and max over the timed steps
        hw = {k: [round(statistics.median(v), 3), round(max(v), 3)] for k, v in host.items() if v}
        hw["fields"] = ("[median, max] ms per step; ctypes = the clast_map call, inside = measured in clast_map, "
                        "map_device = CUDA-event time of the map's uploads and stages")
        hw["map_per_step"] = [round(x, 1) for x in host["map"]]
        return ms, launches, res, st, hw

    with ClockSampler(local) as clk:
        ms_dev, launches, res, st, hw_dev = timed(t_dev, q_dev)
    scores = res["score"].copy()
    del res
    ms_e2e, _, res2, st2, hw_e2e = timed(t_pin, q_pin)
    assert np.array_equal(scores, res2["score"])
    mbp_rank = q.offsets[-1] / 1e6
    value = mbp_rank * world * args.steps / (ms_dev / 1e3)
    e2e = mbp_rank * world * args.steps / (ms_e2e / 1e3)
    # roofline of the dominant device stage of one step
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    n_tw = max(1, st["seed_launches"] // 2)
    # algorithmic bytes of k_seed_fused per target window: 3/8 B per query base
    # (2-bit code + N mask), one 8 B filter word per valid l-mer, 12 B written
    # + 8 B of entry read per seed
    seed_bytes = n_tw * st["query_bases"] * 3 / 8 + 8 * st["query_kmers"] + 20 * st["seeds"]
    stages = {"seeding": st["seed_ms"], "banded_dp": st["dp_ms"], "seed_sort_filter": st["sort_ms"],
              "result_order": st["final_ms"]}
    seed_gbs = seed_bytes / (st["seed_ms"] / 1e3) / 1e9 if st["seed_ms"] > 0 else 0.0
    roofline = {
        "kernel": "seeding (k_seed_fused: l-mer keys, filter + table lookups, seed writes)",
        "bound": "hbm", "achieved": round(seed_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
        "frac": round(seed_gbs / hbm_peak, 4),
        "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
        "bytes_per_launch": int(seed_bytes / max(1, st["seed_launches"])),
        "ms_per_launch": round(st["seed_ms"] / max(1, st["seed_launches"]), 3),
        "launches_per_step": st["seed_launches"],
        "traffic": int(SEED_DRAM_BYTES_PER_KMER * st["query_kmers"] / max(1, st["seed_launches"])),
        "traffic_source": "ncu DRAM bytes per l-mer on the half-size workload x l-mers per launch",
        "stage_ms_per_step": {k: round(v, 3) for k, v in stages.items()},
        "step_device_ms": round(st["index_ms"] + st["map_ms"], 3),
        "index_ms": round(st["index_ms"], 3), "map_ms": round(st["map_ms"], 3),
        "dp": {"cells": st["dp_cells"], "ms": round(st["dp_ms"], 3), "launches": st["dp_launches"],
               "gcups": round(st["dp_cells"] / (st["dp_ms"] / 1e3) / 1e9, 1) if st["dp_ms"] > 0 else None,
               "int32_ops_per_cell": 13,
               "int32_tops": round(13 * st["dp_cells"] / (st["dp_ms"] / 1e3) / 1e12, 2) if st["dp_ms"] > 0 else None,
               "int32_peak_tops": round(int32_peak, 2),
               "frac": round(13 * st["dp_cells"] / (st["dp_ms"] / 1e3) / 1e12 / int32_peak, 4)
               if st["dp_ms"] > 0 else None,
               "peak_source": "measured (clast_int32_peak: add/max/logic chains)"},
    }
    out = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mbp/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_dev / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator clast_b200/synth.py; no public dataset)",
        "config": dict(workload_config(args, t, q), parallelism="replicated index, reads sharded" if world > 1
                       else "single GPU"),
        "e2e": {"value": round(e2e, 2), "unit": "Mbp/s", "ms_per_step": round(ms_e2e / args.steps, 3),
                "h2d_bytes_per_step": int(t.offsets[-1] + q.offsets[-1]),
                "d2h_bytes_per_step": int(st2["results"] * 36)},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "counts_per_step": {k: st[k] for k in ("query_bases", "query_kmers", "seeds", "hits", "results",
                                               "dp_cells", "index_launches", "map_launches")},
        "clocks": clk.summary(),
        "host_wall_ms_per_step": {"value_loop": hw_dev, "e2e_loop": hw_e2e},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_reference_rate(t, q, min(args.ref_sample_reads, len(q)))
        except Exception as e:  # reported, never fatal
            out["cpu_baseline"] = {"error": str(e)[:300]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t, q = synth.workload(args.workload, seed=args.seed, scale=args.scale)
    vals = []
    for _ in range(max(1, args.steps)):
        vals.append(cpu_reference_rate(t, q, min(args.ref_sample_reads, len(q))))
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[0], value=v)
    out = {
        "metric": METRIC, "value": round(v, 4), "unit": "Mbp/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator clast_b200/synth.py; no public dataset)",
        "config": workload_config(args, t, q), "impl": "reference", "cpu_baseline": cb,
        "e2e": {"value": round(v, 4), "unit": "Mbp/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
