#!/usr/bin/env python
"""Benchmark of the B200 Datalog fixpoint engine.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sg_rmat_s14|tc_grid_64|cspa_v300]

Default workload: same generation on an R-MAT graph of scale 14 (16,384
nodes), 40,000 directed edges, a,b,c,d = .57,.19,.19,.05, seed 14, self loops
and duplicates removed; the reference's SG program (test/sg.cu:93-191: an
init LIE, then the recursive LIE with a tmp relation).  One step = both
fixpoints of that program over one synthetic input.

Metric: derived tuples per second = |sg| / fixpoint seconds.
  value  device time of the fixpoint loops (CUDA events on the engine's
         stream) with the input relations already loaded in HBM;
  e2e    the same metric through the public API from host buffers:
         host->device copy and load of the edges, both fixpoints, and the
         device->host read of the result's size and digest, every step.
The roofline object is the dominant kernel family of one extra profiled
step (an event pair around every launch) against the measured HBM copy
bandwidth.  cpu_baseline times the CPU oracle (a C++/OpenMP restatement of
the reference's semi-naive loop) on all host cores.

--impl reference runs that same CPU implementation as the reference arm
(the reference's own CPU path, its Souffle programs, cannot be built
offline); on a GPU machine that line also carries `reference_gpu`: the
reference's CUDA engine, built unmodified from its sources, timed live on
the same input.  `e2e_phases_ms` splits one extra end-to-end step by
public-API call.
Under torchrun every rank runs one replica of the workload (the single
fixpoint does not shard); value sums the ranks' tuples over the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "gdlog-multinode_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

import programs as P  # noqa: E402
import workloads as W  # noqa: E402

WORKLOADS = {
    "sg_rmat_s14": dict(
        prog=P.sg, make=lambda: (W.rmat_edges(14, 40000, seed=14),),
        desc="same generation, R-MAT scale 14 (16,384 nodes), 40,000 edges, "
             "a,b,c,d=.57,.19,.19,.05, seed 14"),
    # the same program and input on the sorted-list path (radix sort +
    # merge-path dedup of every candidate), so the sort kernels dominate
    "sg_rmat_s14_sort": dict(
        prog=P.sg, make=lambda: (W.rmat_edges(14, 40000, seed=14),), tuning={"dedup": "sort"},
        desc="same generation, R-MAT scale 14 (16,384 nodes), 40,000 edges, "
             "a,b,c,d=.57,.19,.19,.05, seed 14; sorted-list path (dedup=sort)"),
    # the sorted-list path on a small case (profiling the sort kernels)
    "sg_rmat_s12_sort": dict(
        prog=P.sg, make=lambda: (W.rmat_edges(12, 8000, seed=12),), tuning={"dedup": "sort"},
        desc="same generation, R-MAT scale 12 (4,096 nodes), 8,000 edges, seed 12; "
             "sorted-list path (dedup=sort)"),
    "tc_grid_64": dict(
        prog=P.tc, make=lambda: (W.grid_edges(64, 64),),
        desc="transitive closure, 64x64 directed grid, 8,064 edges"),
    "sg_rmat_s13": dict(
        prog=P.sg, make=lambda: (W.rmat_edges(13, 20000, seed=14),),
        desc="same generation, R-MAT scale 13 (8,192 nodes), 20,000 edges, "
             "a,b,c,d=.57,.19,.19,.05, seed 14 (profiling case)"),
    "cspa_v300": dict(
        prog=P.cspa, make=lambda: W.cspa_facts(300, 600, 225, seed=3),
        desc="CSPA, 300 variables, 600 assign, 225 dereference, Zipf(1.1) sources, seed 3"),
    # ids above 2^15: bitmaps over a 2^32-bit domain (the sorted-list path
    # cannot hold this program's candidates); no CPU baseline (the oracle
    # would take many minutes)
    "sg_rmat_s16": dict(
        prog=P.sg, make=lambda: (W.rmat_edges(16, 120000, seed=16),), no_cpu=True,
        desc="same generation, R-MAT scale 16 (65,536 nodes), 120,000 edges, seed 16"),
    # C3: the full CSPA configuration, about a minute per step on one B200
    "cspa_c3": dict(
        prog=P.cspa, make=lambda: W.cspa_facts(), no_cpu=True,
        desc="CSPA, 20,000 variables, 40,000 assign, 15,000 dereference, Zipf(1.1), seed 3"),
    # arity 3 rows load from the host (the fixpoint's device time excludes loads)
    "plen_grid_64": dict(
        prog=P.path_length, make=lambda: (W.grid_edges(64, 64),), host_inputs=True, max_arity=3,
        desc="path_length (arity 3, dependent length column), 64x64 directed grid, 8,064 edges"),
}


def derived(result) -> int:
    return sum(r.size() for r in result.relations.values())


def measured_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi's start-up (NVML initialisation) takes the driver for
            # a while; let it finish before the timed region opens, so that
            # only the periodic queries overlap the measured steps
            t_end = time.time() + 5.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def oracle_run(wl: dict, inputs, threads: int = 0):
    """One run of the workload on the CPU oracle: (fixpoint seconds, tuples)."""
    from gdlog_b200 import Engine
    with Engine("oracle", threads=threads, max_arity=wl.get("max_arity", 2)) as eng:
        r = wl["prog"](eng, *inputs)
        secs = sum(lie.stats()["ms"] for lie in r.lies.values()) / 1e3
        return secs, derived(r), eng.threads


def roofline_of(prof: dict, workload: str, peaks: dict) -> dict:
    """Roofline object of the dominant kernel family (most device time) of
    one profiled step: its algorithmic bytes per launch over its mean
    launch time (CUDA events on the engine stream), against the measured
    HBM copy bandwidth."""
    kind, rec = max(prof.items(), key=lambda kv: kv[1]["ms"])
    per_launch_ms = rec["ms"] / max(rec["launches"], 1)
    per_launch_bytes = rec["bytes"] / max(rec["launches"], 1)
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9 if per_launch_ms else 0.0
    traffic = traffic_for(workload, kind, per_launch_bytes)
    dram_gbs = traffic / (per_launch_ms / 1e3) / 1e9 if (traffic and per_launch_ms) else None
    return {"bound": "hbm", "kernel": kind, "achieved": achieved,
            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
            "traffic": traffic,
            "dram_gbs": dram_gbs,
            "frac_dram": dram_gbs / peaks["hbm_gbs"] if dram_gbs else None,
            "alg_bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
            "launches": rec["launches"],
            "peak_source": peaks["source"] + " (MEASURED_PEAKS.json hbm_gbs)"}


def single_families(prof):
    return {kd: {"launches": v["launches"], "alg_bytes": v["bytes"]}
            for kd, v in prof.items() if v["launches"]}


def traffic_for(workload: str, kind: str, alg_bytes_per_launch: float):
    """DRAM bytes per launch of a kernel family: the family's DRAM bytes
    (dram__bytes_read.sum + dram__bytes_write.sum over all its launches in
    one ncu capture of `bench.py --single --workload <workload>`, committed
    in profiles/traffic.json) per algorithmic byte of that same step, times
    this launch's algorithmic bytes."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    rec = json.load(open(p)).get(workload, {}).get(kind)
    if not rec or not rec.get("alg_bytes"):
        return None
    return rec["dram_bytes"] / rec["alg_bytes"] * alg_bytes_per_launch


# Workloads on which the reference CUDA build runs (oracle/_ref/ref_runner):
# program and input files.  It is not run on the larger points-to inputs,
# where it made an illegal memory access (2,000 variables) or ran out of
# device memory (6,000 variables).
REF_GPU_RUNS = {"sg_rmat_s14": "sg", "sg_rmat_s14_sort": "sg", "sg_rmat_s13": "sg",
                "tc_grid_64": "tc", "cspa_v300": "cspa", "plen_grid_64": "plen"}


def reference_gpu_live(workload: str, inputs, runs: int = 3):
    """The reference CUDA engine (built unmodified from its sources into
    oracle/_ref/ref_runner) on the same input, timed as its drivers time
    fixpoint_loop (test/tc.cu:120-140): median fixpoint seconds of `runs`
    runs, with the clocks sampled meanwhile.  None when the runner is not
    built or the workload is not one it runs on."""
    import tempfile
    exe = os.path.join(REPO, "oracle", "_ref", "ref_runner")
    prog = REF_GPU_RUNS.get(workload)
    if not prog or not os.path.exists(exe):
        return None
    secs, rec = [], None
    with tempfile.TemporaryDirectory() as d, ClockSampler(0) as clocks:
        files = []
        for i, rows in enumerate(inputs):
            f = os.path.join(d, f"in{i}.tsv")
            W.write_tsv(f, rows)
            files.append(f)
        for _ in range(runs):
            r = subprocess.run([exe, prog, *files], stdout=subprocess.DEVNULL,
                               stderr=subprocess.PIPE, text=True, timeout=600)
            line = [ln for ln in r.stderr.splitlines() if ln.startswith("REF ")]
            if r.returncode != 0 or not line:
                return {"unavailable": f"ref_runner exit {r.returncode}"}
            rec = json.loads(line[-1][4:])
            secs.append(rec["seconds"])
    t = sum(rec["sizes"].values())
    sec = statistics.median(secs)
    return {"value": t / sec, "unit": "tuples/s", "seconds": sec, "runs": runs,
            "tuples": t, "iterations": rec["iterations"], "clocks": clocks.summary(),
            "source": "reference CUDA engine built unmodified from its sources "
                      "(oracle/_ref/ref_runner), same input, this GPU, timed like its drivers"}


def e2e_phases(eng, wl: dict, pinned) -> dict:
    """One more end-to-end step (untimed by the line's e2e number) with every
    public-API call timed on the host and the engine stream synchronised
    after each call, so the phases add up to where an e2e step's time goes:
    engine clear, relation creation, loads (host->device copy, pack, sort,
    deduplicate, index), LIE creation, the fixpoints (with their host setup,
    graph capture and device time from gdl_lie_stats), size and digest."""
    import gdlog_b200 as G
    acc: dict = {}
    patched = []

    def wrap(obj, name, label):
        fn = getattr(obj, name)
        patched.append((obj, name, obj.__dict__.get(name)))

        def timed(*args, **kw):
            t0 = time.perf_counter()
            out = fn(*args, **kw)
            eng.sync()
            acc[label] = acc.get(label, 0.0) + (time.perf_counter() - t0) * 1e3
            return out
        setattr(obj, name, timed)

    wrap(eng, "relation", "create_relations")
    wrap(eng, "load", "loads")
    wrap(eng, "lie", "create_lies")
    wrap(G.Lie, "fixpoint", "fixpoints")
    wrap(G.Relation, "size", "size")
    wrap(G.Relation, "digest", "digest")
    try:
        t_all = time.perf_counter()
        t0 = time.perf_counter()
        eng.clear()
        eng.sync()
        acc["clear"] = (time.perf_counter() - t0) * 1e3
        r = wl["prog"](eng, *pinned)
        for rel in r.relations.values():
            rel.size()
            rel.digest()
        total = (time.perf_counter() - t_all) * 1e3
    finally:
        for obj, name, orig in reversed(patched):
            if orig is None:
                delattr(obj, name)
            else:
                setattr(obj, name, orig)
    st = [lie.stats() for lie in r.lies.values()]
    out = {k: round(v, 4) for k, v in acc.items()}
    out["fixpoint_device_ms"] = round(sum(x["ms"] for x in st), 4)
    out["fixpoint_host_setup_ms"] = round(sum(x["setup_ms"] for x in st), 4)
    out["fixpoint_graph_ms"] = round(sum(x["graph_ms"] for x in st), 4)
    out["other_host_ms"] = round(total - sum(acc.values()), 4)
    out["total_ms"] = round(total, 4)
    return out


def run_ours(a) -> None:
    import torch
    from gdlog_b200 import DeviceRows, Engine

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    wl = WORKLOADS[a.workload]
    inputs = wl["make"]()
    stream = torch.cuda.Stream(device=dev)
    eng = Engine("gpu", device=local, stream=stream.cuda_stream)
    from autotune import Tuner
    tuner = Tuner()
    if a.tune:
        # time every candidate configuration on this workload and cache the best
        rec = tuner.tune(eng, wl["prog"], inputs)
        print(json.dumps({"tuned": a.workload, "bucket": tuner.key(wl["prog"].__name__, inputs),
                          **rec}), flush=True)
        eng.close()
        return
    rec = tuner.apply(eng, wl["prog"], inputs)
    tuning = rec["config"] if rec else "engine defaults (no cached tuning for this size bucket)"
    if wl.get("tuning"):
        eng.set_tuning(**wl["tuning"])
        tuning = {"workload_setting": wl["tuning"], "cached": tuning}
    dev_inputs = inputs if wl.get("host_inputs") else \
        [DeviceRows(torch.from_numpy(x.astype(np.int64)).to(dev)) for x in inputs]
    pinned = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() for x in inputs]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    host = {"setup_ms": 0.0, "grow_ms": 0.0, "graph_ms": 0.0, "retries": 0}

    def device_step():
        eng.clear()
        with torch.cuda.stream(stream):
            flush.fill_(1)  # L2 flush between steps (256 MB > 126 MB L2)
        r = wl["prog"](eng, *dev_inputs)
        st = [lie.stats() for lie in r.lies.values()]
        for key in host:
            host[key] += sum(s[key] for s in st)
        return sum(s["ms"] for s in st), derived(r), sum(s["kernels"] for s in st)

    n_out = [0]

    def e2e_step():
        eng.clear()
        r = wl["prog"](eng, *pinned)
        out = [(rel.size(), rel.digest()) for rel in r.relations.values()]
        n_out[0] = len(out)
        return sum(n for n, _ in out)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()

    if a.single:
        # one step with an event pair around every launch; the algorithmic
        # bytes per kernel family are what an ncu capture of this same
        # command is compared against
        eng.profile_reset()
        eng.set_profile(True)
        ms, t, k = device_step()
        eng.set_profile(False)
        print(json.dumps({"single_step_ms": ms, "tuples": t, "launches": k,
                          "families": single_families(eng.profile())}), flush=True)
        eng.close()
        return
    for _ in range(a.warmup):
        device_step()
    e2e_step()
    barrier()
    ms_total, tuples, kernels = 0.0, 0, 0
    for key in host:
        host[key] = 0
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            ms, t, k = device_step()
            ms_total += ms
            tuples += t
            kernels += k
        barrier()
        # e2e: public API from pinned host buffers, events on the engine stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_tuples = 0
        e0.record(stream)
        for _ in range(a.steps):
            e2e_tuples += e2e_step()
        e1.record(stream)
        barrier()
    e2e_ms = e0.elapsed_time(e1)
    host_per_step = {k: v / a.steps for k, v in host.items()}
    phases = e2e_phases(eng, wl, pinned)
    # profiled step: an event pair around every launch
    eng.profile_reset()
    eng.set_profile(True)
    device_step()
    eng.set_profile(False)
    prof = eng.profile()
    sort_prof = None
    if a.workload == "sg_rmat_s14":
        # the same step on the sorted-list path (radix sort + merge-path
        # dedup of every candidate; the path for domains too large for
        # bitmaps), so that its kernels get a measured fraction too
        eng.set_tuning(dedup="sort")
        device_step()
        eng.profile_reset()
        eng.set_profile(True)
        device_step()
        eng.set_profile(False)
        sort_prof = eng.profile()
    eng.close()

    vals = torch.tensor([ms_total, float(tuples), e2e_ms, float(e2e_tuples)], dtype=torch.float64,
                        device=dev)
    if dist:
        mx = vals.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = vals.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms_total, e2e_ms = mx[0].item(), mx[2].item()
        tuples, e2e_tuples = sm[1].item(), sm[3].item()
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks = measured_peaks()
    line = {
        "metric": "derived tuples/s (SG fixpoint)" if a.workload == "sg_rmat_s14"
        else "derived tuples/s", "value": tuples / (ms_total / 1e3), "unit": "tuples/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_total / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": wl["desc"], "program": wl["prog"].__name__,
                   "tuples_per_step": tuples / a.steps / world,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "tuning": tuning,
                   "l2": "flushed between steps (256 MB write); within a step the bitmaps "
                         "(2^(2*bits) bits, 32 MB each at 2^14 ids, about five in use at once) "
                         "are partly resident in the 126 MB L2"},
        "e2e": {"value": e2e_tuples / (e2e_ms / 1e3), "unit": "tuples/s",
                "h2d_bytes_per_step": int(sum(x.nbytes for x in pinned)),
                "d2h_bytes_per_step": 16 * n_out[0]},
        "gpu_launches": int(kernels),
        "roofline": roofline_of(prof, a.workload, peaks),
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 4),
                        "gbs": (v["bytes"] / (v["ms"] / 1e3) / 1e9) if v["ms"] else None,
                        "frac": (v["bytes"] / (v["ms"] / 1e3) / 1e9 / peaks["hbm_gbs"])
                        if v["ms"] else None}
                    for k, v in prof.items() if v["launches"]},
        "clocks": clocks.summary(),
        "host_ms_per_step": host_per_step,
        "e2e_phases_ms": phases,
    }
    if sort_prof is not None:
        line["sort_path"] = {
            "workload": "the same step with dedup=sort (sorted lists, radix sort + merge)",
            "step_ms": round(sum(v["ms"] for v in sort_prof.values()), 4),
            "roofline": roofline_of(sort_prof, "sg_rmat_s14_sort", peaks),
            "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 4),
                            "frac": (v["bytes"] / (v["ms"] / 1e3) / 1e9 / peaks["hbm_gbs"])
                            if v["ms"] else None}
                        for k, v in sort_prof.items() if v["launches"]}}
    if world == 1 and not a.no_cpu_baseline and not wl.get("no_cpu"):
        runs = [oracle_run(wl, inputs) for _ in range(3)]
        secs = statistics.median(r[0] for r in runs)
        t, threads = runs[0][1], runs[0][2]
        line["cpu_baseline"] = {"value": t / secs, "unit": "tuples/s", "cores": threads,
                                "kind": "port",
                                "sample": "median of 3 full runs of the same workload on the "
                                          "CPU oracle (fixpoint seconds)"}
    elif wl.get("no_cpu"):
        line["cpu_baseline"] = {"value": None, "unavailable":
                                "the CPU oracle would need many minutes (or more host memory) "
                                "for this workload"}
    print(json.dumps(line), flush=True)


def run_reference(a) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    if a.workload == "dag_batch384":
        run_reference_dag(a, world)
        return
    wl = WORKLOADS[a.workload]
    if wl.get("no_cpu"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "the CPU implementation would need many minutes (or more host "
                          "memory) for this workload"}), flush=True)
        return
    inputs = wl["make"]()
    secs0, _, _ = oracle_run(wl, inputs)  # one warm-up run (CPU caches, page faults)
    budget = 330.0  # seconds of timed CPU work
    steps = max(1, min(a.steps, int(budget // max(secs0, 1e-3))))
    total, tuples, threads = 0.0, 0, 0
    for _ in range(steps):
        s, t, threads = oracle_run(wl, inputs)
        total += s
        tuples += t
    v = tuples / total
    line = {
        "impl": "reference", "metric": "derived tuples/s (SG fixpoint)"
        if a.workload == "sg_rmat_s14" else "derived tuples/s",
        "value": v, "unit": "tuples/s", "n_gpus": world,
        # what ran: `steps` timed runs after one warm-up run (each run is
        # the whole workload; the steps are capped by a CPU-time budget)
        "steps": steps, "warmup": 1, "steps_requested": a.steps,
        "warmup_requested": a.warmup,
        "ms_per_step": total / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": wl["desc"], "program": wl["prog"].__name__,
                   "parallelism": "cpu"},
        "cpu_baseline": {"value": v, "unit": "tuples/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full run(s) of the workload, after one warm-up run"},
        "e2e": {"value": v, "unit": "tuples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        gpu = False
    if gpu:
        ref = reference_gpu_live(a.workload, inputs)
        if ref:
            line["reference_gpu"] = ref
    print(json.dumps(line), flush=True)


def run_reference_dag(a, world) -> None:
    """The reference arm of the batched workload: one plain fixpoint per DAG
    (the reference has no batched form) on the CPU, over a bounded sample."""
    import batch as B
    from gdlog_b200 import Engine
    dags = W.dag_batch(384)
    inst = [(e,) for (_, _, e) in dags[:4]]
    with Engine("oracle") as o:
        B.run_plain_loop(o, P.tc, inst[:1])  # warm-up
        r = B.run_plain_loop(o, P.tc, inst)
        threads = o.threads
    v = len(inst) / r.seconds
    print(json.dumps({
        "impl": "reference", "metric": "batched TC instances/s (384 layered DAGs)", "value": v,
        "unit": "instances/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 384 / v * 1e3, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "384 layered DAGs, L in [8,128], W in [16,256] log-uniform",
                   "program": "tc", "parallelism": "cpu"},
        "cpu_baseline": {"value": v, "unit": "instances/s", "cores": threads, "kind": "port",
                         "sample": "the first 4 of the 384 DAGs, one plain fixpoint each"},
        "e2e": {"value": v, "unit": "instances/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def run_dag_batch(a) -> None:
    """Batched TC over 384 layered DAGs (L log-uniform in [8,128], W in
    [16,256], 2 out-edges per node, seed 2024 + instance): one batched
    fixpoint vs a loop of plain single-instance fixpoints, instances/s on
    device time, every instance checked bit-exact between the two."""
    import torch

    import batch as B
    from gdlog_b200 import Engine

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dags = W.dag_batch(384)
    # Instances are independent: each rank takes its share (largest first to
    # the least-loaded rank; cost ~ closure size ~ L * W^2), no exchange.
    mine = B.shard_instances([float(L) * Wd * Wd for (L, Wd, _) in dags], world, rank)
    dags = [dags[i] for i in mine]
    inst = [(e,) for (_, _, e) in dags]
    counts = [L * Wd for (L, Wd, _) in dags]
    eng = Engine("gpu", device=local)
    import autotune as A
    tuner = A.Tuner()
    tkey = f"{tuner.gpu}|{A.batch_bucket('tc', inst)}"
    if a.tune:
        # the batched fixpoint's device time under every candidate (the
        # sort path does not take the batched form: dense candidates only)
        space = dict(A.SPACE, dedup=["dense"])
        rec = tuner.tune_runner(
            eng, tkey, lambda e: B.run_batched(e, P.tc, inst, node_counts=counts).device_ms,
            space=space, reps=1)
        print(json.dumps({"tuned": "dag_batch384", "bucket": tkey, **rec}), flush=True)
        eng.close()
        return
    rec = tuner.apply_key(eng, tkey)
    tuning = rec["config"] if rec else "engine defaults (no cached tuning for this size bucket)"
    if a.single:
        eng.profile_reset()
        eng.set_profile(True)
        rb = B.run_batched(eng, P.tc, inst, node_counts=counts)
        eng.set_profile(False)
        print(json.dumps({"single_step_ms": rb.device_ms, "launches": rb.kernels,
                          "families": single_families(eng.profile())}), flush=True)
        eng.close()
        return
    for _ in range(a.warmup):
        B.run_batched(eng, P.tc, inst, node_counts=counts)
    ms_b, wall_b = [], []
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            rb = B.run_batched(eng, P.tc, inst, node_counts=counts)
            ms_b.append(rb.device_ms)
            wall_b.append(rb.seconds)
    # the plain loop warmed up as the batched steps were (every instance once:
    # its graphs instantiated and cached), then timed
    B.run_plain_loop(eng, P.tc, inst)
    rp = B.run_plain_loop(eng, P.tc, inst)
    same = sum((x.sizes, x.digests, x.iterations) == (y.sizes, y.digests, y.iterations)
               for x, y in zip(rb.results, rp.results))
    # profiled batched step: an event pair around every launch
    eng.profile_reset()
    eng.set_profile(True)
    B.run_batched(eng, P.tc, inst, node_counts=counts)
    eng.set_profile(False)
    prof = eng.profile()
    eng.close()
    ms = statistics.median(ms_b)
    wall = statistics.median(wall_b)
    tuples = sum(r.sizes["path"] for r in rb.results)
    plain_ms = rp.device_ms
    if dist:
        v = torch.tensor([ms, wall, plain_ms, float(tuples), float(same)], dtype=torch.float64,
                         device=torch.device("cuda", local))
        mx, sm = v.clone(), v.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms, wall, plain_ms = mx[0].item(), mx[1].item(), mx[2].item()
        tuples, same = int(sm[3].item()), int(sm[4].item())
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "batched TC instances/s (384 layered DAGs)", "value": 384 / (ms / 1e3),
        "unit": "instances/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": "384 layered DAGs, L in [8,128], W in [16,256] log-uniform",
                   "program": "tc", "tuples_per_step": tuples, "tuning": tuning,
                   "parallelism": f"instances sharded over {world} ranks (LPT, no exchange)"
                   if world > 1 else "single"},
        "e2e": {"value": 384 / wall, "unit": "instances/s",
                "h2d_bytes_per_step": int(sum(x[0].nbytes for x in inst)) * world,
                "d2h_bytes_per_step": 384 * 16},
        "plain_loop": {"value": 384 / (plain_ms / 1e3), "unit": "instances/s", "ms": plain_ms},
        "batched_over_plain": plain_ms / ms,
        "bit_exact_instances": f"{same}/384",
        "gpu_launches": rb.kernels, "clocks": clocks.summary(),
        "roofline": roofline_of(prof, "dag_batch384", measured_peaks()),
    }
    if world == 1 and not a.no_cpu_baseline:
        # bounded sample (~20 s on 16 cores): the first 4 DAGs, one after
        # another on the oracle
        from gdlog_b200 import Engine as _E
        with _E("oracle") as o:
            ro = B.run_plain_loop(o, P.tc, inst[:4])
            cores = o.threads
        line["cpu_baseline"] = {"value": 4 / ro.seconds, "unit": "instances/s",
                                "cores": cores, "kind": "port",
                                "sample": "the first 4 of the 384 DAGs, one plain fixpoint "
                                          "each on the CPU oracle (wall time)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sg_rmat_s14", choices=sorted(WORKLOADS) + ["dag_batch384"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--single", action="store_true",
                    help="run one device step and exit (for profiler captures)")
    ap.add_argument("--tune", action="store_true",
                    help="autotune this workload's size bucket, save the cache, and exit")
    a = ap.parse_args()
    if a.warmup < 3 and a.impl == "ours":
        a.warmup = 3
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "dag_batch384":
        run_dag_batch(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
