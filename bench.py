#!/usr/bin/env python3
"""Benchmark: ms per kaffpa-fast partition of a 2D random geometric graph,
n = 2^24 (r = 0.55*sqrt(ln n / n), ~265M directed CSR entries, int32, unit
weights), k = 64, imbalance 3%, seed 0, on one B200 -- plus the LP sweep's
achieved HBM bandwidth against the measured peak and the edge cut.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms
  ours       value   = device-resident ms per partition (graph already in HBM,
                       kb200_kaffpa_device), CUDA events on the library's stream
             e2e     = the same through the host C ABI (kb200_kaffpa, pinned
                       host CSR in, part[] out), H2D + D2H inside the timer
  reference  the reference kaffpa() (KaHIP built from its sources into
             oracle/_ref) on the full workload graph, on the host cores:
             K partitions (one per step, seeds W..W+K-1) run as concurrent
             single-threaded processes; value = wall / K.  The 1-process
             latency (seed 0 alone) is reported beside it.

With N > 1 (torchrun), every rank partitions its own replica (weak scaling,
no collective on the data path); value = max-over-ranks time / (K*N).
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms per kaffpa-fast partition & GE/s LP sweep (% HBM peak); cut vs plain at eps=3%"
FULL_LOGN = 24

# single-graph workloads: generator, description, log2 size of the bounded
# reference sample
GRAPH_KINDS = {
    "rgg2d": ("RGG2D", "r=0.55*sqrt(ln n/n), unit weights", 22),
    "rgg3d": ("RGG3D", "r=0.55*cbrt(ln n/n), unit weights", 20),
    "rmat": ("R-MAT", "16n samples, a,b,c,d=.57,.19,.19,.05, duplicate multiplicity as edge weight", 14),
}


def make_graph(kind: str, logn: int):
    from kahip_b200 import graphs
    if kind == "rgg2d":
        return graphs.rgg2d(1 << logn, seed=0)
    if kind == "rgg3d":
        return graphs.rgg3d(1 << logn, seed=0)
    return graphs.rmat(logn, seed=0)
K_BLOCKS = 64
IMBALANCE = 0.03
MODE_FAST = 0
MODES = {"fast": 0, "eco": 1}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--logn", type=int, default=FULL_LOGN, help="log2 of the RGG size (default 24)")
    p.add_argument("--k", type=int, default=K_BLOCKS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", choices=["rgg", "batch", "population", "learned", "evolve"], default="rgg",
                   help="rgg: the headline single-graph workload (default); batch: many independent graphs "
                        "of uneven size; population: many seeds of one device-resident RGG2D n=2^20")
    p.add_argument("--mode", choices=["fast", "eco"], default="fast",
                   help="kaffpa preset of the single-graph workload (fast, the headline: LP refinement; "
                        "eco: Jet refinement)")
    p.add_argument("--graph", choices=sorted(GRAPH_KINDS), default="rgg2d",
                   help="single-graph workload kind (default rgg2d, the headline)")
    p.add_argument("--batch-count", type=int, default=512, help="graphs in the batch workload")
    p.add_argument("--learned-logn", type=int, default=23,
                   help="learned workload: RGG2D n=2^L and R-MAT n=2^(L-1) (default 23)")
    p.add_argument("--population", type=int, default=64, help="seeds in the population workload")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 10:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        rows = [r for r in self.rows if self.uuid is None or r[1] == self.uuid] or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[2]) for r in rows if num(r[2]) is not None]
        mx = [num(r[3]) for r in rows if num(r[3]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, val in zip(names, r[6:10]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------ reference arm
#
# The reference kaffpa() (KaHIP built from its sources into oracle/_ref, its
# own interface/kaHIP_interface.cpp entry point) partitions the FULL workload
# graph, in-process, in worker processes that map one shared copy of the CSR.
# kaffpa is single-threaded, so the host cores run independent partitions
# (seed = step index) concurrently; each worker times its kaffpa() call alone
# (the reference CLI's "time spent for partitioning", app/kaffpa.cpp:79,118).

# reference presets: R-MAT uses fastsocial (the reference's LP preset) because
# reference fast does not finish in reasonable time on it (and misses the
# balance bound); every other graph uses the arm's own preset
REF_MODE_FOR_RMAT = 3


def ref_mode(args) -> int:
    return REF_MODE_FOR_RMAT if args.graph == "rmat" else MODES[args.mode]


def _ref_worker_init():
    os.environ["KBGEN_THREADS"] = "1"


def _ref_full_task(task):
    """One reference kaffpa() on the shared graph: (ms, cut, peak RSS bytes)."""
    import resource

    import numpy as np

    from oracle import oracle
    gdir, unit, k, seed, mode = task
    g = {key: np.load(os.path.join(gdir, key + ".npy"), mmap_mode="r") for key in ("xadj", "adjncy", "adjwgt", "vwgt")}
    g["n"] = len(g["xadj"]) - 1
    if unit:
        g["vwgt"] = g["adjwgt"] = None
    t = time.perf_counter()
    cut, _ = oracle.ref_kaffpa(g, k, IMBALANCE, seed, mode)
    ms = (time.perf_counter() - t) * 1e3
    return ms, int(cut), resource.getrusage(resource.RUSAGE_SELF).ru_maxrss * 1024


# peak resident bytes of one reference kaffpa process per directed entry
# (graph_access edges, ratings, coarse levels and the mapped input: 52 B
# measured on RGG2D n=2^22, fast, k=64), with a margin
REF_BYTES_PER_ENTRY = 64


def host_procs_for_reference(m_directed: int) -> int:
    n = os.cpu_count() or 1
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) for l in f if l.startswith("MemAvailable")) * 1024
        n = min(n, max(1, int(avail // max(1, REF_BYTES_PER_ENTRY * m_directed))))
    except (OSError, StopIteration):
        pass
    return max(1, n)


class SharedGraph:
    """The workload graph written once as .npy files (tmpfs where there is
    one) for the reference workers to map."""

    def __init__(self, g: dict):
        import shutil
        import tempfile

        import numpy as np
        base = "/dev/shm" if os.path.isdir("/dev/shm") else None
        need = sum(g[k].nbytes for k in ("xadj", "adjncy", "adjwgt", "vwgt"))
        if base and shutil.disk_usage(base).free < 2 * need:
            base = None
        self.dir = tempfile.mkdtemp(prefix="kb200_ref_", dir=base)
        for key in ("xadj", "adjncy", "adjwgt", "vwgt"):
            np.save(os.path.join(self.dir, key + ".npy"), g[key])

    def close(self):
        import shutil
        shutil.rmtree(self.dir, ignore_errors=True)


def reference_runs(gdir: str, unit: bool, k: int, mode: int, seeds, procs: int):
    """Runs the reference on `seeds` with `procs` concurrent processes;
    returns (wall ms, [(ms, cut, rss)])."""
    ctx = mp.get_context("spawn")
    t = time.perf_counter()
    with ctx.Pool(procs, initializer=_ref_worker_init) as pool:
        res = pool.map(_ref_full_task, [(gdir, unit, k, s, mode) for s in seeds], chunksize=1)
    return (time.perf_counter() - t) * 1e3, res


def run_reference_arm(args, rank):
    if rank != 0:
        return
    from oracle import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkahip_ref.so was not built "
                          "(reference sources absent when __graft_entry__.build() ran)"}))
        return
    g = make_graph(args.graph, args.logn)
    m_full = g["m"]
    unit = args.graph != "rmat"
    mode = ref_mode(args)
    procs = host_procs_for_reference(m_full)
    shared = SharedGraph(g)
    del g
    try:
        # warm-up: seed 0 alone (the 1-process latency and the cut on the
        # timed workload's own seed), then the other warm-up seeds together
        _, solo = reference_runs(shared.dir, unit, args.k, mode, [0], 1)
        if args.warmup > 1:
            reference_runs(shared.dir, unit, args.k, mode, list(range(1, args.warmup)),
                           min(procs, args.warmup - 1))
        # timed: K partitions (seeds W .. W+K-1) in waves of equal size on
        # the host cores; value = wall / K
        waves = -(-args.steps // procs)
        conc = -(-args.steps // waves)
        wall, res = reference_runs(shared.dir, unit, args.k, mode,
                                   list(range(args.warmup, args.warmup + args.steps)), conc)
    finally:
        shared.close()
    value = wall / args.steps
    per = [r[0] for r in res]
    cuts = [r[1] for r in res]
    mode_name = {0: "fast", 1: "eco", 3: "fastsocial"}.get(mode, str(mode))
    sample = (f"full workload: reference kaffpa {mode_name} (KaHIP built from its sources, its kaffpa() entry "
              f"point, single-threaded) on {GRAPH_KINDS[args.graph][0]} n=2^{args.logn} (m_directed={m_full}); "
              f"{args.steps} partitions (seeds {args.warmup}..{args.warmup + args.steps - 1}) in {waves} wave(s) "
              f"of {conc} concurrent processes; ms per partition = wall / {args.steps}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": f"synthetic (seeded {GRAPH_KINDS[args.graph][0]} generator)",
        "config": workload_config(args, m_full),
        "cpu_baseline": {"value": value, "unit": "ms", "cores": conc, "kind": "reference", "sample": sample,
                         "latency_1proc": {"value": solo[0][0], "unit": "ms", "cores": 1,
                                           "sample": f"seed 0 alone, cut {solo[0][1]}"},
                         "per_partition_ms_under_load": {"mean": statistics.mean(per), "min": min(per),
                                                         "max": max(per)},
                         "peak_rss_bytes_per_process": max(r[2] for r in res)},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_preset": mode_name,
        "reference_cut_seed0": solo[0][1],
        "reference_cut_mean": statistics.mean(cuts),
        "host": host_description(),
    }
    print(json.dumps(line))


def host_description() -> dict:
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            model = next((l.split(":", 1)[1].strip() for l in f if l.startswith("model name")), None)
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def workload_config(args, m):
    name, desc, _ = GRAPH_KINDS[args.graph]
    return {"workload": f"kaffpa {args.mode} on {name} n=2^{args.logn} ({desc}), k={args.k}, eps=3%",
            "n": 1 << args.logn, "m_directed": m, "k": args.k, "imbalance": IMBALANCE, "preset": args.mode,
            "seed": 0, "graph_seed": 0, "l2": "inputs (~2.2 GB CSR) exceed the 126 MB L2; no flush",
            "parallelism": "replicas" if args.gpus > 1 else "single GPU"}


# ------------------------------------------------------------------- ours

def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    from kahip_b200 import graphs, native, replicas

    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if args.workload == "evolve":
        if rank == 0:
            run_evolve(args)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload == "learned":
        run_learned(args, rank, dev)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.workload != "rgg":
        run_many(args, world, rank, dev)
        if world > 1:
            dist.destroy_process_group()
        return

    g = make_graph(args.graph, args.logn)
    unit = args.graph != "rmat"
    n, m = g["n"], g["m"]
    d_xadj = torch.from_numpy(g["xadj"]).to(dev)
    d_adj = torch.from_numpy(g["adjncy"]).to(dev)
    d_w = torch.from_numpy(g["adjwgt"]).to(dev)
    d_vw = torch.from_numpy(g["vwgt"]).to(dev)
    d_part = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def call(st=None):
        return native.kaffpa_device(n, d_xadj, d_adj, d_w, d_vw, d_part, args.k, IMBALANCE, 0, MODES[args.mode],
                                    stream=stream, stats=st)

    for _ in range(max(3, args.warmup)):
        call()
    torch.cuda.synchronize()

    # ---- timed region: K device-resident partitions, instrumented ----
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    fam = {}
    cuts = []
    sweep_v = sweep_e = sweep_o = 0
    ms_phase = {"coarsen": 0.0, "initial": 0.0, "uncoarsen": 0.0}
    levels = None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = native.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # inside the timed region only the roofline family (the LP clustering
    # sweep) is bracketed by CUDA events (timing 2): events around every
    # family cost about 2.5 ms of host time per call at this size
    ev0.record(stream)
    for _ in range(args.steps):
        st = native.Stats()
        st.timing = 2
        rc, cut = call(st)
        cuts.append(cut)
        for name, f in st.families().items():
            a = fam.setdefault(name, {"ms": 0.0, "bytes": 0.0, "launches": 0})
            a["ms"] += f["ms"]
            a["bytes"] += f["bytes"]
            a["launches"] += f["launches"]
        sweep_v += st.sweep_vertices
        sweep_e += st.sweep_edges
        sweep_o += st.sweep_overflow_vertices
        ms_phase["coarsen"] += st.ms_coarsen
        ms_phase["initial"] += st.ms_initial
        ms_phase["uncoarsen"] += st.ms_uncoarsen
        levels = [(st.level_n[i], st.level_m[i]) for i in range(st.levels)]
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = native.kernel_launches() - launches0
    sampler.stop()
    elapsed = replicas.max_over_ranks(ev0.elapsed_time(ev1), dev)
    ms_per_step = elapsed / args.steps
    value = elapsed / (args.steps * world)

    # breakdown: every kernel family timed, in calls after the timed region
    br_steps = max(1, min(3, args.steps))
    fam_all = {}
    eb0 = torch.cuda.Event(enable_timing=True)
    eb1 = torch.cuda.Event(enable_timing=True)
    eb0.record(stream)
    for _ in range(br_steps):
        st = native.Stats()
        st.timing = 1
        call(st)
        for name, f in st.families().items():
            a = fam_all.setdefault(name, {"ms": 0.0, "bytes": 0.0, "launches": 0})
            a["ms"] += f["ms"]
            a["bytes"] += f["bytes"]
            a["launches"] += f["launches"]
    eb1.record(stream)
    torch.cuda.synchronize()
    instrumented_ms = eb0.elapsed_time(eb1) / br_steps

    # quality of the (deterministic) partition of the last timed call
    part = d_part.cpu().numpy()
    bw = np.bincount(part, minlength=args.k)
    kn = native.derive_knobs(n, None, args.k, IMBALANCE, 0, MODES[args.mode])

    # ---- end to end through the host C ABI (pinned host buffers) ----
    h_xadj = torch.from_numpy(g["xadj"]).pin_memory()
    h_adj = torch.from_numpy(g["adjncy"]).pin_memory()
    h_w = None if unit else torch.from_numpy(g["adjwgt"]).pin_memory()
    h_part = torch.empty(n, dtype=torch.int32).pin_memory()
    L = native.lib()
    import ctypes
    e2e_cut = ctypes.c_longlong()

    def e2e_call():
        rc = L.kb200_kaffpa(n, None, h_xadj.data_ptr(), None if h_w is None else h_w.data_ptr(), h_adj.data_ptr(),
                            args.k, IMBALANCE, 0, MODES[args.mode],
                            ctypes.byref(e2e_cut), h_part.data_ptr(), None)
        if rc < 0:
            raise RuntimeError(L.kb200_last_error().decode())

    # untimed warm-up of the host path (its first call sizes the arenas for a
    # copied input)
    for _ in range(max(1, min(args.warmup, 2))):
        e2e_call()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        e2e_call()
    e2e_ms = replicas.max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, dev) / world
    e2e_same = bool(np.array_equal(h_part.numpy(), part)) and e2e_cut.value == cuts[-1]

    # ---- roofline: the LP clustering sweep (every vertex swept once per round) ----
    peak, peak_kind = measured_peaks()
    sweep = fam.get("lp_cluster_sweep", {"ms": 0, "bytes": 0, "launches": 0})
    achieved = sweep["bytes"] / (sweep["ms"] * 1e-3) / 1e9 if sweep["ms"] else None
    bytes_per_launch = sweep["bytes"] / max(1, sweep["launches"])
    # DRAM traffic per launch: the DRAM/algorithmic ratio of an ncu capture of
    # the same kernel (profiles/lp_cluster_sweep_traffic.json) applied to this
    # run's algorithmic bytes per launch
    traffic = None
    traffic_src = None
    tpath = os.path.join(ROOT, "profiles", "lp_cluster_sweep_traffic.json")
    if os.path.exists(tpath) and bytes_per_launch:
        with open(tpath) as f:
            tj = json.load(f)
        if tj.get("dram_over_algorithmic"):
            traffic = tj["dram_over_algorithmic"] * bytes_per_launch
            traffic_src = f"ncu dram bytes / algorithmic bytes = {tj['dram_over_algorithmic']} ({tj['workload']})"
    total_fam_ms = sum(f["ms"] for f in fam_all.values()) or 1.0
    sweep_all = fam_all.get("lp_cluster_sweep", {"ms": 0})
    roofline = {
        "kernel": "lp_cluster_sweep (lane_kernel<CLUSTER> + chunk_process + heavy_kernel)", "bound": "hbm",
        "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "peak_source": f"hbm_gbs of {peak_kind}",
        "traffic": traffic, "traffic_source": traffic_src,
        "bytes_per_launch": bytes_per_launch,
        "ms_per_launch": sweep["ms"] / max(1, sweep["launches"]),
        "share_of_timed_kernels": sweep_all["ms"] / total_fam_ms,
        "ge_per_s": (sweep_e / args.steps / (sweep["ms"] / args.steps * 1e-3) / 1e9) if sweep["ms"] else None,
    }

    line = {
        "metric": METRIC, "value": value, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": f"synthetic (seeded {GRAPH_KINDS[args.graph][0]} generator)",
        "config": workload_config(args, m),
        "roofline": roofline,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 4 * (n + 1 + m) + (0 if unit else 4 * m),
                "d2h_bytes_per_step": 4 * n, "api": "kb200_kaffpa (host C ABI, pinned buffers, NULL = unit weights)",
                "same_partition_as_device_path": e2e_same},
        "gpu_launches": launches,
        "clocks": sampler.summary(),
        "quality": {"cut": cuts[-1], "max_block": int(bw.max()), "bound": int(kn.final_bound),
                    "balanced": bool(bw.max() <= kn.final_bound), "deterministic_over_steps": len(set(cuts)) == 1},
        "phases_ms_per_step": {k: v / args.steps for k, v in ms_phase.items()},
        "kernel_families_ms_per_step": {k: v["ms"] / br_steps
                                        for k, v in sorted(fam_all.items(), key=lambda x: -x[1]["ms"])},
        "kernel_families_source": (f"{br_steps} calls after the timed region with every family bracketed by "
                                   f"CUDA events ({instrumented_ms:.2f} ms per call so instrumented)"),
        "levels": levels,
        "sweep_work_per_step": {"vertices": sweep_v / args.steps, "edges": sweep_e / args.steps,
                                "overflow_vertices": sweep_o / args.steps},
    }

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        if oracle.ref_available():
            # the reference kaffpa() on the same full graph, alone on one core
            mode = ref_mode(args)
            shared = SharedGraph(g)
            try:
                _, res = reference_runs(shared.dir, unit, args.k, mode, [0], 1)
            finally:
                shared.close()
            mode_name = {0: "fast", 1: "eco", 3: "fastsocial"}.get(mode, str(mode))
            line["cpu_baseline"] = {
                "value": res[0][0], "unit": "ms", "cores": 1, "kind": "reference",
                "sample": (f"full workload: one reference kaffpa {mode_name} run (KaHIP built from its sources, its "
                           f"kaffpa() entry point, single-threaded) on the same {GRAPH_KINDS[args.graph][0]} "
                           f"n=2^{args.logn} graph (m_directed={m}), seed 0"),
                "reference_cut": res[0][1], "host": host_description()}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "ms", "cores": 0, "kind": "reference",
                                    "sample": "unavailable: oracle/_ref not built"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ------------------------------------------------------ learned edge rating

def run_learned(args, rank, dev):
    """Held-out evaluation of the learned edge rating: RGG2D n=2^23 and R-MAT
    n=2^22 (16n samples), k=64, eps=3%, kaffpa fast knobs with three
    coarsenings -- LP clustering (the default), heavy-edge matching on
    expansion*^2 (the plain rating) and on the learned rating -- device
    resident, CUDA events on the library's stream.  value = ms per partition
    of the learned form on the RGG2D graph."""
    import ctypes

    import numpy as np
    import torch

    from kahip_b200 import graphs, native
    from kahip_b200.learned import load_model

    model = load_model()
    if model is None:
        if rank == 0:
            print(json.dumps({"metric": "learned edge rating", "unavailable": "kahip_b200/data/rating_mpnn.f32 absent"}))
        return
    P, meta = model
    results = {}
    stream = torch.cuda.Stream(device=dev)
    L = args.learned_logn
    for name, g in ((f"rgg2d_2^{L}", graphs.rgg2d(1 << L, seed=77)), (f"rmat_2^{L - 1}", graphs.rmat(L - 1, seed=78))):
        n = g["n"]
        t = {key: torch.from_numpy(np.ascontiguousarray(g[key], np.int32)).to(dev)
             for key in ("xadj", "adjncy", "adjwgt", "vwgt")}
        part = torch.empty(n, dtype=torch.int32, device=dev)
        res = {"n": n, "m_directed": g["m"]}
        for label, coarsening, guard, levels in (("lp", 0, 0.0, 0), ("plain_rating", 1, 0.0, 0),
                                                 ("learned_rating", 2, 0.0, 0),
                                                 ("learned_rating_level0", 2, 0.0, 1),
                                                 ("learned_rating_levels01", 2, 0.0, 2),
                                                 ("learned_rating_guarded", 2, 1.0, 0)):
            kn = native.derive_knobs(n, g["vwgt"], 64, IMBALANCE, 0, MODE_FAST)
            kn.coarsening = coarsening
            kn.rating_model = P.ctypes.data_as(ctypes.c_void_p) if coarsening == 2 else None
            kn.rating_fallback = guard
            kn.rating_levels = levels
            for _ in range(max(1, args.warmup)):
                native.kaffpa_device_knobs(n, t["xadj"], t["adjncy"], t["adjwgt"], t["vwgt"], part, kn, stream=stream)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            st = native.Stats()
            e0.record(stream)
            for _ in range(args.steps):
                _, cut = native.kaffpa_device_knobs(n, t["xadj"], t["adjncy"], t["adjwgt"], t["vwgt"], part, kn,
                                                    stream=stream, stats=st)
            e1.record(stream)
            torch.cuda.synchronize()
            bw = np.bincount(part.cpu().numpy(), minlength=64)
            res[label] = {"ms": e0.elapsed_time(e1) / args.steps, "cut": int(cut),
                          "balanced": bool(bw.max() <= kn.final_bound), "levels": st.levels,
                          "ms_coarsen": st.ms_coarsen, "ms_initial": st.ms_initial,
                          "ms_uncoarsen": st.ms_uncoarsen}
        res["learned_over_plain_cut"] = res["learned_rating"]["cut"] / max(1, res["plain_rating"]["cut"])
        res["learned_over_plain_ms"] = res["learned_rating"]["ms"] / max(1e-9, res["plain_rating"]["ms"])
        results[name] = res
        del t, part
        torch.cuda.empty_cache()
    if rank != 0:
        return
    line = {
        "metric": "ms per kaffpa-fast partition with the learned-rating matching; cut vs the plain rating",
        "value": results[f"rgg2d_2^{L}"]["learned_rating"]["ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": False, "dtype": "bf16 (network) / int32 (partitioning)",
        "data": "synthetic (seeded generators), held out from training",
        "config": {"workload": f"learned edge rating: RGG2D n=2^{L} and R-MAT n=2^{L - 1}, k=64, eps=3%",
                   "model": {k: meta[k] for k in ("training_graphs", "steps", "validated") if k in meta}},
        "results": results,
    }
    print(json.dumps(line))


def run_evolve(args):
    """KaFFPaE-style evolution (kb200_kaffpae) on RGG2D n=2^20, k=64, eps=3%:
    population 8 (seeds 0..7), 4 rounds of 4 combines each, for both presets.
    value = ms per call of the eco form through the host C ABI (graph upload
    and partition download included; wall clock around the call, the
    library synchronises before returning), with the best cut after the
    initial population and after every round."""
    import time

    import numpy as np

    from kahip_b200 import graphs, native

    g = graphs.rgg2d(1 << 20, seed=0)
    P, G, W = 8, 4, 4
    res = {}
    for name, mode in (("fast", MODES["fast"]), ("eco", MODES["eco"])):
        kn = native.derive_knobs(g["n"], None, K_BLOCKS, IMBALANCE, 0, mode)
        native.kaffpae(g, kn, P, 1, 1, unit_weights=True)  # warm-up (contexts, arenas)
        t0 = time.perf_counter()
        _, cut, part, hist = native.kaffpae(g, kn, P, G, W, unit_weights=True)
        ms = (time.perf_counter() - t0) * 1e3
        bw = np.bincount(part, minlength=K_BLOCKS)
        res[name] = {"ms": ms, "cut": int(cut), "history": [int(x) for x in hist],
                     "improvement_over_best_member": 1.0 - cut / max(1, int(hist[0])),
                     "balanced": bool(bw.max() <= kn.final_bound), "partitions": P + G * W}
    print(json.dumps({
        "metric": "ms per KaFFPaE-style evolution (8 members, 4 rounds x 4 combines); best cut per round",
        "value": res["eco"]["ms"], "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 1, "higher_is_better": False,
        "dtype": "int32", "data": "synthetic (seeded RGG2D generator)",
        "config": {"workload": "kaffpae on RGG2D n=2^20 (unit weights), k=64, eps=3%", "population": P,
                   "generations": G, "per_generation": W, "api": "kb200_kaffpae (host C ABI)"},
        "results": res}))


# ------------------------------------------------- batch / population forms

def _ref_batch_task(args):
    idx, count, seed = args
    from kahip_b200 import graphs
    from oracle import oracle
    spec = graphs.batch_specs(count, seed=seed)[idx]
    g, k = graphs.batch_graph(spec), spec[2]
    t = time.perf_counter()
    oracle.ref_kaffpa(dict(g, vwgt=None), k, IMBALANCE, idx, MODE_FAST)
    return (time.perf_counter() - t) * 1e3


def run_many(args, world, rank, dev):
    """Many independent partitions per step: `batch` (graphs of uneven size,
    n log-uniform in [1e3, 2e5], RGG2D / grid / R-MAT mix, k in {2..64}) or
    `population` (seeds of one device-resident RGG2D n=2^20, k=64).  value =
    partitions/s of the whole job; the serial GPU loop (one worker, same
    inputs) is timed beside it."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from kahip_b200 import graphs, native, replicas

    ranks_seed = 1000 * rank
    if args.workload == "batch":
        mix = graphs.batch_mix(args.batch_count, seed=ranks_seed)
        gs = [g for g, _ in mix]
        ks = [k for _, k in mix]
        seeds = list(range(len(gs)))
        nodes = sum(g["n"] for g in gs)
        entries = sum(g["m"] for g in gs)
        h2d = sum(4 * (g["n"] + 1 + 2 * g["m"] + g["n"]) for g in gs)
        d2h = sum(4 * g["n"] for g in gs)

        def step(workers):
            cuts, parts, status, rep = native.kaffpa_batch(gs, ks, IMBALANCE, seeds, MODE_FAST, workers=workers)
            assert rep.failed == 0
            return rep.ms_total, rep.workers, cuts

        count = len(gs)
        workload = (f"batch of {count} independent graphs, n log-uniform in [1e3, 2e5] (total {nodes} nodes, "
                    f"{entries} directed entries), RGG2D/grid/R-MAT mix, k in {{2..64}}, kaffpa fast, eps=3%")
    else:
        g = graphs.rgg2d(1 << 20, seed=0)
        n = g["n"]
        t = {key: torch.from_numpy(np.ascontiguousarray(g[key], np.int32)).to(dev)
             for key in ("xadj", "adjncy", "adjwgt", "vwgt")}
        count = args.population
        seeds = [replicas.member_seed(i, rank, world) for i in range(count)]
        parts = torch.empty(count * n, dtype=torch.int32, device=dev)
        nodes, entries, h2d, d2h = count * n, count * g["m"], 0, 0

        def step(workers):
            torch.cuda.synchronize()
            cuts, rep = native.kaffpa_population(n, t["xadj"], t["adjncy"], t["adjwgt"], t["vwgt"], parts, 64,
                                                 seeds, IMBALANCE, MODE_FAST, workers=workers)
            torch.cuda.synchronize()
            assert rep.failed == 0
            return rep.ms_total, rep.workers, cuts

        workload = (f"population of {count} seeds of one device-resident RGG2D n=2^20 "
                    f"({g['m']} directed entries), k=64, kaffpa fast, eps=3%")

    for _ in range(max(1, args.warmup)):
        step(0)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    if world > 1:
        dist.barrier()
    ms = []
    workers = 0
    launches0 = native.kernel_launches()
    for _ in range(args.steps):
        t_ms, workers, cuts = step(0)
        ms.append(t_ms)
    launches = native.kernel_launches() - launches0
    if world > 1:
        dist.barrier()
    sampler.stop()
    elapsed = replicas.max_over_ranks(sum(ms), dev)
    value = count * args.steps * world / (elapsed * 1e-3)
    serial_ms, _, cuts1 = step(1)
    same = bool(np.array_equal(np.asarray(cuts1), np.asarray(cuts)))
    cpu = None
    if rank == 0 and args.workload == "batch" and not args.no_cpu_baseline:
        from oracle import oracle
        if oracle.ref_available():
            procs = host_procs_for_reference(max(g["m"] for g in gs))
            sample = min(count, 4 * procs)
            ctx = mp.get_context("spawn")
            t0 = time.perf_counter()
            with ctx.Pool(procs, initializer=_ref_worker_init) as pool:
                pool.map(_ref_batch_task, [(i, args.batch_count, ranks_seed) for i in range(sample)])
            wall = time.perf_counter() - t0
            cpu = {"value": sample / wall, "unit": "partitions/s", "cores": procs, "kind": "reference",
                   "sample": f"reference kaffpa fast on the first {sample} graphs of the batch, {procs} processes"}
    if rank != 0:
        return
    line = {
        "metric": f"partitions/s ({args.workload} form)", "value": value, "unit": "partitions/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": elapsed / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (seeded generators)",
        "config": {"workload": workload, "workers": workers, "graphs_per_step": count,
                   "l2": "each step streams more than the 126 MB L2; no flush"},
        "serial_gpu_loop": {"value": count / (serial_ms * 1e-3), "unit": "partitions/s", "workers": 1,
                            "same_cuts_as_batched": same},
        "e2e": {"value": value, "unit": "partitions/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "kb200_kaffpa_batch" if args.workload == "batch" else "kb200_kaffpa_population"},
        "gpu_launches": launches,
        "clocks": sampler.summary(),
        "mean_cut": float(np.mean(cuts)),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
