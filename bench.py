"""Benchmark of the untangling hot path on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload folded256]

A step is one untangling pass over one batch of synthetic input (the precision-form
cloth scene: one 256 x 256-vertex sheet, 130,050 triangles, folded once about a seeded
line with 0.3 x edge-length Gaussian vertex noise). The pass runs the stages built on
the device: face-tree refit, fused EF broad+narrow phase, canonical EF ordering.

value     = ray-primitive tests per second over the whole job (segment-triangle leaf
            tests of the pass), inputs resident in HBM, device time (CUDA events).
e2e       = the same metric through the public C ABI with host buffers: the positions
            are copied host->device and the EF list device->host inside the timed step.
roofline  = algorithmic bytes of the dominant kernel / its CUDA-event time vs the
            measured HBM copy bandwidth.
cpu_baseline = the CPU oracle of the same pass on the host cores (bounded sample).

--impl reference times the reference's algorithm on the host cores: the reference
cannot be built here (its LuisaCompute runtime is not in the checkout), so its CPU
restatement (the oracle port) runs with all host threads, same workload and metric.

Multi-GPU: the pass shards by independent scenes (weak scaling, no collective). With
--gpus N under torchrun each rank runs its own scene replica; value = total tests of
all ranks / max rank time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "ray-prim tests/s & untangle passes/s: chosen vs plain form, 1 B200, same hits"
UNIT = "ray-prim tests/s"


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name):
    from untangling26_b200 import synthetic
    if name == "folded256":
        return synthetic.folded_sheet(256, seed=1), {"workload": "folded_sheet_256x256", "triangles": 130050,
                                                     "fold_noise_sigma_edge_lengths": 0.3, "seed": 1}
    if name == "two_sheets64":
        return synthetic.two_sheets(64, seed=0), {"workload": "two_sheets_64x64", "triangles": 15876, "seed": 0}
    raise SystemExit(f"unknown workload {name}")


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_pass_oracle(mesh, d_hat, th):
    """One pass of the same stages with the CPU oracle; returns (tests, pairs)."""
    from oracle import oracle as o
    tree = o.lbvh_build(o.TREE_FACE, mesh.x, mesh.faces)
    o.lbvh_refit(tree, mesh.x, mesh.x, th, mesh.faces)
    broad, total, _ = o.lbvh_query(tree, o.QUERY_EDGES_UNCULLED, mesh.x, mesh.x, mesh.edges, d_hat, th)
    ef, idx = o.ef_narrow(broad, mesh.x, mesh.edges, mesh.faces, d_hat, mesh.vert_property)
    return total, len(ef)


def run_cpu(mesh, seconds=15.0):
    """Bounded CPU sample: repeat the oracle pass until ~`seconds` of work."""
    from oracle import oracle as o
    o.build()
    d_hat = np.full(mesh.num_verts, 1e-3, np.float32)
    th = np.zeros(mesh.num_verts, np.float32)
    cpu_pass_oracle(mesh, d_hat, th)  # warm
    t0 = time.perf_counter()
    n, tests = 0, 0
    while True:
        t, _ = cpu_pass_oracle(mesh, d_hat, th)
        tests += t
        n += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": tests / dt, "unit": UNIT, "cores": o.threads(), "kind": "port", "passes": n,
            "sample": f"{n} full passes (tree build + refit + EF broad/narrow phase) of the workload in {dt:.1f} s",
            "passes_per_s": n / dt}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="folded256")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    ws, rank, local = _dist_env()
    mesh, config = make_workload(args.workload)

    if args.impl == "reference":
        if rank != 0:
            return
        steps_sec = []
        from oracle import oracle as o
        o.build()
        d_hat = np.full(mesh.num_verts, 1e-3, np.float32)
        th = np.zeros(mesh.num_verts, np.float32)
        for _ in range(max(args.warmup, 0)):
            cpu_pass_oracle(mesh, d_hat, th)
        tests = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            t1 = time.perf_counter()
            t, _ = cpu_pass_oracle(mesh, d_hat, th)
            steps_sec.append(time.perf_counter() - t1)
            tests += t
        dt = time.perf_counter() - t0
        value = tests / dt
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": dict(config, parallelism="host threads", l2="n/a (CPU)"),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": o.threads(), "kind": "port",
                                 "sample": f"{args.steps} full passes of the workload (reference algorithm, CPU restatement; "
                                           "the reference's LuisaCompute runtime is absent so its own build cannot run)"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "untangle_passes_per_s": args.steps / dt}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist

    from untangling26_b200 import Context
    from untangling26_b200.intersection_resolver import CollisionScene

    if ws > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    ctx = Context(local)
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0, max_ef_pairs=max(1 << 16, mesh.num_edges))
    sc.construct_lbvh()
    dev = torch.device("cuda", local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def device_pass(stats=True):
        sc.detect_ef_fused(with_stats=stats)
        n = sc.resolver.ef_count  # stays on device
        return n

    # warm-up
    for _ in range(max(args.warmup, 3)):
        device_pass()
        sc.resolver.canonicalize(mesh.num_edges, mesh.num_faces)
    torch.cuda.synchronize()

    # ---- device-resident timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tests_total = 0
    launches0 = ctx.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record(stream)
        # refit + fused detect (the dominant kernel is timed on its own event pair)
        sc.refit_face_tree()
        sc.resolver.reset()
        sc.stats.zero_()
        kev[i][0].record(stream)
        sc.ef_detect(with_stats=True)
        kev[i][1].record(stream)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    kern_ms = [a.elapsed_time(b) for a, b in kev]
    st = sc.stats.cpu().numpy()
    nodes_per_pass, tests_per_pass = int(st[0]), int(st[1])
    tests_total = tests_per_pass * args.steps
    total_ms = sum(step_ms)
    if ws > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = tests_total * ws / (total_ms / 1e3)

    # ---- roofline of the dominant kernel (fused EF traversal): algorithmic bytes per launch
    # 44 B per node box tested (32 B box + 8 B children + 4 B object id), 48 B per leaf
    # triangle tested (12 B indices + 36 B positions), 28 B per edge query (8 B indices +
    # 24 B positions - shared), 48 + 8 B per EF pair written.
    n_ef = int(sc.resolver.ef_count.item())
    alg_bytes = 44 * nodes_per_pass + 48 * tests_per_pass + 32 * mesh.num_edges + 56 * n_ef
    kmean = statistics.mean(kern_ms)
    achieved = alg_bytes / (kmean / 1e3) / 1e9
    peak, peak_kind = _peaks()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_kind, "kernel": "ef_detect_kernel", "kernel_ms": kmean,
            "traffic": None, "algorithmic_bytes_per_launch": alg_bytes}
    prof = os.path.join(ROOT, "profiles", "ef_detect_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            roof["traffic"] = json.load(f).get("dram_bytes_per_launch")

    # ---- e2e through the C ABI with host buffers
    x_host = torch.from_numpy(mesh.x).pin_memory()
    out_host = torch.empty((sc.resolver.max_ef, 12), dtype=torch.int32).pin_memory()
    cnt_host = torch.empty(1, dtype=torch.int32).pin_memory()
    e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    d2h_bytes = 0
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        e_ev[i][0].record(stream)
        sc.x.copy_(x_host, non_blocking=True)
        device_pass(stats=False)
        cnt_host.copy_(sc.resolver.ef_count, non_blocking=True)
        stream.synchronize()
        k = int(cnt_host.item())
        sc.resolver.canonicalize(mesh.num_edges, mesh.num_faces)
        out_host[:k].copy_(sc.resolver.ef_list[:k], non_blocking=True)
        e_ev[i][1].record(stream)
        d2h_bytes = 4 + 48 * k
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e_ev)
    e2e_value = tests_per_pass * args.steps * ws / (e2e_ms / 1e3)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = run_cpu(mesh, args.cpu_seconds)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config, l2="flushed between steps (256 MB write)", parallelism=f"scene replica per GPU x{ws}",
                               stages="refit + fused EF detect (+ canonical sort in e2e)"),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(mesh.x.nbytes),
                        "d2h_bytes_per_step": int(d2h_bytes), "ms_per_step": e2e_ms / args.steps},
                "untangle_passes_per_s": 1e3 * args.steps / total_ms,
                "gpu_launches": int(launches), "roofline": roof, "clocks": clk,
                "ef_pairs": n_ef, "tests_per_pass": tests_per_pass, "node_tests_per_pass": nodes_per_pass,
                "cpu_baseline": cpu}
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    ctx.close()


if __name__ == "__main__":
    main()
