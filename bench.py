"""Benchmark of the untangling hot path on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload batch64]

A step is one untangling pass over one batch of synthetic input: face-tree refit, fused EF
broad+narrow phase, canonical EF order, edge-tree refit, PRP evaluation of every contour
(contours, runtime, adaptive k-ring levels of batched VF/EE/FV ray casting, cluster
culling, J, selection, suppression) and the response assembly.

Default workload: the batching form, 64 independent two-body scenes (icosphere-derived
shells or bumped cloth sheets, 2k-60k triangles each, 1.97 M triangles). The reference's
CPU path cannot run the whole batch K times within minutes, so both arms time the same
quarter of it: the 16 scenes s with s % 4 == 0 (a systematic sample, 0.49 M triangles).
This arm times K passes over those scenes as one batch; the reference arm evaluates the
same 16 scenes once, split over its K steps. The whole 64-scene batch, chosen and plain
form, is timed beside (`full_batch`).

value  = ray-primitive tests per second: the leaf primitive tests the pass executes (VF / FV
         ray-triangle and EE swept-edge tests of every primitive whose box the ray meets,
         the reference's BatchedRaycastStats::tested_leaf_primitive_count,
         cached_bvh.cpp:224, 451) over the pass time. Each arm counts its own executions:
         this arm's per-object LBVHs (one primitive per leaf, rays clipped to the task's
         candidate box) execute fewer tests for the same hits than the reference's
         median-split CachedBVH (8 primitives per leaf), so the tests/s ratio understates
         the pass speed-up; untangle_passes_per_s and pass_seconds give the time ratio.
e2e    = the same through the public API with host buffers: positions copied host->device
         and the per-contour results and supports device->host inside every timed step.
parity = the oracle's results on the timed scenes (cpu_baseline leg) compared with the
         GPU's timed pass, every per-contour field, direction and support hit; a mismatch
         ends the run with an error.
roofline = raycast_kernel (the dominant kernel, profiles/launch_list_*): the DRAM bytes
         its launches move (ncu, profiles/roofline_traffic.json, keyed by workload) over
         their CUDA-event time, and its issue rate (ncu warp instructions over the same
         time) against 4 warp instructions per SM cycle at the sampled clock.
cpu_baseline = the CPU oracle of the same 16 scenes on the host cores (all threads).

--profile-pass / --profile-refit run one pass / one face-tree refit of the workload between
cudaProfilerStart and cudaProfilerStop for `ncu --profile-from-start off` (profiles/ names the
commands); --raycast-config fixes the traversal configuration instead of the autotuner's choice.

--impl reference times the reference's algorithm on the host cores: the reference cannot
be built here (its LuisaCompute runtime is not in the checkout), so the CPU restatement
(the oracle) runs with all host threads over the same scenes.

Multi-GPU: the scenes are independent, so the timed scenes are split round robin across
ranks (no collective on the data path; strong scaling of a fixed workload); the job time
is the maximum over ranks.
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
RESPONSE = (3e-3, 1e8)  # untangling_response_depth, stiffness_untangling (scene_params.h:66, 121-122)
ALL_CONTOURS = 1 << 20
TIMED_STRIDE = 4        # batch workloads: the timed scenes are s % TIMED_STRIDE == 0


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _gpu_query_id(local):
    """nvidia-smi's id for this process's CUDA device: its UUID (nvidia-smi ignores
    CUDA_VISIBLE_DEVICES, so the CUDA ordinal may name another GPU)."""
    try:
        import torch
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if local < len(ids):
                return ids[local]
        return str(local)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
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
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "gpu": self.gpu_id}
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
                "reasons": sorted(reasons), "samples": len(sm), "gpu": self.gpu_id}


class Workload:
    """A bench workload: the full mesh, the scenes both arms time and the pass settings."""

    def __init__(self, name):
        from untangling26_b200 import synthetic
        self.name = name
        self.batch = name.startswith("batch")
        self.repair = False
        self.repair_scale = 1.0
        self.params = dict(max_contours=ALL_CONTOURS, batch_size=ALL_CONTOURS)
        # single-mesh workloads: the contours the CPU legs evaluate (None: every 8th)
        self.oracle_contours = None
        if name == "batch64":
            self.full = synthetic.batch_scenes(64, seed=2)
            self.timed_ids = list(range(0, 64, TIMED_STRIDE))
            self.config = {"workload": "batch_64_two_body_scenes", "seed": 2, "scenes": 64, "triangles": int(len(self.full.faces)),
                           "tris_per_scene": "U[2000, 60000]", "bodies": "icosphere-derived shells or bumped sheets",
                           "timed_scenes": f"s % {TIMED_STRIDE} == 0 (16 of 64)", "directions": "reference seeds (<=10)",
                           "opt_iterations": 0, "contours": "all"}
        elif name == "batch8":  # a small batch for tests of the bench itself
            self.full = synthetic.batch_scenes(8, seed=5, tris_lo=2000, tris_hi=4000)
            self.timed_ids = list(range(0, 8, 2))
            self.config = {"workload": "batch_8_small_scenes", "seed": 5, "scenes": 8, "triangles": int(len(self.full.faces)),
                           "timed_scenes": "s % 2 == 0 (4 of 8)", "directions": "reference seeds (<=10)", "opt_iterations": 0,
                           "contours": "all"}
        elif name == "folded256":
            # the precision form's scene: 26 candidate directions, up to 8 S^2 steps
            self.full = synthetic.folded_sheet(256, seed=1)
            self.timed_ids = None
            self.params = dict(max_contours=256, batch_size=32, direction_mode=1, opt_iterations=8)
            self.config = {"workload": "folded_sheet_256x256", "seed": 1, "triangles": 130050, "fold_noise_sigma_edge_lengths": 0.3,
                           "directions": "26 lattice", "opt_iterations": 8, "contours": "first 256"}
        elif name == "folded128":  # a small case of the folded sheet (profiling)
            self.full = synthetic.folded_sheet(128, seed=1)
            self.timed_ids = None
            self.params = dict(max_contours=256, batch_size=32)
            self.config = {"workload": "folded_sheet_128x128", "seed": 1, "triangles": int(self.full.num_faces),
                           "directions": "reference seeds (<=10)", "opt_iterations": 0, "contours": "first 256"}
        elif name == "two_sheets64":
            self.full = synthetic.two_sheets(64, seed=0)
            self.timed_ids = None
            self.params = dict(max_contours=256, batch_size=32)
            self.config = {"workload": "two_sheets_64x64", "seed": 0, "triangles": 15876, "directions": "reference seeds (<=10)",
                           "opt_iterations": 0, "contours": "first 256"}
        elif name == "layered5x512":
            # the scale form: five stacked 512 x 512 sheets 1 mm apart with multi-octave
            # displacement of 2-20 mm; every step is one untangling pass followed by a fixed step
            # along its assembled response (the repair loop), so the K steps are K passes of it
            self.full = synthetic.layered_sheets(512, layers=5, seed=4)
            self.timed_ids = None
            # one batch of 32 contours per pass: the 199 contours of the first pass grow to whole
            # sheets (4.9 G requests, 75 s per pass); the traversal configuration is the batch
            # workload's tuned one (tuning here would run 18 full ray-casting passes)
            self.params = dict(max_contours=32, batch_size=32, autotune=0, raycast_config=2)
            self.repair = True
            # the fixed step: a quarter of the assembled response, so that no vertex moves more
            # than 0.375 mm (a pair asks for up to the 3 mm response depth, half per side) between
            # sheets 1 mm apart
            self.repair_scale = 0.25
            # the oracle needs 3-30 s for most contours of this mesh and minutes for the largest
            # regions (contour 0): the CPU legs evaluate contours 1, 3 and 5
            self.oracle_contours = (1, 3, 5)
            self.config = {"workload": "layered_sheets_5x512x512", "seed": 4, "layers": 5, "triangles": int(self.full.num_faces),
                           "spacing_mm": 1, "displacement_mm": "U[2, 20] multi-octave", "directions": "reference seeds (<=10)",
                           "opt_iterations": 0, "contours": "first 32 of each pass (one batch)", "update": "response step, scale 0.25",
                           "raycast_config": "fixed 4x7"}
        else:
            raise SystemExit(f"unknown workload {name}")
        self.config["l2"] = "flushed between steps (256 MB write)"

    def timed_scene_ids(self, rank=0, world=1):
        from untangling26_b200.multirank import scene_shard
        return [self.timed_ids[i] for i in scene_shard(len(self.timed_ids), rank, world)]

    def timed_mesh(self, rank=0, world=1):
        from untangling26_b200 import synthetic
        if not self.batch:
            return self.full
        return synthetic.sub_batch(self.full, self.timed_scene_ids(rank, world))

    def scene_meshes(self, ids):
        from untangling26_b200 import synthetic
        return [synthetic.scene_mesh(self.full, s) for s in ids]


def _dist_env():
    from untangling26_b200.multirank import dist_env
    return dist_env()


# ---------------------------------------------------------------- CPU (oracle) legs
def oracle_pass(mesh, params, stride=1, offset=0):
    """The pass with the CPU oracle: LBVH + EF detection + PRP (+ response). Returns
    (PrpRun, executed leaf tests, seconds)."""
    from oracle import oracle as o
    t0 = time.perf_counter()
    dh = np.full(mesh.num_verts, 1e-3, np.float32)
    th = np.zeros(mesh.num_verts, np.float32)
    tree = o.lbvh_build(o.TREE_FACE, mesh.x, mesh.faces)
    o.lbvh_refit(tree, mesh.x, mesh.x, th, mesh.faces)
    broad, _, _ = o.lbvh_query(tree, o.QUERY_EDGES_UNCULLED, mesh.x, mesh.x, mesh.edges, dh, th)
    ef, idx = o.ef_narrow(broad, mesh.x, mesh.edges, mesh.faces, dh, mesh.vert_property)
    run = o.PrpRun(mesh, ef, idx, o.prp_params(contour_stride=stride, contour_offset=offset, **params), response=RESPONSE)
    return run, run.tested, time.perf_counter() - t0


def reference_arm(args, wl):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return
    from oracle import oracle as o
    o.build()
    if wl.batch:
        scenes = wl.scene_meshes(wl.timed_ids)
        chunks = np.array_split(np.arange(len(scenes)), max(args.steps, 1))
        step = lambda i: [oracle_pass(scenes[j], wl.params)[1:] for j in chunks[i]]
        smallest = min(range(len(scenes)), key=lambda j: scenes[j].num_faces)
        warm = lambda: oracle_pass(scenes[smallest], wl.params)
        sample = (f"the {len(scenes)} timed scenes ({wl.config['timed_scenes']}), each a full pass (EF detection, every "
                  f"contour, response), split over the {args.steps} steps: one pass over the timed workload")
    elif wl.oracle_contours:
        cs = wl.oracle_contours
        step = lambda i: [oracle_pass(wl.full, wl.params, stride=1 << 20, offset=cs[i % len(cs)])[1:]]
        warm = lambda: None
        sample = f"EF detection and one of the contours {list(cs)} each step (step i: contour {list(cs)}[i % {len(cs)}])"
    else:
        stride = max(args.steps, 1)
        step = lambda i: [oracle_pass(wl.full, wl.params, stride=stride, offset=i)[1:]]
        warm = lambda: None
        sample = (f"EF detection every step; the contours c with c % {stride} == step index, so the {args.steps} steps "
                  "evaluate each contour once")
    for _ in range(max(args.warmup, 0)):
        warm()
    tests, sec = 0, 0.0
    for i in range(args.steps):
        for t, s in step(i):
            tests += t
            sec += s
    value = tests / sec if sec > 0 else 0.0
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec / max(args.steps, 1), "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "impl": "reference", "config": wl.config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": o.threads(), "kind": "port",
                         "sample": sample + " (the reference's algorithm restated on the CPU; its LuisaCompute build is absent)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "untangle_passes_per_s": 1.0 / sec if sec > 0 else 0.0, "pass_seconds": sec, "leaf_tests_per_pass": tests}))


def cpu_baseline_and_parity(wl, res, tmesh):
    """The oracle over the timed scenes (rank 0, one rank): its throughput, and the GPU's
    last timed pass compared with it."""
    from oracle import oracle as o
    from oracle.compare import compare_contours, compare_scene
    o.build()
    tests, sec, ncont, nhits = 0, 0.0, 0, 0
    if wl.batch:
        ids = [s["batch_scene"] for s in tmesh.meta["scenes"]]
        for j, m in enumerate(wl.scene_meshes(ids)):
            run, t, s = oracle_pass(m, wl.params)
            tests += t
            sec += s
            c, h = compare_scene(res, tmesh, j, run)
            ncont += c
            nhits += h
        sample = f"the {len(ids)} timed scenes, one full pass each (every contour, response)"
    elif wl.oracle_contours:
        for c in wl.oracle_contours:
            run, t, s = oracle_pass(wl.full, wl.params, stride=1 << 20, offset=c)
            tests += t
            sec += s
            nhits += compare_contours(res, run, [c])
            ncont += 1
        sample = f"EF detection and one contour, for each of the contours {list(wl.oracle_contours)} of the timed pass"
    else:
        stride = 8
        run, t, s = oracle_pass(wl.full, wl.params, stride=stride)
        tests, sec = t, s
        cs = [c for c in range(min(len(run.contours), wl.params["max_contours"])) if c % stride == 0]
        nhits = compare_contours(res, run, cs)
        ncont = len(cs)
        sample = f"EF detection and the contours c % {stride} == 0 of the timed pass"
    cpu = {"value": tests / sec, "unit": UNIT, "cores": o.threads(), "kind": "port", "sample": f"{sample}, {sec:.1f} s",
           "pass_seconds": sec if wl.batch else None}
    parity = {"ok": True, "contours_compared": ncont, "hits_compared": nhits,
              "fields": "every per-contour result field, candidate directions, support hits (bytes)",
              "against": "oracle (CPU restatement of the reference)",
              # executed leaf tests of the same work: the oracle's CachedBVH (8 primitives per leaf,
              # rays from the object root) and this pass's per-object LBVHs
              "oracle_leaf_tests": int(tests)}
    if not wl.batch and wl.oracle_contours is None:
        parity["oracle_leaf_tests_note"] = "EF detection and the sampled contours only"
    return cpu, parity


# ---------------------------------------------------------------- GPU arm
class PassRunner:
    """One CollisionScene and the pass of the bench over it."""

    def __init__(self, ctx, mesh, params):
        from untangling26_b200.intersection_resolver import CollisionScene
        from untangling26_b200.prp import prp_params, response_params
        self.mesh = mesh
        self.sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0, max_ef_pairs=max(1 << 16, mesh.num_edges))
        self.sc.construct_lbvh()
        # the chosen form: FP64 recheck of the in-band predicates, traversal configuration
        # autotuned on the scene's first (warm-up) pass
        self.params = prp_params(**dict(dict(fp64_recheck=1, autotune=1), **params))
        self.rparams = response_params(*RESPONSE)

    def run(self, with_stats=True):
        sc = self.sc
        sc.refit_face_tree()
        sc.resolver.reset()
        if with_stats:
            sc.stats.zero_()
        sc.ef_detect(with_stats=with_stats)
        n = sc.resolver.canonicalize(self.mesh.num_edges, self.mesh.num_faces)
        return sc.host_resolve(self.params, num_pairs=n, response=self.rparams)

    def close(self):
        self.sc.close()


def _timed_passes(runner, steps, flush, stream, repair=False, scale=1.0):
    """K timed passes; with repair, each pass is followed (inside its timed step) by the fixed
    step along its assembled response, so the passes form the repair sequence."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    out = []
    for i in range(steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record(stream)
        res = runner.run()
        if repair:
            runner.sc.response_step(res.response, scale)
        out.append(res)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev], out


def refit_rate(sc, mesh, flush, stream, peak, n=10):
    """Median time of the fused leaf update + refit of the scene's face tree over n launches
    (L2 flushed before each). Algorithmic bytes, each once (the refit's byte count with
    positions read once, x_start = x_end): V x (12 B position + 4 B thickness) + F x (12 B face
    + 4 B leaf order + 32 B leaf box written) + (F - 1) x (8 B children + 4 B parent + 64 B
    child boxes read + 32 B box written)."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n + 2)]
    for i, (a, b) in enumerate(ev):
        flush.fill_((i + 7) & 0xFF)
        a.record(stream)
        sc.refit_face_tree()
        b.record(stream)
    torch.cuda.synchronize()
    ms = statistics.median(a.elapsed_time(b) for a, b in ev[2:])
    byts = 16 * mesh.num_verts + 48 * mesh.num_faces + 108 * max(mesh.num_faces - 1, 0)
    out = {"kernel": "refit_chunk_kernel + refit_top_kernel", "triangles": int(mesh.num_faces), "ms": ms, "algorithmic_bytes": byts,
           "achieved": byts / (ms / 1e3) / 1e9, "unit": "GB/s", "peak": peak}
    out["frac"] = out["achieved"] / peak
    return out


def _traffic(kernel, workload):
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(prof):
        return None
    with open(prof) as f:
        return json.load(f).get(kernel, {}).get(workload)


def profile_pass(args, wl):
    """The pass an ncu capture measures: the bench's warm-up passes (the autotuner runs in the
    first unless --raycast-config fixes the configuration), then one pass of the timed workload
    between cudaProfilerStart and cudaProfilerStop."""
    import torch
    from untangling26_b200 import Context
    ctx = Context(0)
    runner = PassRunner(ctx, wl.timed_mesh(), wl.params)
    for _ in range(max(args.warmup, 1)):
        runner.run()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    res = runner.run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_pass": args.workload, "leaf_tests": res.tested, "requests": res.requests, "contours": len(res.contours),
                      "raycast_config": {k: res.raycast_config[k] for k in ("parts", "blocks_per_sm", "queue")},
                      "gpu_ms": {k: round(v, 3) for k, v in res.gpu_ms.items()}}))
    runner.close()
    ctx.close()


def profile_refit(args, wl):
    """The refit an ncu capture measures: --warmup refits of the workload's timed mesh's face
    tree, then one between cudaProfilerStart and cudaProfilerStop."""
    import torch
    from untangling26_b200 import Context
    from untangling26_b200.intersection_resolver import CollisionScene
    ctx = Context(0)
    mesh = wl.timed_mesh()
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0, max_broad_pairs=1, max_ef_pairs=1)
    sc.construct_lbvh()
    for _ in range(max(args.warmup, 1)):
        sc.refit_face_tree()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    sc.refit_face_tree()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_refit": args.workload, "triangles": int(mesh.num_faces)}))
    sc.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batch64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-batch", action="store_true", help="skip the whole-batch chosen / plain timing")
    ap.add_argument("--raycast-config", default=None,
                    help="a fixed traversal configuration ('4x7', '8x7q', ...) instead of the autotuner's choice")
    ap.add_argument("--profile-pass", action="store_true",
                    help="for ncu (--profile-from-start off): warm-up passes, then one pass of the timed workload "
                         "inside cudaProfilerStart / Stop; prints one line and exits")
    ap.add_argument("--profile-refit", action="store_true",
                    help="for ncu (--profile-from-start off): the face-tree refit (fused leaf update) of the timed mesh, "
                         "--warmup refits, then one inside cudaProfilerStart / Stop; prints one line and exits")
    args = ap.parse_args()
    ws, rank, local = _dist_env()
    wl = Workload(args.workload)
    if args.raycast_config:
        from untangling26_b200.prp import RAYCAST_CONFIGS, config_name
        names = [config_name(c) for c in RAYCAST_CONFIGS]
        if args.raycast_config not in names:
            raise SystemExit(f"--raycast-config must be one of {names}")
        wl.params = dict(wl.params, autotune=0, raycast_config=names.index(args.raycast_config) + 1)
        wl.config["raycast_config"] = f"fixed {args.raycast_config}"
    if args.impl == "reference":
        return reference_arm(args, wl)
    if args.profile_pass:
        return profile_pass(args, wl)
    if args.profile_refit:
        return profile_refit(args, wl)

    import torch
    import torch.distributed as dist

    from untangling26_b200 import Context
    from untangling26_b200.multirank import job_time_ms

    if ws > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = Context(local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    peak, peak_kind = _peaks()

    tmesh = wl.timed_mesh(rank, ws)
    runner = PassRunner(ctx, tmesh, wl.params)
    tuned = None
    for _ in range(max(args.warmup, 3)):
        r = runner.run()
        if r.raycast_config.get("tuned_this_pass"):
            tuned = r.raycast_config
    torch.cuda.synchronize()

    # ---- device-resident timed region: K passes over the timed scenes
    launches0 = ctx.launch_count()
    clocks = ClockSampler(_gpu_query_id(local))
    clocks.start()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms, results = _timed_passes(runner, args.steps, flush, stream, repair=wl.repair, scale=wl.repair_scale)
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    # the pass compared with the oracle: the last one, or with repair the first (the input's positions)
    r0 = results[0] if wl.repair else results[-1]
    ef_rc = (int(runner.sc.stats[2].item()), int(runner.sc.stats[3].item()))
    tests_pass = sum(r.tested for r in results) / len(results)
    for r in results:
        if r.device_error_flags:
            raise SystemExit(f"device error flags 0x{r.device_error_flags:x}")
        # every timed pass returns the same results (the leaf-test count may differ by a few between
        # passes: see the packet walk's node tests)
        if not wl.repair and (r.results.tobytes() != r0.results.tobytes() or any(a.tobytes() != b.tobytes() for a, b in zip(r.hits, r0.hits))):
            raise SystemExit("timed passes returned different results")
    repair = None
    if wl.repair:
        repair = {"ef_pairs_per_pass": [int(r.num_orig_pairs) for r in results], "contours_per_pass": [len(r.contours) for r in results],
                  "response_pairs_per_pass": [int(r.response.num_pairs) for r in results], "pass_ms": [round(t, 2) for t in step_ms],
                  "passes_per_s": 1e3 * len(step_ms) / sum(step_ms)}
    total_ms = job_time_ms(sum(step_ms), device=dev)  # max over ranks
    tests_all = tests_pass
    if ws > 1:
        t = torch.tensor([float(tests_pass)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        tests_all = int(t.item())
    value = tests_all * args.steps / (total_ms / 1e3)
    pass_ms = total_ms / args.steps

    # ---- e2e through the public API with host buffers (positions in, results out)
    x_host = torch.from_numpy(tmesh.x).pin_memory()
    e_ms, d2h, e_tests = [], 0, 0
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        runner.sc.x.copy_(x_host, non_blocking=True)
        res = runner.run()  # the per-contour results and supports come back to the host inside u26_prp_resolve
        torch.cuda.synchronize()
        e_ms.append(1e3 * (time.perf_counter() - t0))
        e_tests += res.tested
        d2h = int(sum(h.nbytes for h in res.hits) + res.results.nbytes + res.pairs.nbytes)
    e2e_ms = job_time_ms(sum(e_ms), device=dev)
    if ws > 1:
        t = torch.tensor([float(e_tests)], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        e_tests = t.item()
    e2e_value = e_tests / (e2e_ms / 1e3)

    # ---- roofline of the dominant kernel: raycast_kernel. Its CUDA-event time per pass is
    # measured here; the DRAM bytes and warp instructions per pass come from one ncu capture
    # of the same workload (profiles/roofline_traffic.json).
    rc_ms = r0.gpu_ms["raycast"]
    tr = _traffic("raycast_kernel", args.workload)
    roof = {"bound": "hbm", "kernel": "raycast_kernel", "peak": peak, "unit": "GB/s", "peak_source": peak_kind,
            "limiter": "instruction issue (see issue.frac): the tree and mesh are served from L1 / L2",
            "kernel_ms_per_pass": rc_ms, "traffic": None, "achieved": None, "frac": None}
    if tr:
        roof["traffic"] = tr["dram_bytes"]
        roof["achieved"] = tr["dram_bytes"] / (rc_ms / 1e3) / 1e9
        roof["frac"] = roof["achieved"] / peak
        mhz = clk.get("sm_mhz") or 1965.0
        issue_peak = 148 * 4 * mhz * 1e6
        roof["issue"] = {"warp_inst_per_pass": tr["warp_inst"], "achieved": tr["warp_inst"] / (rc_ms / 1e3), "peak": issue_peak,
                         "unit": "warp inst/s", "frac": tr["warp_inst"] / (rc_ms / 1e3) / issue_peak,
                         "peak_basis": f"148 SMs x 4 schedulers x {mhz:.0f} MHz (sampled median)"}
        roof["traffic_source"] = tr.get("source")
        # the capture's traversal configuration against this run's (the DRAM bytes and
        # instructions of a pass depend a little on it)
        from untangling26_b200.prp import config_name
        mine = config_name((r0.raycast_config["parts"], r0.raycast_config["blocks_per_sm"], r0.raycast_config["queue"]))
        roof["traffic_config"] = {"captured": tr.get("raycast_config"), "this_run": mine, "same": tr.get("raycast_config") == mine}
    roof["packet_record_bytes_per_pass"] = 32 * r0.node_fetches + 48 * r0.tri_fetches + 32 * r0.edge_fetches + 24 * r0.requests

    # ---- LBVH refit alone (fused leaf update + bottom-up refit of a face tree), L2 flushed
    # before each launch: the timed batch's scene tree and the scale form's mesh (five stacked
    # 512 x 512 sheets, 2.6 M triangles), where the refit is long enough to be bandwidth-bound
    refit = {"timed_batch": refit_rate(runner.sc, tmesh, flush, stream, peak)}
    if ws == 1:
        from untangling26_b200 import synthetic
        from untangling26_b200.intersection_resolver import CollisionScene
        lm = synthetic.layered_sheets(512, layers=5, seed=4)
        lsc = CollisionScene(ctx, lm, d_hat=1e-3, thickness=0.0, max_broad_pairs=1, max_ef_pairs=1)
        lsc.construct_lbvh()
        refit["layered_5x512"] = refit_rate(lsc, lm, flush, stream, peak)
        lsc.close()
    runner.close()

    # ---- the whole batch: chosen form and the plain form (per-scene passes, one thread per
    # request from the tree root, per-contour launches), same results
    full = None
    if wl.batch and not args.no_full_batch and ws == 1:
        fr = PassRunner(ctx, wl.full, wl.params)
        for _ in range(2):
            fr.run()
        torch.cuda.synchronize()
        f_ms, f_res = _timed_passes(fr, 3, flush, stream)
        fr.close()
        f_tests = f_res[-1].tested
        fpass = statistics.median(f_ms)
        plain_params = dict(wl.params, form=1)
        prs = [PassRunner(ctx, m, plain_params) for m in wl.scene_meshes(range(wl.full.meta["num"]))]
        for p in prs:
            p.run()
        torch.cuda.synchronize()
        pev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        flush.fill_(1)
        pev[0].record(stream)
        p_res = [p.run() for p in prs]
        pev[1].record(stream)
        torch.cuda.synchronize()
        p_ms = pev[0].elapsed_time(pev[1])
        p_tests = sum(r.tested for r in p_res)
        for p in prs:
            p.close()
        full_passes = (f_res[-1], p_res)  # compared in the checking leg below
        full = {"scenes": wl.full.meta["num"], "triangles": int(wl.full.num_faces), "pass_ms": fpass, "leaf_tests": f_tests,
                "value": f_tests / (fpass / 1e3), "untangle_passes_per_s": 1e3 / fpass,
                "plain_pass_ms": p_ms, "plain_leaf_tests": p_tests, "chosen_over_plain": p_ms / fpass}

    cpu, parity = None, None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu, parity = cpu_baseline_and_parity(wl, r0, tmesh)
            if full is not None:
                # same results: each scene's plain pass against its part of the batched chosen pass
                from oracle.compare import compare_scene
                same = [compare_scene(full_passes[0], wl.full, j, r) for j, r in enumerate(full_passes[1])]
                full["same_results"] = {"contours": sum(c for c, _ in same), "hits": sum(h for _, h in same)}
        except AssertionError as e:
            print(json.dumps({"parity_failure": str(e)}), file=sys.stderr)
            raise SystemExit(f"parity check failed: {e}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": pass_ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": wl.config,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(tmesh.x.nbytes), "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": int(launches), "clocks": clk, "roofline": roof, "cpu_baseline": cpu, "lbvh_refit": refit,
            "leaf_tests_per_step": [int(r.tested) for r in results],
            "pass": {"scenes": len(tmesh.meta.get("scenes", [0])), "triangles": int(tmesh.num_faces), "ef_pairs": int(len(r0.pairs)),
                     "contours": len(r0.contours), "levels": r0.levels, "requests": r0.requests, "leaf_tests": r0.tested,
                     "candidate_leaf_tests": r0.candidate_tests, "ray_node_visits": r0.ray_visits,
                     "request_candidate_pairs": r0.pairs_tested, "response_pairs": r0.response.num_pairs,
                     "response_ms": round(r0.response.ms, 2),
                     "gpu_ms": {k: round(v, 2) for k, v in r0.gpu_ms.items()},
                     "stage_ms": {k: round(v, 2) for k, v in r0.stage_ms.items()}},
            "parity": parity,
            "repair": repair,
            "fp64": dict(r0.fp64, ef_rechecks=ef_rc[0], ef_flips=ef_rc[1],
                         note="rechecks / flips: leaf tests of the timed pass inside their FP32 error band, re-decided in FP64 "
                              "(sets keep FP32); *_rel_err: the selected supports' FP32 depth, D_C and J against FP64"),
            "raycast_config": {"parts": r0.raycast_config["parts"], "blocks_per_sm": r0.raycast_config["blocks_per_sm"],
                               "queue": r0.raycast_config["queue"],
                               "autotune_ms": tuned.get("tune_ms") if tuned else None,
                               "note": "chosen by the autotuner on the first warm-up pass: ray-casting ms of each parts x blocks/SM "
                                       "(q: persistent work-queue grid)"},
            "untangle_passes_per_s": 1e3 / pass_ms, "pass_seconds": pass_ms / 1e3,
            "speedup_vs_cpu_pass": (cpu["pass_seconds"] / (pass_ms / 1e3)) if cpu and cpu.get("pass_seconds") else None,
            "full_batch": full,
            "plain_form": {"chosen_over_plain": full["chosen_over_plain"], "plain_pass_ms": full["plain_pass_ms"],
                           "chosen_pass_ms": full["pass_ms"], "same_results": full.get("same_results")} if full else None,
        }
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    ctx.close()


if __name__ == "__main__":
    main()
