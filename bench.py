"""Benchmark of the untangling hot path on B200 (one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload folded256]

A step is one untangling pass over one batch of synthetic input. Default workload: the
precision-form cloth scene, one 256 x 256-vertex sheet (130,050 triangles) folded once
about a seeded line with 0.3 x edge-length Gaussian vertex noise. The pass: face-tree
refit, fused EF broad+narrow phase, canonical EF order, edge-tree refit, PRP contour
evaluation of the first 256 contours (contours, runtime, adaptive k-ring levels of
batched VF/EE/FV ray casting, cluster culling, J, selection, suppression).

value  = ray-primitive tests per second of the whole job. Tests of a pass = the EF
         segment-triangle tests (edge-face pairs whose AABBs overlap) + the ray-primitive
         pairs of the PRP stage, i.e. every (VF/EE/FV request, candidate target primitive)
         pair the pass decides, whether by a primitive test or by BVH culling. This count
         is fixed by the algorithm and the inputs, so the CPU oracle and the GPU report the
         same number for the same pass; executed leaf tests are reported beside it. Time:
         CUDA events around the pass (host orchestration included), inputs resident in HBM.
e2e    = the same metric through the public API with host buffers: positions copied
         host->device and the selected responses device->host inside every timed step.
roofline = the dominant kernel (per the ncu launch list in profiles/): achieved
         algorithmic bytes / its CUDA-event time vs the measured HBM copy bandwidth.
cpu_baseline = the CPU oracle of the same pass on the host cores, bounded sample.

--impl reference times the reference's algorithm on the host cores: the reference cannot
be built here (its LuisaCompute runtime is not in the checkout), so the CPU restatement
(the oracle) runs with all host threads on a bounded sample of the same workload.

Multi-GPU: the path shards by independent scenes (weak scaling, no collective). With
--gpus N under torchrun every rank runs its own scene replica; value = total tests of all
ranks / max rank time.
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
# CPU samples evaluate every STRIDE-th contour of the first max_contours (the contour mix of
# the full pass: small loops, boundary-ending contours and the large ones that grow to many
# k-ring levels), with the full EF detection in front.
CPU_BASELINE_STRIDE = 4   # cpu_baseline: one sample, 64 of 256 contours
CPU_REFERENCE_STRIDE = 8  # --impl reference: every step, 32 of 256 contours


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
    if name == "folded128":
        return synthetic.folded_sheet(128, seed=1), {"workload": "folded_sheet_128x128", "triangles": 32258, "seed": 1}
    if name == "two_sheets64":
        return synthetic.two_sheets(64, seed=0), {"workload": "two_sheets_64x64", "triangles": 15876, "seed": 0}
    if name == "layered5x512":
        m = synthetic.layered_sheets(512, layers=5, seed=4)
        return m, {"workload": "layered_sheets_5x512x512", "triangles": int(len(m.faces)), "layers": 5, "seed": 4,
                   "spacing_mm": 1, "displacement_mm": "U[2, 20] multi-octave"}
    if name == "batch64":
        m = synthetic.batch_scenes(64, seed=2)
        return m, {"workload": "batch_64_two_body_scenes", "triangles": int(len(m.faces)), "scenes": 64, "seed": 2,
                   "tris_per_scene": "U[2000, 60000]", "bodies": "icosphere-derived shells or bumped sheets"}
    raise SystemExit(f"unknown workload {name}")


def _dist_env():
    from untangling26_b200.multirank import dist_env
    return dist_env()


def cpu_pass(mesh, max_contours, stride):
    """The same pass with the CPU oracle: LBVH + EF detection + PRP of the contours c <
    max_contours with c % stride == 0. Returns (ray-prim tests, seconds)."""
    from oracle import oracle as o
    t0 = time.perf_counter()
    dh = np.full(mesh.num_verts, 1e-3, np.float32)
    th = np.zeros(mesh.num_verts, np.float32)
    tree = o.lbvh_build(o.TREE_FACE, mesh.x, mesh.faces)
    o.lbvh_refit(tree, mesh.x, mesh.x, th, mesh.faces)
    broad, n_broad, _ = o.lbvh_query(tree, o.QUERY_EDGES_UNCULLED, mesh.x, mesh.x, mesh.edges, dh, th)
    ef, idx = o.ef_narrow(broad, mesh.x, mesh.edges, mesh.faces, dh, mesh.vert_property)
    run = o.PrpRun(mesh, ef, idx, o.prp_params(max_contours=max_contours, contour_stride=stride), response=RESPONSE)
    return n_broad + run.pairs_tested, time.perf_counter() - t0


CPU_BATCH_SCENES = 8  # scenes of the batch workload in the CPU sample
RESPONSE = (3e-3, 1e8)  # untangling_response_depth, stiffness_untangling (scene_params.h:66, 121-122)


def run_cpu_baseline(mesh, max_contours, samples=1):
    from oracle import oracle as o
    o.build()
    tests, sec = 0, 0.0
    if mesh.meta.get("kind") == "batch_scenes":
        from untangling26_b200 import synthetic
        for s_i in range(CPU_BATCH_SCENES):
            t, s = cpu_pass(synthetic.scene_mesh(mesh, s_i), max_contours, 1)
            tests += t
            sec += s
        return {"value": tests / sec, "unit": UNIT, "cores": o.threads(), "kind": "port",
                "sample": f"the full pass of the first {CPU_BATCH_SCENES} of {mesh.meta['num']} scenes, {sec:.1f} s"}
    for _ in range(samples):
        t, s = cpu_pass(mesh, max_contours, CPU_BASELINE_STRIDE)
        tests += t
        sec += s
    return {"value": tests / sec, "unit": UNIT, "cores": o.threads(), "kind": "port",
            "sample": f"{samples} pass(es) of the workload: full EF detection, then PRP of every "
                      f"{CPU_BASELINE_STRIDE}th of the first {max_contours} contours, {sec:.1f} s"}


def reference_arm(args, mesh, config):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return
    from oracle import oracle as o
    o.build()
    if mesh.meta.get("kind") == "batch_scenes":
        # each step: the full pass of two scenes of the batch, in turn
        from untangling26_b200 import synthetic
        scenes = [synthetic.scene_mesh(mesh, s_i) for s_i in range(mesh.meta["num"])]
        step = lambda i: [cpu_pass(scenes[(2 * i + k) % len(scenes)], args.max_contours, 1) for k in range(2)]
        sample = "each step the full pass of two scenes of the batch"
    else:
        step = lambda i: [cpu_pass(mesh, args.max_contours, CPU_REFERENCE_STRIDE)]
        sample = (f"each step the full EF detection + PRP of every {CPU_REFERENCE_STRIDE}th "
                  f"of the first {args.max_contours} contours")
    for i in range(max(args.warmup, 0)):
        step(i)
    tests, sec = 0, 0.0
    for i in range(args.steps):
        for t, s in step(i):
            tests += t
            sec += s
    value = tests / sec
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": dict(config, parallelism="host threads", l2="n/a (CPU)", max_contours=args.max_contours,
                       directions="reference seeds (<=10 per contour)"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": o.threads(), "kind": "port",
                         "sample": f"{args.steps} steps, {sample} "
                                   "(the reference's algorithm restated on the CPU; its LuisaCompute build is absent)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def _pair_filter_block(sc, mesh, dev, flush, stream, response, num_ef, peak, steps=5):
    import torch
    nv = mesh.num_verts
    dh = torch.full((nv,), 1e-3, dtype=torch.float32, device=dev)
    cap = 32 * nv
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    vfl = torch.zeros((cap, 2), dtype=torch.int32, device=dev)
    sc.face_tree.broad_phase_query_from_verts(sc.x, sc.x, cnt, vfl, dh, sc.thickness)
    nvf = min(int(cnt.item()), cap)
    cnt.zero_()
    eel = torch.zeros((cap, 2), dtype=torch.int32, device=dev)
    sc.edge_tree.broad_phase_query_from_edges(sc.x, sc.x, sc.edges, cnt, eel, dh, sc.thickness)
    nee = min(int(cnt.item()), cap)
    vf, ee = vfl[:nvf], eel[:nee]
    # proximity pairs between primitives that share no vertex
    fv = sc.faces[vf[:, 1].long()]
    vf = vf[(fv != vf[:, :1]).all(1)].contiguous()
    ea, eb = sc.edges[ee[:, 0].long()], sc.edges[ee[:, 1].long()]
    ee = ee[((ea[:, :1] != eb) & (ea[:, 1:] != eb)).all(1)].contiguous()
    nvf, nee = int(vf.shape[0]), int(ee.shape[0])
    bit = torch.tensor(-2 ** 31, dtype=torch.int32, device=dev)
    fv = sc.faces[vf[:, 1].long()]
    ea, eb = sc.edges[ee[:, 0].long()], sc.edges[ee[:, 1].long()]
    idx = torch.cat([torch.stack([vf[:, 0], fv[:, 0], fv[:, 1] | bit, fv[:, 2]], 1),
                     torch.stack([ea[:, 0], ea[:, 1], eb[:, 0], eb[:, 1] | bit], 1)])
    n = nvf + nee
    vec = torch.zeros((n, 12), dtype=torch.float32, device=dev)
    vec[:, 2] = 1.0
    vec[:, 4], vec[:, 5] = -1e3, 1e5
    vec[:nvf, 6], vec[:nvf, 7] = 1.0 / 3.0, 1.0 / 3.0
    vec[nvf:, 6], vec[nvf:, 7] = 0.5, 0.5
    pairs0 = torch.cat([idx, vec.view(torch.int32)], 1).contiguous()
    pidx = torch.cat([vf, ee]).contiguous()
    offset = torch.full((nv,), 2.5e-4, dtype=torch.float32, device=dev)
    vf0, ee0 = vf.clone(), ee.clone()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    pairs = torch.empty_like(pairs0)
    inv = torch.zeros(nv, dtype=torch.int32, device=dev)
    for i in range(steps + 1):
        pairs.copy_(pairs0)
        vf.copy_(vf0)
        ee.copy_(ee0)
        inv.zero_()
        flush.fill_((i + 3) & 0xFF)
        if i:
            evs[i - 1][0].record(stream)
        sc.filter_invalid_pairs(pairs, pidx, n, offset, inv, response=response, num_ef=num_ef)
        sc.filter_broad_phase_pairs(vf, nvf, ee, nee, inv, response, num_ef=num_ef)
        if i:
            evs[i - 1][1].record(stream)
    torch.cuda.synchronize()
    ms = statistics.median(a.elapsed_time(b) for a, b in evs)
    byts = n * (64 + 48 + 8) + n * (64 + 8 + 16 + 16) + nvf * (8 + 12 + 16 + 16 + 8) + nee * (8 + 16 + 16 + 16 + 8)
    disabled = int((pairs[:, 9].view(torch.float32) == 0).sum().item())  # k2 (vec2[1])
    flagged = int(((vf[:, 0] >> 30) != 0).sum().item() + ((ee[:, 0] >> 30) != 0).sum().item())
    out = {"kernels": ["identify_invalid_kernel", "filter_pairs_kernel", "filter_broad_vf_kernel", "filter_broad_ee_kernel"],
           "proximity_pairs": n, "broad_vf": nvf, "broad_ee": nee, "disabled": disabled, "flagged_broad": flagged,
           "invalid_verts": int(inv.sum().item()), "ms": ms, "algorithmic_bytes": byts,
           "achieved": byts / (ms / 1e3) / 1e9, "unit": "GB/s", "peak": peak,
           "note": "proximity / CCD pairs within 1 mm (box overlap, no shared vertex) from the scene trees, "
                   "offsets 0.25 mm; median of 5, L2 flushed"}
    out["frac"] = out["achieved"] / peak
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="folded256")
    ap.add_argument("--max-contours", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=1, help="timed passes of the plain form (0: skip)")
    args = ap.parse_args()
    ws, rank, local = _dist_env()
    mesh, config = make_workload(args.workload)
    batch = args.workload.startswith("batch")
    if batch:
        # every contour of every scene, one merge batch (contour indices shift between the
        # batched and the per-scene runs; the results stay the same)
        args.max_contours = 1 << 20
    if args.impl == "reference":
        return reference_arm(args, mesh, config)

    import torch
    import torch.distributed as dist

    from untangling26_b200 import Context
    from untangling26_b200.intersection_resolver import CollisionScene
    from untangling26_b200.prp import prp_params, response_params

    if ws > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    ctx = Context(local)
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0, max_ef_pairs=max(1 << 16, mesh.num_edges))
    sc.construct_lbvh()
    params = prp_params(max_contours=args.max_contours, batch_size=(1 << 20) if batch else 32)
    dev = torch.device("cuda", local)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    rparams = response_params(*RESPONSE)

    def device_pass():
        sc.refit_face_tree()
        sc.resolver.reset()
        sc.stats.zero_()
        sc.ef_detect(with_stats=True)
        n = sc.resolver.canonicalize(mesh.num_edges, mesh.num_faces)
        res = sc.host_resolve(params, num_pairs=n, response=rparams)
        return res

    for _ in range(max(args.warmup, 3)):
        device_pass()
    torch.cuda.synchronize()

    # ---- device-resident timed region
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = ctx.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    results = []
    ef_tests = []
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record(stream)
        sc.refit_face_tree()
        sc.resolver.reset()
        sc.stats.zero_()
        kev[i][0].record(stream)
        sc.ef_detect(with_stats=True)
        kev[i][1].record(stream)
        n = sc.resolver.canonicalize(mesh.num_edges, mesh.num_faces)
        res = sc.host_resolve(params, num_pairs=n, response=rparams)
        ev[i][1].record(stream)
        results.append(res)
        ef_tests.append(sc.stats[1])
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    ef_ms = [a.elapsed_time(b) for a, b in kev]
    ef_tests_pass = int(ef_tests[-1].item())
    prp_tests_pass = results[-1].pairs_tested
    tests_pass = ef_tests_pass + prp_tests_pass
    from untangling26_b200.multirank import job_throughput, job_time_ms
    total_ms = job_time_ms(sum(step_ms), device=dev)  # max over ranks (each rank runs its own scene replica)
    value = job_throughput(tests_pass * args.steps, ws, total_ms)
    r0 = results[-1]
    proc = r0.results[(r0.results["flags"] & 16) > 0]

    # ---- roofline of the dominant kernel (raycast_kernel, per the ncu launch list):
    # algorithmic bytes of all its launches in a pass / their CUDA-event time, per ray as
    # the survey defines them: 44 B per BVH node the ray's own traversal visits (32 B box +
    # 8 B children + 4 B leaf id), 48 B per triangle leaf test (12 B indices + 36 B
    # positions), 32 B per edge leaf test (8 B + 24 B), 24 B per request (source positions).
    # The packet kernel shares each node / leaf record among its 32 rays (packet fetches are
    # reported beside), so most of these bytes come from L1 / L2 (traffic: ncu).
    peak, peak_kind = _peaks()
    rc_bytes = 44 * r0.ray_visits + 48 * (r0.tested - r0.edge_tests) + 32 * r0.edge_tests + 24 * r0.requests
    rc_ms = r0.gpu_ms["raycast"]
    roof = {"bound": "hbm", "achieved": rc_bytes / (rc_ms / 1e3) / 1e9 if rc_ms > 0 else 0.0, "peak": peak, "unit": "GB/s",
            "peak_source": peak_kind, "kernel": "raycast_kernel", "kernel_ms_per_pass": rc_ms,
            "launches_per_pass": r0.levels + 1, "algorithmic_bytes_per_pass": rc_bytes, "traffic": None,
            "ray_node_visits": r0.ray_visits, "packet_node_tests": r0.nodes_visited, "packet_node_fetches": r0.node_fetches,
            "packet_leaf_fetches": r0.tri_fetches + r0.edge_fetches,
            "packet_bytes_per_pass": 32 * r0.node_fetches + 48 * r0.tri_fetches + 32 * r0.edge_fetches + 24 * r0.requests,
            "note": ("achieved: the per-ray bytes of all raycast launches of one pass over their time; a warp packet "
                     "shares each node and leaf record among its 32 rays, so these bytes come mostly from L1 / L2 and "
                     "the packet's own record traffic (packet_bytes_per_pass) is far below HBM bandwidth")}
    roof["frac"] = roof["achieved"] / peak
    st = sc.stats.cpu().numpy()
    ef_nodes, ef_prims = int(st[0]), int(st[1])
    n_ef = int(sc.resolver.ef_count.item())
    ef_bytes = 44 * ef_nodes + 48 * ef_prims + 32 * mesh.num_edges + 56 * n_ef
    ef_kms = statistics.mean(ef_ms)
    roof_ef = {"kernel": "ef_detect_kernel", "achieved": ef_bytes / (ef_kms / 1e3) / 1e9, "unit": "GB/s", "kernel_ms": ef_kms,
               "algorithmic_bytes_per_launch": ef_bytes}
    roof_ef["frac"] = roof_ef["achieved"] / peak
    prof = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            tr = json.load(f)
            roof["traffic"] = tr.get(roof["kernel"])
            roof_ef["traffic"] = tr.get("ef_detect_kernel")

    # ---- response assembly (inside every timed pass): collision pair templates + region CSRs.
    # Algorithmic bytes: per pair 44 B hit in, 2 x 12 B normals + 2 x 4 B areas, 64 B template +
    # 16 B info out, 4 vertex-label keys of 8 B written, sorted (4 radix passes of read + write)
    # and read; per EF pair 5 keys likewise; the three CSR arrays written once.
    rr = r0.response
    nkeys = 4 * rr.num_pairs + 5 * len(r0.pairs)
    rs_bytes = (44 + 32 + 80) * rr.num_pairs + 8 * nkeys * (2 + 2 * 4) + 4 * (
        int(rr.vert_regions.numel()) + int(rr.edge_regions.numel()) + int(rr.face_regions.numel()))
    resp = {"pairs": rr.num_pairs, "ms_per_pass": rr.ms, "algorithmic_bytes": rs_bytes,
            "achieved": rs_bytes / (rr.ms / 1e3) / 1e9 if rr.ms > 0 else 0.0, "unit": "GB/s",
            "region_words": [int(rr.vert_regions.numel()), int(rr.edge_regions.numel()), int(rr.face_regions.numel())],
            "note": "host wall time of u26_prp_make_response (hit upload, 12 launches, 2 synchronisations)"}

    # ---- region-based pair filtering on this pass's regions: proximity VF / EE pairs within
    # 1 mm (no shared vertex) from the scene trees (as narrow-phase templates) through u26_filter_invalid_pairs,
    # the same pairs as CCD broad-phase lists through u26_filter_broad_phase_pairs; L2 flushed
    # before each call pair. Algorithmic bytes: per proximity pair 64 B template + 48 B
    # positions + 8 B offsets (marking), then 64 B template + 8 B indices + 16 B marks +
    # 16 B region offsets (filter); per broad pair 8 B ids + 12 / 16 B primitive + 16 B marks
    # + 16 B region offsets + 8 B write.
    pf = _pair_filter_block(sc, mesh, dev, flush, stream, rr, n_ef, peak)

    # ---- LBVH refit: the fused leaf update + bottom-up refit of the face tree alone, L2
    # flushed before every launch. Algorithmic bytes (each byte once): V x (12 B position +
    # 4 B thickness) + F x (12 B face + 4 B leaf order + 32 B leaf box write) + (F - 1) x
    # (8 B children + 4 B parent + 64 B child boxes + 32 B box write).
    rf_n = 10
    rf_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(rf_n)]
    for i in range(rf_n):
        flush.fill_((i + 7) & 0xFF)
        rf_ev[i][0].record(stream)
        sc.refit_face_tree()
        rf_ev[i][1].record(stream)
    torch.cuda.synchronize()
    rf_ms = statistics.median(a.elapsed_time(b) for a, b in rf_ev)
    nvv, nff = mesh.num_verts, mesh.num_faces
    rf_bytes = 16 * nvv + 48 * nff + 108 * max(nff - 1, 0)
    refit = {"kernel": "refit_fused_kernel", "ms": rf_ms, "algorithmic_bytes": rf_bytes,
             "achieved": rf_bytes / (rf_ms / 1e3) / 1e9, "unit": "GB/s", "peak": peak, "launches": rf_n}
    refit["frac"] = refit["achieved"] / peak

    # ---- the plain form on the same input (same pairs and results): one thread per request
    # from the tree root, per-contour launches; for a batch of scenes, one pass per scene
    plain = None
    if args.plain_steps > 0:
        pparams = prp_params(max_contours=args.max_contours, batch_size=(1 << 20) if batch else 32, form=1)
        if batch:
            from untangling26_b200 import synthetic
            pscs = []
            for s_i in range(mesh.meta["num"]):
                m_i = synthetic.scene_mesh(mesh, s_i)
                sc_i = CollisionScene(ctx, m_i, d_hat=1e-3, thickness=0.0, max_ef_pairs=max(1 << 16, m_i.num_edges))
                sc_i.construct_lbvh()
                pscs.append((sc_i, m_i))
        else:
            pscs = [(sc, mesh)]

        def plain_pass():
            tests = 0
            for sc_i, m_i in pscs:
                sc_i.refit_face_tree()
                sc_i.resolver.reset()
                sc_i.stats.zero_()
                sc_i.ef_detect(with_stats=True)
                n_i = sc_i.resolver.canonicalize(m_i.num_edges, m_i.num_faces)
                r_i = sc_i.host_resolve(pparams, num_pairs=n_i, response=rparams)
                tests += int(sc_i.stats[1].item()) + r_i.pairs_tested
            return tests

        plain_pass()
        torch.cuda.synchronize()
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.plain_steps)]
        ptests = 0
        for i in range(args.plain_steps):
            flush.fill_(i & 0xFF)
            pev[i][0].record(stream)
            ptests = plain_pass()
            pev[i][1].record(stream)
        torch.cuda.synchronize()
        p_ms = sum(a.elapsed_time(b) for a, b in pev) / args.plain_steps
        plain = {"value": ptests / (p_ms / 1e3), "unit": UNIT, "ms_per_step": p_ms, "steps": args.plain_steps,
                 "same_tests": ptests == tests_pass, "untangle_passes_per_s": 1e3 / p_ms,
                 "chosen_over_plain": value / ws / (ptests / (p_ms / 1e3)),
                 "form": "one thread per request from the tree root, per-contour launches" + (", one pass per scene" if batch else "")}
        if batch:
            for sc_i, _ in pscs:
                sc_i.close()

    # ---- e2e through the public API with host buffers
    x_host = torch.from_numpy(mesh.x).pin_memory()
    e_ms = []
    d2h = 0
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sc.x.copy_(x_host, non_blocking=True)
        res = device_pass()  # the result arrays come back to the host inside u26_prp_resolve
        torch.cuda.synchronize()
        e_ms.append(1e3 * (time.perf_counter() - t0))
        d2h = int(sum(h.nbytes for h in res.hits) + res.results.nbytes + res.pairs.nbytes)
    e2e_ms = sum(e_ms)
    e2e_value = tests_pass * args.steps * ws / (e2e_ms / 1e3)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(mesh, args.max_contours)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(config, l2="flushed between steps (256 MB write)", parallelism=f"scene replica per GPU x{ws}",
                           max_contours=args.max_contours, directions="reference seeds (<=10 per contour)",
                           form="batched packet ray casting clipped to candidate boxes, all scenes in one pass"),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(mesh.x.nbytes), "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / args.steps},
            "untangle_passes_per_s": 1e3 * args.steps / total_ms,
            "plain_form": plain,
            "response": resp,
            "pair_filter": pf,
            "gpu_launches": int(launches), "roofline": roof, "lbvh_refit": refit, "clocks": clk,
            "pass": {"ef_pairs": n_ef, "contours": len(r0.contours), "processed": int(len(proc)),
                     "responses": int((proc["combo_idx"] != 0xFFFFFFFF).sum()), "levels": r0.levels,
                     "ef_leaf_tests": ef_tests_pass, "ray_pair_tests": prp_tests_pass,
                     "ray_leaf_tests_executed": r0.tested, "ray_requests": r0.requests,
                     "stage_ms": {k: round(v, 3) for k, v in r0.stage_ms.items()},
                     "gpu_ms": {k: round(v, 3) for k, v in r0.gpu_ms.items()}, "ef_detect_ms": ef_kms,
                     "nodes_visited": r0.nodes_visited, "roofline_ef_detect": roof_ef},
            "cpu_baseline": cpu}
        print(json.dumps(line))
    sc.close()
    if ws > 1:
        dist.destroy_process_group()
    ctx.close()


if __name__ == "__main__":
    main()
