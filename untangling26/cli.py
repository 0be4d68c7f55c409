"""Headless untangling of self-intersecting meshes or intersecting bodies.

Mirrors the reference's command line (PythonBindings/python/untangling26/cli.py:34-227:
make_parser, configure_solver, run_repair, repair, main; report keys of cli.py:194-215) over
this build's path. The reference drives its Newton / IP solver, which consumes the response
pairs as penalty terms; that solver is not part of this build, so each repair update here is
a fixed step along the assembled response (u26_response_step): every response pair pushes
its two sides apart along the contour's chosen direction by its requested depth, half each.
The intersection report of an update is taken at the positions it starts from, like the
reference's (cli.py:122-135), and a repair stops at zero EF intersections and contours.
"""
import argparse
import json
import math
from pathlib import Path
import sys
import time

VERSION = "0.2 (B200, sm_100a)"


def positive_int(value):
    result = int(value)
    if result <= 0:
        raise argparse.ArgumentTypeError("must be a positive integer")
    return result


def nonnegative_int(value):
    result = int(value)
    if result < 0:
        raise argparse.ArgumentTypeError("must be a nonnegative integer")
    return result


def positive_float(value):
    result = float(value)
    if not math.isfinite(result) or result <= 0:
        raise argparse.ArgumentTypeError("must be finite and positive")
    return result


def make_parser():
    p = argparse.ArgumentParser(
        prog="untangling26",
        description="Repair self-intersecting meshes or intersecting bodies on a B200 (no viewer).",
        epilog="Examples: untangling26 folded.obj repaired.obj\n"
               "          untangling26 body_a.obj body_b.obj out/ --material rigid",
        formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("inputs", nargs="+", type=Path, help="input OBJ files in shared world coordinates")
    p.add_argument("output", type=Path, help="output OBJ or directory (with per-body OBJ files)")
    p.add_argument("--material", choices=("cloth", "rigid"), default="cloth",
                   help="cloth: surface responses; rigid: bodies are solid (interior hit links) (default: cloth)")
    p.add_argument("--split-components", action=argparse.BooleanOptionalAction, default=None,
                   help="register disconnected components as separate bodies (default: on for rigid)")
    p.add_argument("--backend", choices=("auto", "cuda"), default="auto", help="compute backend: CUDA sm_100a (default: auto)")
    p.add_argument("--device", type=nonnegative_int, default=0, help="CUDA device ordinal (default: 0)")
    p.add_argument("--max-iters", type=nonnegative_int, default=200,
                   help="maximum repair updates; 0 checks and exports the input (default: 200)")
    p.add_argument("--response-depth", type=positive_float, default=1.0,
                   help="maximum requested correction in normalized scene units (default: 1)")
    p.add_argument("--direction-iters", type=nonnegative_int, default=0,
                   help="S^2 direction refinement steps per contour (default: 0)")
    p.add_argument("--max-contours", type=positive_int, default=256, help="contours processed per repair update (default: 256)")
    p.add_argument("--step-scale", type=positive_float, default=1.0,
                   help="fraction of the requested response applied per update (default: 1)")
    p.add_argument("--overwrite", action="store_true", help="replace existing outputs; input files are always protected")
    p.add_argument("--version", action="version", version=f"%(prog)s {VERSION}")
    return p


def configure(args):
    """(PRP parameters, response parameters) of the repair: the reference CLI's solver settings
    on this path (cli.py:93-118): PRP with solid-interior adjacency, ignore_near_zero_dist_pairs
    off, the requested direction refinement, response depth and contour count."""
    from untangling26_b200.prp import prp_params, response_params
    params = prp_params(max_contours=args.max_contours, opt_iterations=args.direction_iters, solid_interior=1,
                        ignore_near_zero_dist_pairs=0)
    return params, response_params(args.response_depth, 1e8)


def run_repair(scene, params, response, args, log=print):
    """Repair updates until the report shows no EF intersection and no contour, or the budget
    ends. Returns (positions of the last reported state, history records, converged): like the
    reference, the state returned is the one the last report describes, not the update after."""
    records = []
    snapshot = None
    for iteration in range(args.max_iters + 1):
        snapshot = scene.x.cpu().numpy().copy()
        res = scene.untangle_pass(params, response=response)
        ef, contours = int(res.num_orig_pairs), len(res.contours)
        records.append({"iteration": iteration, "ef_pairs": ef, "contours": contours, "response_pairs": res.response.num_pairs})
        log(f"Iteration {iteration}: {ef} EF intersections, {contours} contours", flush=True)
        if ef == 0 and contours == 0:
            return snapshot, records, True
        if iteration == args.max_iters:
            break
        if scene.response_step(res.response, args.step_scale) == 0:
            log("No response pairs: stopping", flush=True)
            break
    return snapshot, records, False


def repair(args):
    import numpy as np
    from untangling26_b200 import Context
    from untangling26_b200.intersection_resolver import CollisionScene
    from untangling26_b200.mesh_io import (Body, check_outputs, load_bodies, mesh_from_bodies, normalize_bodies, output_paths,
                                           validate_mesh, write_mesh)

    split = args.material == "rigid" if args.split_components is None else args.split_components
    bodies = load_bodies(args.inputs, split=split)
    mesh_paths, report_path = output_paths(args.output, bodies)
    check_outputs([*mesh_paths, report_path], args.inputs, overwrite=args.overwrite)
    normalized, center, scale = normalize_bodies(bodies)
    mesh = mesh_from_bodies(normalized)
    if args.material == "rigid":
        mesh.object_solid = np.ones(mesh.num_objects, np.uint32)
    print(f"Untangling {len(bodies)} bodies with {args.material} material; backend=cuda (sm_100a)", flush=True)
    start = time.perf_counter()
    ctx = Context(args.device)
    scene = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0)
    try:
        scene.construct_lbvh()
        params, response = configure(args)
        x, records, converged = run_repair(scene, params, response, args)
    finally:
        scene.close()
        ctx.close()
    repaired = []
    for k, body in enumerate(bodies):
        v0, v1 = int(mesh.prefix_num_verts[k]), int(mesh.prefix_num_verts[k + 1])
        v, f = validate_mesh(np.asarray(x[v0:v1], np.float64) * scale + center, body.faces, body.name)
        repaired.append(Body(body.name, v, f, body.source))
    write_mesh(mesh_paths[0], repaired)
    for path, body in zip(mesh_paths[1:], repaired):
        write_mesh(path, [body])
    report = {
        "inputs": [str(Path(p).resolve()) for p in args.inputs],
        "outputs": [str(p) for p in mesh_paths],
        "bodies": [{"name": b.name, "source": b.source, "vertices": len(b.vertices), "faces": len(b.faces)} for b in repaired],
        "converged": converged,
        "stop_reason": "zero_intersections" if converged else "iteration_budget",
        "initial_ef_pairs": records[0]["ef_pairs"],
        "final_ef_pairs": records[-1]["ef_pairs"],
        "iterations": records[-1]["iteration"],
        "solver_calls": len(records),
        "elapsed_seconds": time.perf_counter() - start,
        "configuration": {"backend": "cuda", "material": args.material, "split_components": split,
                          "update": "fixed step along the assembled response", "step_scale": args.step_scale,
                          "max_iters": args.max_iters, "response_depth": args.response_depth,
                          "direction_iters": args.direction_iters, "max_contours": args.max_contours},
        "normalization": {"center": [float(c) for c in center], "scale": scale, "largest_extent": 1.0},
        "history": records,
    }
    report_path.parent.mkdir(parents=True, exist_ok=True)
    report_path.write_text(json.dumps(report, indent=2) + "\n", encoding="utf-8")
    status = "Resolved" if converged else "Iteration budget reached with remaining intersections"
    print(f"{status}. Mesh: {mesh_paths[0]}\nReport: {report_path}", flush=True)
    return 0 if converged else 1


def main(argv=None):
    args = make_parser().parse_args(argv)
    try:
        return repair(args)
    except (ImportError, OSError, ValueError, RuntimeError, KeyError, IndexError) as exc:
        print(f"untangling26: {exc}", file=sys.stderr)
        return 2


if __name__ == "__main__":
    sys.exit(main())
