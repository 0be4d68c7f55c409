"""Test infrastructure: comparisons of a GPU pass with the oracle's (or of two GPU passes),
used by tests/ and by bench.py's cpu_baseline leg. Every comparison is exact: per-contour
result fields bit for bit, candidate directions and support hits byte for byte."""
import numpy as np

# fields that name a contour's place in a batch rather than its result
BATCH_PLACE_FIELDS = ("contour_idx", "object_id0", "object_id1")
# fields set before cross-contour suppression (the result record of a suppressed contour
# keeps these; its support and metrics are cleared)
PRE_SUPPRESSION_FIELDS = ("contour_idx", "contour_type", "num_pairs", "num_dirs", "object_id0", "object_id1", "init_k_src",
                          "init_k_dst", "diam_src", "diam_dst", "num_boundary_src", "num_boundary_dst", "pre_finalize_area")
SUPPRESSED = 4


def map_batch_hits(h, v0, e0, f0):
    """Hits of a batched pass renumbered to their scene's own vertex / edge / face ids."""
    h = h.copy()
    vf, ee, fv = h["type"] == 0, h["type"] == 1, h["type"] == 2
    h["src_id"][vf] -= v0
    h["dst_id"][vf] -= f0
    h["src_id"][ee] -= e0
    h["dst_id"][ee] -= e0
    h["src_id"][fv] -= f0
    h["dst_id"][fv] -= v0
    for k in ("sv", "dv"):
        a = h[k]
        a[a != 0xFFFFFFFF] -= v0
    return h


def compare_scene(batched, batch_mesh, j, own):
    """Scene j of a batched pass (its contours are those of objects 2j, 2j + 1) against the
    scene's own pass `own` (GPU or oracle). Returns (contours, hits) compared; raises
    AssertionError at the first difference."""
    info = batch_mesh.meta["scenes"][j]
    tag = info.get("batch_scene", j)
    v0, f0 = info["verts"][0], info["faces"][0]
    e0 = int(np.searchsorted(batch_mesh.edges[:, 0], v0))
    mine = [c for c in range(len(batched.contours)) if batched.results[c]["object_id0"] // 2 == j]
    assert len(mine) == len(own.contours), f"scene {tag}: {len(mine)} contours, other pass {len(own.contours)}"
    nh = 0
    for cs, cb in enumerate(mine):
        ra, rb = own.results[cs], batched.results[cb]
        for name in ra.dtype.names:
            if name in BATCH_PLACE_FIELDS or name.startswith("reserved"):
                continue
            assert np.array_equal(ra[name], rb[name]), f"scene {tag} contour {cs} field {name}: {rb[name]} vs {ra[name]}"
        assert own.directions[cs].tobytes() == batched.directions[cb].tobytes(), f"scene {tag} contour {cs} directions"
        assert own.hits[cs].tobytes() == map_batch_hits(batched.hits[cb], v0, e0, f0).tobytes(), f"scene {tag} contour {cs} support"
        nh += len(own.hits[cs])
    return len(mine), nh


def compare_contours(gpu, ref, contours):
    """The listed contours of a whole-scene GPU pass against an oracle pass that evaluated
    (at least) those contours. Suppression pairs contours of one object pair, and a sampled
    oracle pass sees only some of them, so a contour suppressed in either pass is compared on
    its pre-suppression fields and candidate directions. Returns the hits compared."""
    nh = 0
    for c in contours:
        ra, rb = ref.results[c], gpu.results[c]
        suppressed = bool((int(ra["flags"]) | int(rb["flags"])) & SUPPRESSED)
        for name in (PRE_SUPPRESSION_FIELDS if suppressed else ra.dtype.names):
            if name.startswith("reserved"):
                continue
            assert np.array_equal(ra[name], rb[name]), f"contour {c} field {name}: gpu {rb[name]} oracle {ra[name]}"
        assert ref.directions[c].tobytes() == gpu.directions[c].tobytes(), f"contour {c} directions"
        if not suppressed:
            assert ref.hits[c].tobytes() == gpu.hits[c].tobytes(), f"contour {c} support"
            nh += len(ref.hits[c])
    return nh
