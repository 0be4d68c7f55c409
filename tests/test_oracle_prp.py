"""Known-answer tests of the oracle's PRP decision rules, from the reference's own unit test
UnitTest/test_prp_selection.cpp (its cases restated here, expected values as it states
them), plus properties of the S^2 direction refinement on small scenes. CPU only.

Reference functions pinned: contour-side ownership and restriction predicates
(intersection_resolver2.h:405-506), the response comparator (h:807-912), contour
classification (intersection_resolver2.cpp:311-375), pre-finalize suppression (453-592),
the adaptive k-ring control (1058-1230), direction seeds (1488-1569), penetration metrics
(1883-1954) and the direction optimisation step (1268-1368).
"""
import numpy as np
import pytest

FMAX = float(np.finfo(np.float32).max)
INV = 0xFFFFFFFF


# ---- contour roles and the contour-side restriction

def test_roles_share_topology(oracle):
    assert oracle.ccr_roles_share((3, 3), (5, 5))
    assert not oracle.ccr_roles_share((3, 3), (5, 8))       # disconnected components
    assert not oracle.ccr_roles_share((3, 7), (5, 5))       # different objects
    assert not oracle.ccr_roles_share((3, 3), (INV, INV))   # no component identity


def test_restriction_applies(oracle):
    assert oracle.ccr_applies(True, (3, 3), (5, 5))
    assert not oracle.ccr_applies(False, (3, 3), (5, 5))    # opt-in
    assert not oracle.ccr_applies(True, (3, 7), (5, 5))
    assert not oracle.ccr_applies(True, (3, 3), (5, 8))
    # with current-space (deformed) distances: any two valid object identities
    assert oracle.ccr_applies(True, (3, 7), (5, 8), use_deformed=True)
    assert oracle.ccr_applies(True, (3, 3), (5, 8), use_deformed=True)
    assert not oracle.ccr_applies(True, (INV, 7), (5, 8), use_deformed=True)


def test_single_metric_ownership(oracle):
    assert oracle.ccr_owns(0.25, 1.0)
    assert not oracle.ccr_owns(1.0, 0.25)
    assert oracle.ccr_owns(0.5, 0.5)            # the bisector belongs to both covers
    assert oracle.ccr_owns(0.5, FMAX)           # opposite contour unreachable
    assert not oracle.ccr_owns(FMAX, 0.5)       # own contour unreachable


def test_dual_metric_ownership(oracle):
    d = oracle.ccr_owns_dual
    assert not d(10.0, 1.0, 0.1, 0.2)           # failed rest constraint wins
    assert not d(1.0, 10.0, 0.9, 0.1)           # failed current constraint wins
    assert d(2.0, 3.0, 0.3, 0.2)
    assert not d(2.0, 3.0, 0.3, 0.2, tau=0.0)   # tau applies to both metrics
    assert d(5.0, 3.0, 0.5, 0.3)                # closed tau = 0.25 boundary
    assert d(0.5, FMAX, 0.1, 0.2)
    assert not d(0.5, FMAX, 0.9, 0.1)
    assert not d(FMAX, 0.5, 0.1, 0.2)
    for tau in (0.0, 0.25, 1.0):
        assert d(1.0, 10.0, 0.9, 0.1, tau, True, False)                 # rest only
        assert d(10.0, 1.0, 0.1, 0.2, tau, False, True)                 # current only
        assert d(10.0, 1.0, 0.1, 0.2, tau, True, False) == (tau == 1.0)
        assert d(1.0, 10.0, 0.9, 0.1, tau, False, True) == (tau == 1.0)


def test_blended_ownership(oracle):
    b = oracle.ccr_owns_blended
    assert b(8.0, 2.0, 4.0, 6.0, 0.25, 0.5)
    assert not oracle.ccr_owns_dual(8.0, 2.0, 4.0, 6.0)
    assert not b(8.0, 2.0, 4.0, 6.0, 0.25, 0.75)
    assert b(800.0, 200.0, 0.4, 0.6, 0.25, 0.5)     # normalized coordinates, not raw distances
    assert b(8.0, 2.0, 4.0, 6.0, 0.25, 0.0)
    assert not b(8.0, 2.0, 4.0, 6.0, 0.25, 1.0)
    assert not b(1.0, 9.0, 9.0, 1.0, 0.25, 0.0)
    assert b(1.0, 9.0, 9.0, 1.0, 0.25, 1.0)
    assert b(5.0, 3.0, 5.0, 3.0, 0.25, 0.5)
    assert not b(FMAX, 1.0, FMAX, 1.0, 1.0, 0.5)
    assert not b(0.5, FMAX, 0.9, 0.1, 0.25, 1.0)     # incomplete rest pair: current decides
    assert b(1.0, 9.0, FMAX, 0.1, 0.25, 0.0)         # incomplete current pair: rest decides
    for w in (0.0, 0.25, 0.5, 0.75, 1.0):
        assert abs(oracle.ccr_blended_phi(8.0, 2.0, 4.0, 6.0, w) - (0.8 * w - 0.2)) < 1e-6


# ---- response comparator

def test_ineligible_response_does_not_compete(oracle):
    assert oracle.select_response([oracle.response(10.0, 1.0, True), oracle.response(0.01, 1.0, False)]) == 0


def test_comparator_divides_by_squared_coverage(oracle):
    # 4 / 1^2 = 4 beats 1 / 0.25^2 = 16
    assert oracle.select_response([oracle.response(4.0, 1.0), oracle.response(1.0, 0.25)]) == 0
    assert oracle.response_objective(1.0, 0.25) == pytest.approx(16.0)


def test_no_valid_response(oracle):
    empty = oracle.response(0.0, 0.0, False, hit_count=0, covered=0)
    assert oracle.select_response([empty, empty]) == -1


def test_comparator_tolerance_and_tie_breaks(oracle):
    # objectives within 1e-7 + 1e-5 max(|a|,|b|) tie; depth, then cost, then hit count decide
    a = oracle.response(1.0, 1.0, depth=2.0)
    b = oracle.response(1.0 + 5e-6, 1.0, depth=1.0)
    assert oracle.select_response([a, b]) == 1
    c = oracle.response(1.0, 1.0, depth=1.0, cost=3.0)
    d = oracle.response(1.0, 1.0, depth=1.0, cost=2.0)
    assert oracle.select_response([c, d]) == 1
    e = oracle.response(1.0, 1.0, hit_count=5)
    f = oracle.response(1.0, 1.0, hit_count=3)
    assert oracle.select_response([e, f]) == 1
    # a full tie keeps the first (smaller combo index)
    assert oracle.select_response([oracle.response(1.0, 1.0), oracle.response(1.0, 1.0)]) == 0


# ---- pre-finalize suppression

def test_one_way_adjacency_suppresses_the_touched_contour(oracle):
    assert oracle.suppress([[1], []], [1.0, 10.0], [0, 1]) == [1]


def test_mutual_adjacency_keeps_the_larger_area(oracle):
    assert oracle.suppress([[1], [0]], [1.0, 2.0], [0, 1]) == [0]
    assert oracle.suppress([[1], [0]], [2.0, 2.0], [0, 1]) == [1]   # equal areas: smaller index owns


# ---- contour classification (ContourType: 0 Undefined, 1 Closed, 2 Eight, 3 LL, ...)

def test_contour_types(oracle):
    # three non-loop pairs whose EF graph is a cycle: Closed
    assert oracle.classify_contour([0, 0, 0], [0, 0, 0], [2, 2, 2], [0, 0, 0]) == 1
    # a path with degree-one endpoints is not Closed
    assert oracle.classify_contour([0, 0, 0], [0, 0, 0], [1, 2, 1], [0, 0, 0]) == 0
    # loop-vertex storage nodes do not open the contour
    assert oracle.classify_contour([1], [0], [1], [0]) == 2
    assert oracle.classify_contour([1, 1], [0, 0], [1, 1], [0, 0]) == 3
    # boundary-ending contours
    assert oracle.classify_contour([0, 0, 0], [1, 0, 1], [1, 2, 1], [0, 0, 1]) == 6
    assert oracle.classify_contour([0, 0, 0], [1, 0, 1], [1, 2, 1], [0, 0, 0]) == 7
    assert oracle.classify_contour([1, 0], [0, 1], [1, 1], [0, 0]) == 4
    assert oracle.classify_contour([0, 1, 0], [1, 0, 1], [1, 2, 1], [0, 0, 0]) == 5


# ---- penetration metrics

def test_penetration_known_answer(oracle):
    """One VF hit, source vertex rest area 3, depth 0.1, normal along the direction:
    volume = 3 * 1 * 0.1 = 0.3 and J = 3 * 0.1^2 = 0.03."""
    n = np.array([0.0, 1.0, 0.0], np.float32)
    h = oracle.hit(0, 0, 0, [0], [1, 2, 3], (0.2, 0.3), 0.1)
    area3 = np.full(4, 3.0, np.float32)
    mass = np.ones(4, np.float32)
    vn = np.tile(n, (4, 1))
    for target in (n, -n):
        m = oracle.penetration(h, n, area3, np.zeros(0, np.float32), np.array([2.0], np.float32), mass, vn,
                               np.zeros((0, 3), np.float32), target.reshape(1, 3))
        assert abs(m["volume"] - 0.3) < 1e-6
        assert abs(m["objective"] - 0.03) < 1e-6
        assert m["depth"] == pytest.approx(0.1)
        assert m["area"] == pytest.approx(3.0)
        # the target face normal (flip metadata) does not enter the displacement cost
        sd = np.float32(0.1) + np.float32(3e-3)
        kappa = np.float32(1.0) + np.float32(0.2) ** 2 + np.float32(0.3) ** 2 + np.float32(0.5) ** 2
        assert m["cost"] == pytest.approx(float(sd * sd / kappa), rel=1e-6)


# ---- candidate directions

def test_seed_direction_slots(oracle):
    """Ten seeds in slot order: +-e0, +-e1, +-e2 (ascending eigenvalues of the anchors'
    area-weighted scatter about the contour centre), centre - side-0 centroid, centre -
    side-1 centroid, +-(centre - global centroid); all unit length."""
    x = np.array([[-3, -2, -1], [-3, 2, -1], [-3, 0, 1], [3, -2, -1], [3, 2, -1], [3, 0, 1]], np.float32)
    area = np.ones(6, np.float32)
    pts = np.array([[0, 0.4, 0.4], [0, 0.6, 0.4], [0, 0.4, 0.6], [0, 0.6, 0.6]], np.float32)
    d = oracle.seed_directions(pts, np.ones(4, np.float32), [0, 1, 2], [3, 4, 5], x, area)
    assert d.shape == (10, 3)
    assert np.all(np.abs(np.einsum("ij,ij->i", d, d) - 1.0) <= 1e-6)
    c = pts.astype(np.float64).mean(0)
    S = sum(np.outer(v - c, v - c) for v in x.astype(np.float64))
    w, V = np.linalg.eigh(S)
    for k in range(3):
        assert np.allclose(d[2 * k], -d[2 * k + 1])
        assert abs(abs(float(np.dot(d[2 * k], V[:, k]))) - 1.0) < 1e-5
    unit = lambda v: v / np.linalg.norm(v)
    assert np.allclose(d[6], unit(c - x[:3].mean(0)), atol=1e-6)
    assert np.allclose(d[7], unit(c - x[3:].mean(0)), atol=1e-6)
    g = x.astype(np.float64).mean(0)
    assert np.allclose(d[8], unit(c - g), atol=1e-6)
    assert np.allclose(d[9], -unit(c - g), atol=1e-6)


def test_lattice_directions(oracle):
    x = np.zeros((2, 3), np.float32)
    d = oracle.seed_directions(np.zeros((1, 3), np.float32), [1.0], [0], [1], x, np.ones(2, np.float32), mode=1)
    assert d.shape == (26, 3)
    assert len({tuple(np.round(v, 5)) for v in d}) == 26


# ---- adaptive k-ring control

def _info(objective=1.0, coverage=1.0, mfs=0, mfd=0, anchors=1, covered=1, hits=1):
    return dict(hit_count=hits, covered=covered, anchors=anchors, mfs=mfs, mfd=mfd, objective=objective, coverage=coverage)


def test_kring_detachment_needs_frontier_clearance(oracle):
    # full coverage at k = 2 while the support still touches hop 2: grow to 4, then detached
    r = oracle.kring_trace((2, 2), (8, 8), lambda lv, ks, kd, c: _info(mfs=2, mfd=2))
    assert r["evaluations"] == 2 and r["eligible"] == [True]
    assert r["trace"] == [(2, 2), (4, 4)]


def test_kring_grows_only_the_touching_role(oracle):
    # an inactive direction with a better cached result must not prune the active one
    def ev(level, ks, kd, combo):
        return _info(coverage=0.5, anchors=2, mfs=2 if level == 0 else 3, mfd=1)
    cached = [None, dict(_info(objective=0.001), eligible=1)]
    r = oracle.kring_trace((2, 2), (8, 8), ev, active=[1, 0], cached=cached)
    assert r["trace"] == [(2, 2), (4, 2)]
    assert r["eligible"][0]


def test_kring_empty_rays_terminate_at_the_mesh_bound(oracle):
    r = oracle.kring_trace((2, 2), (8, 8), lambda lv, ks, kd, c: {})
    assert r["evaluations"] == 3 and r["no_response"] and r["finished"]
    assert r["trace"] == [(2, 2), (4, 4), (8, 8)]


def test_kring_exhausted_role_does_not_shrink(oracle):
    r = oracle.kring_trace((2, 2), (0, 8), lambda lv, ks, kd, c: {})
    assert all(ks == 2 for ks, _ in r["trace"])
    assert r["no_response"]


def test_kring_exhausted_and_detached_roles_finish_at_once(oracle):
    r = oracle.kring_trace((2, 2), (2, 8), lambda lv, ks, kd, c: _info(coverage=0.5, anchors=2, mfs=2, mfd=1))
    assert r["evaluations"] == 1 and r["eligible"] == [True]


# ---- S^2 direction refinement

def _step_setup(oracle):
    x = np.array([[0, 0, 1], [0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    mass = np.ones(4, np.float32)
    r0 = np.array([0.6, 0.0, 0.8], np.float32)
    h = oracle.hit(0, 0, 0, [0], [1, 2, 3], (0.2, 0.2), 1.0)
    return x, mass, r0, h


def test_direction_step_moves_towards_the_face_normal(oracle):
    """VF hit onto the z = 0 face from a ray along (0.6, 0, 0.8): the depth derivative has a
    tangent component, the step is valid, unit, shorter than the trust radius, predicts a
    reduction and rotates the direction towards the normal (0, 0, 1)."""
    x, mass, r0, h = _step_setup(oracle)
    d, pred, gnorm, valid = oracle.direction_step(h, x, mass, r0, 0.3)
    assert valid and pred > 0.0 and gnorm > 1e-6
    assert abs(float(np.dot(d, d)) - 1.0) < 1e-6
    assert float(np.dot(d, r0)) < 1.0 - 1e-6
    assert d[2] > r0[2]
    ang = np.arccos(np.clip(np.dot(d, r0), -1, 1))
    assert ang <= 0.3 + 1e-5


def test_direction_step_invalid_cases(oracle):
    x, mass, r0, h = _step_setup(oracle)
    # ray along the face normal: no tangent gradient
    assert not oracle.direction_step(h, x, mass, np.array([0, 0, 1], np.float32), 0.3)[3]
    # no hits, zero direction
    assert not oracle.direction_step(h[:0], x, mass, r0, 0.3)[3]
    assert not oracle.direction_step(h, x, mass, np.zeros(3, np.float32), 0.3)[3]


def test_refinement_is_monotone_and_bounded(oracle):
    """On a folded sheet: no refinement by default; with 8 iterations every trial count is
    bounded, accepted <= attempted, and no contour's J / coverage^2 gets worse."""
    from untangling26_b200 import synthetic
    m = synthetic.folded_sheet(32, seed=2)
    ef, idx = oracle.detect_ef(m)
    base = oracle.PrpRun(m, ef, idx, oracle.prp_params(max_contours=32))
    assert all(r["opt_attempted"] == 0 for r in base.results)
    ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(max_contours=32, opt_iterations=8))
    for a, b in zip(base.results, ref.results):
        assert b["opt_attempted"] <= 8 and b["opt_accepted"] <= b["opt_attempted"]
        if a["hit_count"] and b["hit_count"]:
            assert b["normalized_objective"] <= a["normalized_objective"]
        if b["opt_accepted"]:
            assert abs(float(np.dot(b["dir"], b["dir"])) - 1.0) < 1e-5


def test_summation_order_spread(oracle):
    """The selected supports' FP32 area, volume, displacement cost and J summed in the canonical
    order (kernels and oracle) against the reference's deterministic block reduce
    (cpu_parallel.h:505-538) over the hits in key order and in 8 seeded shuffles: within the
    1e-5 relative tolerance the metrics are held to, on supports of several thousand hits."""
    from untangling26_b200 import synthetic
    m = synthetic.two_sheets(64, seed=0)
    ef, idx = oracle.detect_ef(m)
    run = oracle.PrpRun(m, ef, idx, oracle.prp_params(), order_spread=8)
    assert run.results["hit_count"].max() > 4000
    assert 0.0 < run.order_spread.max() < 1e-5
