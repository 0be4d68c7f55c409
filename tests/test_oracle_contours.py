"""The oracle's contour flood fill with mesh parity against the reference's contour-construction
test (UnitTest/test_parallel_contour_construction.cpp).

That test builds eight graphs from one mt19937(42) (609-668) and accepts a contour construction
when (verify_results, 204-249): its components equal the breadth-first CPU reference's, its
"inconsistent" flag equals the reference's, and its parities equal the reference's on every
component whose edges all agree with the reference's parities (elsewhere they depend on the
walk order). The same rule holds here for flood_components, the depth-first fill the PRP
restatement uses for contours and mesh_index. The fixed 14-node case also has a known answer,
worked out by hand below.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _check(row_ptr, col, flip):
    root_b, par_b, bad_b = O.contour_test_bfs(row_ptr, col, flip)
    root_f, par_f, bad_f = O.flood_components(row_ptr, col, flip)
    assert np.array_equal(root_b, root_f)
    assert bad_b == bad_f
    n = len(row_ptr) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(row_ptr.astype(np.int64)))
    dst = col.astype(np.int64)
    # components whose every edge agrees with the reference's parities
    off = (par_b[src] ^ par_b[dst]) != (flip & 1)
    bad_roots = np.unique(root_b[src[off]])
    keep = ~np.isin(root_b, bad_roots)
    assert np.array_equal(par_b[keep], par_f[keep])
    return root_b, par_b, bad_b, keep


def test_small_fixed_known_answer():
    rp, cl, fl = O.contour_test_graph(0)
    root, par, bad, keep = _check(rp, cl, fl)
    # components {0,1,2}, {3,4,5}, {6}, {7,8,9,10}, {11,12,13}; the triangle 11-12-13 has three
    # flips (odd), so it is the one inconsistent component
    assert root.tolist() == [0, 0, 0, 3, 3, 3, 6, 7, 7, 7, 7, 11, 11, 11]
    assert bad
    assert keep.tolist() == [True] * 11 + [False] * 3
    # parities along the flips: 0-1 (1), 1-2 (0); 3-4 (1), 4-5 (1), 5-3 (0); 7-8 (0), 8-9 (1), 9-10 (1)
    assert par[:11].tolist() == [0, 1, 1, 0, 1, 0, 0, 0, 0, 1, 0]


@pytest.mark.parametrize("which", range(1, 8), ids=O.CONTOUR_TEST_GRAPHS[1:])
def test_flood_matches_reference_bfs(which):
    rp, cl, fl = O.contour_test_graph(which)
    n = len(rp) - 1
    root, par, bad, keep = _check(rp, cl, fl)
    ncomp = len(np.unique(root))
    # the shapes the test's generators give
    if which in (1, 2):
        chains, length, cycles = (10000, 10, 500) if which == 1 else (1000, 100, 200)
        assert n == chains * length and ncomp == chains
        # an open chain is always consistent: only closed cycles with an odd flip count are not
        assert keep.sum() >= (chains - cycles) * length
    elif which in (3, 4):
        assert ncomp == 1 and n == (10000 if which == 3 else 50000)
        assert bad  # random flips on a grid's 4-cycles: some are odd
    elif which in (5, 6):
        assert ncomp == (100 if which == 5 else 500)
    else:
        assert n == 100000 and ncomp == 50000 + 25000 and not bad


def test_flood_components_mutations():
    """A planted mistake, on the CPU: flipping one edge's weight in one direction only makes the
    graph's two directions disagree, and both fills report the inconsistency."""
    rp, cl, fl = O.contour_test_graph(0)
    fl = fl.copy()
    e = int(rp[0])  # the first entry of node 0 (0 -> 1)
    fl[e] ^= 1
    _, _, bad_b = O.contour_test_bfs(rp, cl, fl)
    _, _, bad_f = O.flood_components(rp, cl, fl)
    assert bad_b and bad_f
