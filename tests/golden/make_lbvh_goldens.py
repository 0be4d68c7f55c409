"""Extract the reference LBVH unit-test goldens into ``lbvh_unit_test.json``.

The reference pins its LBVH in ``Solver/CollisionDetector/lbvh.cpp``:

* ``LBVH::unit_test`` (lbvh.cpp:920-984): eight leaves at ``pos = lid / 10`` on all
  three axes, with the expected 30-bit Morton codes (``answer_morton32``) and the
  expected 64-bit keys (``answer_morton64``).
* ``fn_build_inner_nodes`` (lbvh.cpp:566-597): the expected Karras ranges, splits,
  children and parents for those eight keys, written as ``// Should be [...]``
  comments.

This script reads that source text (the reference cannot be compiled here: its
LuisaCompute submodule is empty) and writes the numbers as JSON. It is run by hand
in a container that has the reference checked out; the JSON is committed.

Usage: python tests/golden/make_lbvh_goldens.py /path/to/reference
"""
import json
import os
import re
import sys


def _ints(text):
    return [int(v) for v in re.findall(r"-?\d+", text)]


def main(ref_root):
    src_path = os.path.join(ref_root, "Solver", "CollisionDetector", "lbvh.cpp")
    with open(src_path, encoding="utf-8") as f:
        src = f.read()

    m32 = re.search(r"answer_morton32\s*=\s*\{([^}]*)\}", src)
    m64 = re.search(r"answer_morton64\s*=\s*\{([^}]*)\}", src)
    should = re.findall(r"//\s*Should be (\[.*\])", src)
    if not (m32 and m64 and len(should) >= 4):
        raise SystemExit("could not locate the LBVH goldens in " + src_path)

    ranges = [(_ints(a)[0], _ints(b)[0]) for a, b in re.findall(r"(\d+)\s*->\s*(\d+)", should[0])]
    splits = _ints(should[1])
    children = [tuple(_ints(p)) for p in re.findall(r"\[(\d+,\s*\d+)\]", should[2])]
    parents = _ints(should[3])

    out = {
        "source": "Solver/CollisionDetector/lbvh.cpp (LBVH::unit_test and fn_build_inner_nodes comments)",
        "num_leaves": 8,
        "position_rule": "pos = float(lid) / 10.0 on x, y and z",
        "morton32": _ints(m32.group(1)),
        "morton64": _ints(m64.group(1)),
        "ranges": [list(r) for r in ranges],
        "splits": splits,
        "inner_children": [list(c) for c in children[:7]],
        "parents": parents,
        "note": "parents[0] and the leaf children are unset in the reference unit test (it skips fn_reset_tree and fn_apply_sorted); compare parents[1:] and inner children only",
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lbvh_unit_test.json")
    with open(dst, "w", encoding="utf-8") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_lbvh_goldens.py /path/to/reference-checkout")
    main(sys.argv[1])
