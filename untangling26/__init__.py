"""untangling26: the command-line repair entry point over the B200 untangling path.

`untangling26 IN.obj OUT.obj` (or `python -m untangling26 ...`) detects the edge-face
intersections of the input bodies, evaluates every intersection contour's response on the GPU
(untangling26_b200, libu26.so) and moves the vertices along the assembled responses until no
intersection is left or the iteration budget ends, then writes the meshes and a JSON report
(the interface of the reference's PythonBindings/python/untangling26/cli.py)."""
from .cli import configure, main, make_parser, repair, run_repair

__all__ = ["configure", "main", "make_parser", "repair", "run_repair"]
