"""OBJ input and output for the untangling26 entry point, with one shared world-to-solver
transform (the interface of the reference's PythonBindings/python/untangling26/mesh_io.py:
Body, validate_mesh, split_components, load_bodies, normalize_bodies, output_paths,
check_outputs, write_mesh). The reference reads many formats through trimesh, which this
image does not have; this reader takes Wavefront OBJ (vertex and face records, polygons
fan-triangulated, negative indices, `o` / `g` records starting a new body)."""
from dataclasses import dataclass
from pathlib import Path
import re

import numpy as np

INPUT_FORMATS = {".obj"}
OUTPUT_FORMATS = {".obj"}


@dataclass
class Body:
    name: str
    vertices: np.ndarray
    faces: np.ndarray
    source: str


def validate_mesh(vertices, faces, name):
    """Checks of mesh_io.py:24-39: a nonempty finite (N, 3) vertex array and integer
    triangles inside it."""
    vertices = np.asarray(vertices, dtype=np.float64)
    faces = np.asarray(faces)
    if vertices.ndim != 2 or vertices.shape[1] != 3 or len(vertices) == 0:
        raise ValueError(f"{name}: expected a nonempty (N, 3) vertex array")
    if not np.isfinite(vertices).all():
        raise ValueError(f"{name}: vertices contain NaN or infinity")
    if faces.ndim != 2 or faces.shape[1] != 3 or len(faces) == 0:
        raise ValueError(f"{name}: expected a nonempty triangle mesh")
    if not np.issubdtype(faces.dtype, np.integer):
        raise ValueError(f"{name}: triangle indices must be integers")
    if faces.min() < 0 or faces.max() >= len(vertices):
        raise ValueError(f"{name}: triangle index is outside the vertex array")
    if len(vertices) > np.iinfo(np.int32).max:
        raise ValueError(f"{name}: too many vertices for the solver")
    return np.ascontiguousarray(vertices), np.ascontiguousarray(faces, dtype=np.int32)


def split_components(vertices, faces):
    """Connected components by shared vertex indices, each with its used vertices renumbered
    in increasing order (mesh_io.py:42-63)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    nv = len(vertices)
    f = np.asarray(faces, np.int64)
    rows = np.concatenate([f[:, 0], f[:, 1]])
    cols = np.concatenate([f[:, 1], f[:, 2]])
    _, label = connected_components(coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(nv, nv)), directed=False)
    face_label = label[f[:, 0]]
    # components in the order of their first face
    _, first = np.unique(face_label, return_index=True)
    for lab in face_label[np.sort(first)]:
        sel = f[face_label == lab]
        used, inverse = np.unique(sel, return_inverse=True)
        yield vertices[used], inverse.reshape(-1, 3).astype(np.int32)


def _read_obj(path):
    """[(name, vertices, faces)] of an OBJ file: one body per `o` / `g` record that has faces,
    vertex indices global to the file (the format's convention)."""
    verts = []
    bodies = []
    name, faces = path.stem, []
    with open(path, "r", encoding="utf-8", errors="replace") as fh:
        for raw in fh:
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            tag, _, rest = line.partition(" ")
            if tag == "v":
                vals = rest.split()
                if len(vals) < 3:
                    raise ValueError(f"{path}: vertex record with fewer than 3 coordinates")
                verts.append([float(vals[0]), float(vals[1]), float(vals[2])])
            elif tag == "f":
                idx = []
                for tok in rest.split():
                    k = int(tok.split("/", 1)[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)
                if len(idx) < 3:
                    raise ValueError(f"{path}: face record with fewer than 3 vertices")
                for j in range(1, len(idx) - 1):  # fan triangulation of polygons
                    faces.append([idx[0], idx[j], idx[j + 1]])
            elif tag in ("o", "g"):
                if faces:
                    bodies.append((name, faces))
                name, faces = (rest.strip() or path.stem), []
    if faces:
        bodies.append((name, faces))
    v = np.asarray(verts, np.float64).reshape(-1, 3)
    out = []
    for nm, fl in bodies:
        f = np.asarray(fl, np.int64)
        if f.min() < 0 or f.max() >= len(v):
            raise ValueError(f"{path}: triangle index is outside the vertex array")
        used, inverse = np.unique(f, return_inverse=True)  # drop unreferenced vertices
        out.append((nm, v[used], inverse.reshape(-1, 3)))
    return out


def load_bodies(paths, *, split=False):
    """Bodies of the input files in order (mesh_io.py:66-103); with split, every connected
    component becomes a body of its own."""
    bodies = []
    for path in paths:
        path = Path(path).resolve()
        if not path.is_file():
            raise ValueError(f"Input mesh not found: {path}")
        if path.suffix.lower() not in INPUT_FORMATS:
            raise ValueError(f"Unsupported input format: {path.suffix}")
        count = 0
        for node, v, f in _read_obj(path):
            name = re.sub(r"[^\w.-]+", "_", f"{path.stem}_{node}").strip("._") or "body"
            v, f = validate_mesh(v, f, name)
            for pv, pf in (split_components(v, f) if split else [(v, f)]):
                bodies.append(Body(f"{len(bodies):03d}_{name}", pv, pf, str(path)))
                count += 1
        if not count:
            raise ValueError(f"{path}: no triangle meshes found")
    return bodies


def normalize_bodies(bodies):
    """Translate and scale all bodies together so the scene's largest extent is 1
    (mesh_io.py:106-114). Returns (normalized bodies, center, scale)."""
    lower = np.min([b.vertices.min(axis=0) for b in bodies], axis=0)
    upper = np.max([b.vertices.max(axis=0) for b in bodies], axis=0)
    center = 0.5 * lower + 0.5 * upper
    scale = float(np.max(upper - lower))
    if not np.isfinite(scale) or scale <= 0:
        raise ValueError("The scene must have a finite, nonzero extent")
    return [Body(b.name, (b.vertices - center) / scale, b.faces, b.source) for b in bodies], center, scale


def output_paths(destination, bodies):
    """(mesh paths, report path): an .obj file and its .json report, or a directory with
    resolved.obj (+ one OBJ per body when there are several) and summary.json
    (mesh_io.py:117-126)."""
    destination = Path(destination).resolve()
    if destination.suffix.lower() in OUTPUT_FORMATS:
        return [destination], destination.with_suffix(".json")
    if destination.suffix and not destination.is_dir():
        raise ValueError("Output must be an .obj or a directory")
    meshes = [destination / "resolved.obj"]
    if len(bodies) > 1:
        meshes.extend(destination / f"{b.name}.obj" for b in bodies)
    return meshes, destination / "summary.json"


def check_outputs(paths, inputs, *, overwrite=False):
    """Refuse to overwrite an input, or an existing output without overwrite (mesh_io.py:129-135)."""
    input_paths = {Path(p).resolve() for p in inputs}
    for path in paths:
        if Path(path).resolve() in input_paths:
            raise ValueError(f"Output would overwrite an input mesh: {path}")
        if Path(path).exists() and (not overwrite or not Path(path).is_file()):
            raise ValueError(f"Output already exists: {path}; choose another path or use --overwrite")


def write_mesh(path, bodies):
    """All bodies into one OBJ, one `o` record each, vertex indices global to the file."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", encoding="utf-8", newline="\n") as fh:
        fh.write("# untangling26 output; coordinates in the input's units\n")
        base = 1
        for b in bodies:
            fh.write(f"o {b.name}\n")
            for p in np.asarray(b.vertices, np.float64):
                fh.write(f"v {p[0]:.17g} {p[1]:.17g} {p[2]:.17g}\n")
            for t in np.asarray(b.faces, np.int64) + base:
                fh.write(f"f {t[0]} {t[1]} {t[2]}\n")
            base += len(b.vertices)


def mesh_from_bodies(bodies):
    """One Mesh with every body an object of its own (objects own contiguous vertex ranges)."""
    from .mesh import Mesh
    xs, fs, obj = [], [], []
    nv = 0
    for k, b in enumerate(bodies):
        xs.append(np.asarray(b.vertices, np.float64))
        fs.append(np.asarray(b.faces, np.int64) + nv)
        obj.append(np.full(len(b.vertices), k, np.uint32))
        nv += len(b.vertices)
    return Mesh(np.concatenate(xs).astype(np.float32), np.concatenate(fs).astype(np.uint32), object_of_vert=np.concatenate(obj))
