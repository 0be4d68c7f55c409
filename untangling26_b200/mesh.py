"""Mesh topology in the reference's conventions (host-side input preparation).

The reference builds these tables once per scene in its initialiser; the hot path reads
them. Ordering matters because later stages iterate adjacency lists in order:

* edges: sorted unique (v0 < v1) pairs, lexicographic (MeshOperation/mesh_reader.cpp:270-340)
* face_adj_edges[f][j]: the edge joining face[j] and face[(j+1) % 3] (Initializer/init_mesh_data.cpp:436-480)
* edge_adj_faces_ext[e]: incident faces in ascending face id (init_mesh_data.cpp:483-497)
* edge_adj_edges_ext[e]: for each incident face in that order, the face's two other
  edges in face_adj_edges order (init_mesh_data.cpp:499-533)
* vert_adj_verts[v]: other endpoint of each incident edge, in edge id order (init_mesh_data.cpp:337-347)
* vert_adj_edges / vert_adj_faces: incident ids ascending (init_mesh_data.cpp:300-317)
* face_adj_faces_ext[f]: for j in 0..2, the faces of face_adj_edges[f][j] other than f (init_mesh_data.cpp:535-551)
* rest areas: face area = |cross| / 2; vertex and edge areas = sum of incident face areas / 3
  (init_mesh_data.cpp:610-700)

Adjacency lists are CSR pairs (offsets[n+1], data[...]) of uint32 numpy arrays.
"""
import ctypes

import numpy as np

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f32p = ctypes.POINTER(ctypes.c_float)


class MeshDesc(ctypes.Structure):
    """u26_mesh_desc of include/u26.h: host pointers to the mesh tables."""
    _fields_ = [
        ("num_verts", ctypes.c_uint32), ("num_edges", ctypes.c_uint32), ("num_faces", ctypes.c_uint32),
        ("num_objects", ctypes.c_uint32),
        ("x", _f32p), ("rest_x", _f32p), ("edges", _u32p), ("faces", _u32p), ("face_adj_edges", _u32p),
        ("vav_off", _u32p), ("vav", _u32p), ("vae_off", _u32p), ("vae", _u32p), ("vaf_off", _u32p), ("vaf", _u32p),
        ("eaf_off", _u32p), ("eaf", _u32p), ("eae_off", _u32p), ("eae", _u32p),
        ("prefix_verts", _u32p), ("prefix_edges", _u32p), ("prefix_faces", _u32p),
        ("vert_object", _u32p), ("vert_component", _u32p),
        ("rest_vert_area", _f32p), ("rest_edge_area", _f32p), ("rest_face_area", _f32p), ("vert_mass", _f32p),
        ("mesh_orientation", _u32p), ("object_scene", _u32p), ("object_solid", _u32p),
    ]


class CSR:
    __slots__ = ("offsets", "data")

    def __init__(self, offsets, data):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.data = np.ascontiguousarray(data, dtype=np.uint32)

    def __len__(self):
        return len(self.offsets) - 1

    def row(self, i):
        return self.data[self.offsets[i]:self.offsets[i + 1]]

    def counts(self):
        return np.diff(self.offsets.astype(np.int64))

    def one_array(self):
        """upload_2d_csr_from's layout (buffer_allocator.h:26-59): [n + 1] absolute offsets
        into the same array, then the data."""
        n = len(self)
        off = self.offsets.astype(np.int64) - int(self.offsets[0]) + n + 1
        return np.concatenate([off, self.data.astype(np.int64)]).astype(np.uint32)


def _group(keys, values, n):
    """CSR of `values` grouped by `keys` (stable: original order kept inside a group)."""
    order = np.argsort(keys, kind="stable")
    counts = np.bincount(keys, minlength=n)
    offsets = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    return CSR(offsets, np.asarray(values)[order])


def extract_edges(faces):
    f = np.sort(faces.astype(np.int64), axis=1)
    pairs = np.concatenate([f[:, [0, 1]], f[:, [0, 2]], f[:, [1, 2]]], 0)
    nv = int(faces.max()) + 1 if len(faces) else 0
    keys = np.unique(pairs[:, 0] * nv + pairs[:, 1])
    return np.stack([keys // nv, keys % nv], 1).astype(np.uint32)


class Mesh:
    """Triangle mesh (one or more objects) with the reference's topology tables."""

    def __init__(self, x, faces, object_of_vert=None, rest_x=None, vert_property=None):
        self.x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        self.faces = np.ascontiguousarray(faces, dtype=np.uint32).reshape(-1, 3)
        self.rest_x = self.x.copy() if rest_x is None else np.ascontiguousarray(rest_x, dtype=np.float32)
        nv, nf = self.x.shape[0], self.faces.shape[0]
        self.num_verts, self.num_faces = nv, nf
        self.object_of_vert = (np.zeros(nv, np.uint32) if object_of_vert is None
                               else np.ascontiguousarray(object_of_vert, dtype=np.uint32))
        self.num_objects = int(self.object_of_vert.max()) + 1 if nv else 0
        # objects own contiguous vertex ranges (prefix_num_verts in the reference)
        self.prefix_num_verts = np.searchsorted(self.object_of_vert, np.arange(self.num_objects + 1)).astype(np.uint32)
        self.vert_property = (np.ascontiguousarray(vert_property, dtype=np.uint32) if vert_property is not None
                              else (self.object_of_vert.astype(np.uint32) & 0x7FFF) << 16)

        self.edges = extract_edges(self.faces)
        ne = self.edges.shape[0]
        self.num_edges = ne
        f64 = self.faces.astype(np.int64)
        e64 = self.edges.astype(np.int64)
        ekey = e64[:, 0] * nv + e64[:, 1]

        def edge_id(a, b):
            lo, hi = np.minimum(a, b), np.maximum(a, b)
            return np.searchsorted(ekey, lo * nv + hi)

        fae = np.stack([edge_id(f64[:, j], f64[:, (j + 1) % 3]) for j in range(3)], 1)
        self.face_adj_edges = fae.astype(np.uint32)
        fids = np.repeat(np.arange(nf, dtype=np.int64), 3)
        self.edge_adj_faces_ext = _group(fae.reshape(-1), fids, ne)

        # edge_adj_edges_ext: per (edge, incident face) in CSR order, the two other edges
        eaf = self.edge_adj_faces_ext
        row_edge = np.repeat(np.arange(ne, dtype=np.int64), eaf.counts())
        fa = fae[eaf.data.astype(np.int64)]  # (k, 3)
        keep = fa != row_edge[:, None]
        others = fa[keep].reshape(-1, 2)
        offs = (eaf.offsets.astype(np.int64) * 2)
        self.edge_adj_edges_ext = CSR(offs, others.reshape(-1))

        # vertex adjacency (edge id order, endpoint 0 then 1)
        ve_keys = np.stack([e64[:, 0], e64[:, 1]], 1).reshape(-1)
        ve_other = np.stack([e64[:, 1], e64[:, 0]], 1).reshape(-1)
        ve_eid = np.repeat(np.arange(ne, dtype=np.int64), 2)
        self.vert_adj_verts = _group(ve_keys, ve_other, nv)
        self.vert_adj_edges = _group(ve_keys, ve_eid, nv)
        self.vert_adj_faces = _group(f64.reshape(-1), fids, nv)

        # face_adj_faces_ext
        rows = []
        for j in range(3):
            rows.append(fae[:, j])
        # built lazily where needed (not on the EF path)
        self._face_adj_faces_ext = None

        # rest areas (double accumulation, stored float32)
        rx = self.rest_x.astype(np.float64)
        cr = np.cross(rx[f64[:, 1]] - rx[f64[:, 0]], rx[f64[:, 2]] - rx[f64[:, 0]])
        self.rest_face_area = (0.5 * np.linalg.norm(cr, axis=1)).astype(np.float32)
        fa64 = self.rest_face_area.astype(np.float64)
        va = np.zeros(nv, np.float64)
        for j in range(3):
            np.add.at(va, f64[:, j], fa64 / 3.0)
        self.rest_vert_area = va.astype(np.float32)
        ea = np.zeros(ne, np.float64)
        for j in range(3):
            np.add.at(ea, fae[:, j], fa64 / 3.0)
        self.rest_edge_area = ea.astype(np.float32)

        # per-object primitive ranges (edges and faces come grouped by object)
        eobj = self.object_of_vert[self.edges[:, 0]] if ne else np.zeros(0, np.uint32)
        fobj = self.object_of_vert[self.faces[:, 0]] if nf else np.zeros(0, np.uint32)
        self.prefix_num_edges = np.searchsorted(eobj, np.arange(self.num_objects + 1)).astype(np.uint32)
        self.prefix_num_faces = np.searchsorted(fobj, np.arange(self.num_objects + 1)).astype(np.uint32)
        if not (np.all(np.diff(eobj.astype(np.int64)) >= 0) and np.all(np.diff(fobj.astype(np.int64)) >= 0)):
            raise ValueError("edges and faces must be grouped by object (objects own contiguous vertex ranges)")
        # unit density and thickness: vertex mass = rest vertex area
        self.vert_mass = self.rest_vert_area.copy()
        self.mesh_orientation = np.zeros(max(self.num_objects, 1), np.uint32)
        self.vert_component = self._components()

    def _components(self):
        """Connected components of the vertex graph, numbered per object in vertex order."""
        from scipy.sparse import csr_matrix
        from scipy.sparse.csgraph import connected_components
        nv = self.num_verts
        off, data = self.vert_adj_verts.offsets.astype(np.int64), self.vert_adj_verts.data.astype(np.int64)
        g = csr_matrix((np.ones(len(data), np.int8), data, off), shape=(nv, nv))
        _, labels = connected_components(g, directed=False)
        # relabel by first vertex so that components count up in vertex order inside an object
        first = np.full(labels.max() + 1 if nv else 0, nv, np.int64)
        np.minimum.at(first, labels, np.arange(nv))
        order = np.argsort(first, kind="stable")
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        lab = rank[labels]
        comp = np.zeros(nv, np.uint32)
        for obj in range(self.num_objects):
            lo, hi = int(self.prefix_num_verts[obj]), int(self.prefix_num_verts[obj + 1])
            if hi > lo:
                comp[lo:hi] = (lab[lo:hi] - lab[lo:hi].min()).astype(np.uint32)
        return comp

    def desc(self, x=None):
        """ctypes MeshDesc over this mesh's host arrays (keeps references alive)."""
        d = MeshDesc()
        keep = []

        def p(a, t=ctypes.c_uint32):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(t))

        xx = self.x if x is None else np.ascontiguousarray(x, dtype=np.float32)
        d.num_verts, d.num_edges, d.num_faces, d.num_objects = self.num_verts, self.num_edges, self.num_faces, self.num_objects
        d.x = p(xx, ctypes.c_float)
        d.rest_x = p(self.rest_x, ctypes.c_float)
        d.edges = p(self.edges)
        d.faces = p(self.faces)
        d.face_adj_edges = p(self.face_adj_edges)
        for name in ("vert_adj_verts", "vert_adj_edges", "vert_adj_faces", "edge_adj_faces_ext", "edge_adj_edges_ext"):
            csr = getattr(self, name)
            short = {"vert_adj_verts": "vav", "vert_adj_edges": "vae", "vert_adj_faces": "vaf",
                     "edge_adj_faces_ext": "eaf", "edge_adj_edges_ext": "eae"}[name]
            setattr(d, short + "_off", p(csr.offsets))
            setattr(d, short, p(csr.data))
        d.prefix_verts = p(self.prefix_num_verts)
        d.prefix_edges = p(self.prefix_num_edges)
        d.prefix_faces = p(self.prefix_num_faces)
        d.vert_object = p(self.object_of_vert)
        d.vert_component = p(self.vert_component)
        d.rest_vert_area = p(self.rest_vert_area, ctypes.c_float)
        d.rest_edge_area = p(self.rest_edge_area, ctypes.c_float)
        d.rest_face_area = p(self.rest_face_area, ctypes.c_float)
        d.vert_mass = p(self.vert_mass, ctypes.c_float)
        d.mesh_orientation = p(self.mesh_orientation)
        scene = getattr(self, "object_scene", None)
        d.object_scene = p(scene) if scene is not None else None
        solid = getattr(self, "object_solid", None)
        d.object_solid = p(np.asarray(solid, np.uint32)) if solid is not None else None
        d._keep = keep
        return d

    def device_arrays(self, device="cuda"):
        """torch tensors of the arrays the kernels read."""
        import torch
        return {
            "x": torch.from_numpy(self.x).to(device),
            "edges": torch.from_numpy(self.edges.astype(np.int32)).to(device),
            "faces": torch.from_numpy(self.faces.astype(np.int32)).to(device),
            "vert_property": torch.from_numpy(self.vert_property.astype(np.int32)).to(device),
        }
