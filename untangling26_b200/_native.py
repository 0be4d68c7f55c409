"""ctypes binding of libu26.so, the C ABI declared in include/u26.h.

The product path always goes through this library. There is no CPU fallback: if the
shared library is missing or no CUDA device is present, the calls raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libu26.so")

_lib = None

c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_int = ctypes.c_int
c_vp = ctypes.c_void_p
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)

STATUS = {
    0: "OK", 1: "CAPACITY", 2: "UNHEALTHY_TREE", 3: "ITERATION_CAP", 4: "INVALID_INPUT", 5: "CUDA", 6: "NO_DEVICE",
}

TREE_VERT, TREE_FACE, TREE_EDGE = 0, 1, 2
QUERY_VERTS, QUERY_EDGES, QUERY_EDGES_UNCULLED = 0, 1, 2
DEVERR_UNHEALTHY, DEVERR_ITERATION_CAP, DEVERR_STACK_OVERFLOW = 1, 2, 4


class U26Error(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"u26 error {STATUS.get(status, status)}: {message}")
        self.status = status


class U26LbvhArrays(ctypes.Structure):
    _fields_ = [
        ("num_leaves", c_u32), ("num_nodes", c_u32),
        ("morton_sorted", c_vp), ("sorted_get_original", c_vp), ("parent", c_vp), ("children", c_vp),
        ("object_idx", c_vp), ("node_aabb", c_vp), ("global_aabb", c_vp),
    ]


# name -> (restype, argtypes). Pointers to device memory are passed as c_void_p.
_SIGS = {
    "u26_version": (ctypes.c_char_p, []),
    "u26_ctx_create": (c_int, [c_int, c_vp, ctypes.POINTER(c_vp)]),
    "u26_ctx_destroy": (None, [c_vp]),
    "u26_ctx_set_stream": (c_int, [c_vp, c_vp]),
    "u26_ctx_synchronize": (c_int, [c_vp]),
    "u26_ctx_last_error": (ctypes.c_char_p, [c_vp]),
    "u26_ctx_device_errors": (c_int, [c_vp, c_u32p, c_int]),
    "u26_ctx_launch_count": (c_u64, [c_vp]),
    "u26_alloc_count": (c_u64, []),
    "u26_lbvh_create": (c_int, [c_vp, c_int, c_u32, ctypes.POINTER(c_vp)]),
    "u26_lbvh_destroy": (None, [c_vp]),
    "u26_lbvh_reduce_aabb": (c_int, [c_vp, c_vp, c_u32, c_vp]),
    "u26_lbvh_construct_tree": (c_int, [c_vp]),
    "u26_lbvh_update_leaves": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "u26_lbvh_refit": (c_int, [c_vp]),
    "u26_lbvh_update_and_refit": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "u26_lbvh_query": (c_int, [c_vp, c_int, c_vp, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_u32]),
    "u26_lbvh_check_health": (c_int, [c_vp, ctypes.POINTER(c_int)]),
    "u26_lbvh_arrays_get": (c_int, [c_vp, ctypes.POINTER(U26LbvhArrays)]),
    "u26_ef_narrow_phase": (c_int, [c_vp, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_u32]),
    "u26_ef_detect": (c_int, [c_vp, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_u32, c_vp]),
    "u26_lbvh_set_option": (c_int, [c_vp, c_int, c_int]),
    "u26_ef_canonicalize_noalloc": (c_int, [c_vp, c_u32, c_vp, c_vp, c_u32, c_u32]),
    "u26_scene_create": (c_int, [c_vp, c_vp, ctypes.POINTER(c_vp)]),
    "u26_scene_destroy": (None, [c_vp]),
    "u26_prp_resolve": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_u32, c_vp, ctypes.POINTER(c_vp)]),
    "u26_prp_output_view_get": (c_int, [c_vp, c_vp]),
    "u26_prp_output_destroy": (None, [c_vp]),
    "u26_ef_canonicalize": (c_int, [c_vp, c_u32, c_vp, c_vp, c_u32, c_u32]),
    "u26_prp_adjoint": (c_int, [c_vp, c_vp, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "u26_prp_make_response": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_u32, c_u32, c_vp]),
    "u26_response_step": (c_int, [c_vp, c_vp, c_u32, c_vp, c_u32, ctypes.c_float, c_vp, c_vp]),
    "u26_ef_add_from_proximity": (c_int, [c_vp, c_vp, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_u32]),
    "u26_filter_invalid_pairs": (c_int, [c_vp, c_vp, c_vp, c_u32, c_u32, c_vp, c_vp, c_u32, c_vp, c_vp, c_vp, c_vp]),
    "u26_filter_broad_phase_pairs": (c_int, [c_vp, c_vp, c_u32, c_vp, c_u32, c_u32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
}


def declared_symbols():
    """Every entry point declared in include/*.h (parsed from the headers)."""
    import glob
    import re
    names = []
    inc = os.path.join(os.path.dirname(HERE), "include")
    for h in sorted(glob.glob(os.path.join(inc, "*.h"))):
        with open(h) as f:
            names += re.findall(r"U26_API\s+[\w\s\*]+?\b(u26_\w+)\s*\(", f.read())
    return names


def load(path=None):
    """Load libu26.so (building it first when this checkout has nvcc and no library)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(p)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(t):
    """Device pointer of a torch tensor (None passes NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


class Context:
    """One u26_ctx bound to a CUDA device and stream (torch's current stream by default)."""

    def __init__(self, device=0, stream=None):
        import torch
        self.lib = load()
        if not torch.cuda.is_available():
            raise U26Error(6, "no CUDA device: libu26 has no CPU path")
        self.device = device
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        h = c_vp()
        st = self.lib.u26_ctx_create(device, c_vp(stream.cuda_stream), ctypes.byref(h))
        if st != 0:
            raise U26Error(st, "u26_ctx_create failed")
        self.handle = h

    def check(self, st, what=""):
        if st != 0:
            msg = self.lib.u26_ctx_last_error(self.handle)
            raise U26Error(st, f"{what}: {msg.decode() if msg else ''}")

    def synchronize(self):
        self.check(self.lib.u26_ctx_synchronize(self.handle), "synchronize")

    def device_errors(self, reset=True):
        f = c_u32(0)
        self.check(self.lib.u26_ctx_device_errors(self.handle, ctypes.byref(f), int(reset)), "device_errors")
        return f.value

    def launch_count(self):
        return int(self.lib.u26_ctx_launch_count(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.u26_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
