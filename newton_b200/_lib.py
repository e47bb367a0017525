"""ctypes binding of ``libvbd_b200.so`` (declared in ``include/vbd_b200.h``).

The library is the only compute path: if it is missing or cannot be loaded, every solver call
raises -- there is no CPU or eager fallback.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libvbd_b200.so"

VBD_OK = 0
VBD_ERR_INVALID_ARGUMENT = 1
VBD_ERR_CUDA = 2
VBD_ERR_OUT_OF_MEMORY = 3
VBD_ERR_TIMEOUT = 4
VBD_ERR_UNSUPPORTED = 5

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_float_p = ctypes.POINTER(ctypes.c_float)


class VbdShape(ctypes.Structure):
    _fields_ = [
        ("geo_type", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("world", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("xform", ctypes.c_float * 7),
        ("scale", ctypes.c_float * 3),
        ("margin", ctypes.c_float),
        ("material_ke", ctypes.c_float),
        ("material_kd", ctypes.c_float),
        ("material_mu", ctypes.c_float),
    ]


class VbdModelDesc(ctypes.Structure):
    _fields_ = [
        ("particle_count", ctypes.c_int32),
        ("tri_count", ctypes.c_int32),
        ("edge_count", ctypes.c_int32),
        ("shape_count", ctypes.c_int32),
        ("color_count", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("particle_mass", c_float_p),
        ("particle_inv_mass", c_float_p),
        ("particle_radius", c_float_p),
        ("particle_flags", c_int32_p),
        ("particle_world", c_int32_p),
        ("tri_indices", c_int32_p),
        ("tri_poses", c_float_p),
        ("tri_materials", c_float_p),
        ("tri_areas", c_float_p),
        ("edge_indices", c_int32_p),
        ("edge_rest_angle", c_float_p),
        ("edge_rest_length", c_float_p),
        ("edge_bending_properties", c_float_p),
        ("v_adj_tris_offsets", c_int32_p),
        ("v_adj_tris", c_int32_p),
        ("v_adj_edges_offsets", c_int32_p),
        ("v_adj_edges", c_int32_p),
        ("color_group_offsets", c_int32_p),
        ("color_group_particles", c_int32_p),
        ("gravity", ctypes.c_float * 3),
        ("soft_contact_ke", ctypes.c_float),
        ("soft_contact_kd", ctypes.c_float),
        ("soft_contact_mu", ctypes.c_float),
        ("shapes", ctypes.POINTER(VbdShape)),
        ("particle_q", c_float_p),
    ]


class VbdSolverOptions(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("friction_epsilon", ctypes.c_float),
        ("lanes_per_vertex", ctypes.c_int32),
        ("block_size", ctypes.c_int32),
        ("contacts_per_vertex", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("step_kernel", ctypes.c_int32),
        ("self_contact", ctypes.c_int32),
        ("self_contact_radius", ctypes.c_float),
        ("self_contact_margin", ctypes.c_float),
        ("conservative_bound_relaxation", ctypes.c_float),
        ("vertex_contact_buffer_size", ctypes.c_int32),
        ("edge_contact_buffer_size", ctypes.c_int32),
        ("collision_detection_interval", ctypes.c_int32),
        ("edge_parallel_epsilon", ctypes.c_float),
        ("topological_filter_threshold", ctypes.c_int32),
        ("rest_exclusion_radius", ctypes.c_float),
        ("vertex_filter_offsets", ctypes.c_void_p),
        ("vertex_filter_triangles", ctypes.c_void_p),
        ("edge_filter_offsets", ctypes.c_void_p),
        ("edge_filter_edges", ctypes.c_void_p),
    ]


class VbdContacts(ctypes.Structure):
    _fields_ = [
        ("soft_contact_max", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("soft_contact_count", ctypes.c_void_p),
        ("soft_contact_particle", ctypes.c_void_p),
        ("soft_contact_indices", ctypes.c_void_p),
        ("soft_contact_barycentric", ctypes.c_void_p),
        ("soft_contact_shape", ctypes.c_void_p),
        ("soft_contact_body_pos", ctypes.c_void_p),
        ("soft_contact_body_vel", ctypes.c_void_p),
        ("soft_contact_normal", ctypes.c_void_p),
    ]


class VbdStatus(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64),
        ("nonfinite_updates", ctypes.c_int32),
        ("singular_blocks", ctypes.c_int32),
        ("contact_overflow", ctypes.c_int32),
        ("timeouts", ctypes.c_int32),
        ("self_contact_overflow", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class VbdGateStats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64),
        ("iterations", ctypes.c_int64),
        ("capped_steps", ctypes.c_int64),
        ("last_iterations", ctypes.c_int32),
        ("body_kernels", ctypes.c_int32),
        ("last_residual", ctypes.c_float),
        ("last_start_residual", ctypes.c_float),
        ("last_reference_residual", ctypes.c_float),
        ("body_programmatic_edges", ctypes.c_int32),
        ("body_passes", ctypes.c_int64),
    ]


# (name, restype, argtypes) of every exported entry point declared in include/vbd_b200.h
_VP = ctypes.c_void_p
SIGNATURES = {
    "vbd_last_error": (ctypes.c_char_p, []),
    "vbd_version": (ctypes.c_char_p, []),
    "vbd_model_create": (ctypes.c_int, [ctypes.POINTER(VbdModelDesc), ctypes.POINTER(_VP)]),
    "vbd_model_destroy": (ctypes.c_int, [_VP]),
    "vbd_collide": (ctypes.c_int, [_VP, _VP, ctypes.c_float, ctypes.POINTER(VbdContacts), _VP]),
    "vbd_solver_create": (ctypes.c_int, [_VP, ctypes.POINTER(VbdSolverOptions), ctypes.POINTER(_VP)]),
    "vbd_solver_destroy": (ctypes.c_int, [_VP]),
    "vbd_step": (
        ctypes.c_int,
        [_VP, _VP, _VP, _VP, _VP, _VP, ctypes.POINTER(VbdContacts), ctypes.c_float, ctypes.c_int32, _VP],
    ),
    "vbd_batch_step": (
        ctypes.c_int,
        [ctypes.POINTER(_VP), ctypes.c_int32, ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_VP),
         ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(ctypes.POINTER(VbdContacts)), ctypes.c_float,
         ctypes.POINTER(ctypes.c_int32), _VP],
    ),
    "vbd_step_static": (
        ctypes.c_int,
        [_VP, _VP, _VP, _VP, _VP, _VP, ctypes.POINTER(VbdContacts), ctypes.c_float, ctypes.c_int32, ctypes.c_float, _VP],
    ),
    "vbd_step_static_status": (ctypes.c_int, [ctypes.POINTER(VbdStatus)]),
    "vbd_forward": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.POINTER(VbdContacts), ctypes.c_float, _VP]),
    "vbd_sweep_color": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.POINTER(VbdContacts), ctypes.c_float, _VP]),
    "vbd_begin_iteration": (ctypes.c_int, [_VP, ctypes.c_int32, _VP]),
    "vbd_self_contact_detect": (ctypes.c_int, [_VP, _VP, _VP]),
    "vbd_self_contact_lists": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "vbd_finalize": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_float, _VP]),
    "vbd_get_positions": (ctypes.c_int, [_VP, _VP, _VP]),
    "vbd_warm_start": (ctypes.c_int, [_VP, _VP, _VP]),
    "vbd_mlp_sizes": (ctypes.c_int, [c_int32_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p]),
    "vbd_mlp_features": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "vbd_set_feature_set": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "vbd_set_staged_sweep": (ctypes.c_int, [_VP, ctypes.c_int32]),
    "vbd_set_warm_start_correction": (ctypes.c_int, [_VP, _VP, _VP]),
    "vbd_staged_sweep_info": (ctypes.c_int, [_VP, c_int32_p, c_int32_p, ctypes.POINTER(ctypes.c_int64)]),
    "vbd_mlp_forward": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int32, _VP, _VP]),
    "vbd_mlp_forward_mma_sync": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int32, _VP, _VP]),
    "vbd_mlp_timeouts": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int32]),
    "vbd_mlp_workspace_bytes": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "vbd_mlp_backward": (
        ctypes.c_int,
        [_VP, _VP, _VP, _VP, ctypes.c_int32, ctypes.c_float, _VP, _VP, _VP, ctypes.c_int64, _VP],
    ),
    "vbd_mlp_adam": (
        ctypes.c_int,
        [_VP, _VP, _VP, _VP, _VP, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, _VP],
    ),
    "vbd_mlp_pack_weights": (ctypes.c_int, [_VP, _VP, _VP]),
    "vbd_mlp_warm_start": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_int64, _VP]),
    "vbd_set_warm_start": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, ctypes.c_int32]),
    "vbd_residual": (ctypes.c_int, [_VP, ctypes.POINTER(VbdContacts), ctypes.c_float, _VP, _VP, _VP]),
    "vbd_status": (ctypes.c_int, [_VP, ctypes.POINTER(VbdStatus), ctypes.c_int32]),
    "vbd_set_residual_gate": (ctypes.c_int, [_VP, ctypes.c_float, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "vbd_gate_stats": (ctypes.c_int, [_VP, ctypes.POINTER(VbdGateStats), ctypes.c_int32]),
    "vbd_solver_info": (ctypes.c_int, [_VP, c_int32_p, c_int32_p, c_int32_p]),
    "vbd_set_launch": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32]),
    "vbd_solver_step_kernel": (ctypes.c_int, [_VP, c_int32_p, c_int32_p, c_int32_p]),
    "vbd_step_kernel_count": (ctypes.c_int, [_VP, c_int32_p]),
    "vbd_set_spin_limit": (ctypes.c_int, [_VP, ctypes.c_uint32]),
    "vbd_color_graph": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int64, c_int32_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, c_int32_p, c_int32_p],
    ),
    "vbd_coloring_graph_edges": (
        ctypes.c_int,
        [ctypes.c_int32, ctypes.c_int64, c_int32_p, c_int32_p, ctypes.POINTER(ctypes.c_int64)],
    ),
    "vbd_trimesh_graph_edges": (
        ctypes.c_int,
        [ctypes.c_int32, c_int32_p, ctypes.c_int64, c_int32_p, ctypes.c_int64, c_int32_p,
         ctypes.POINTER(ctypes.c_int64)],
    ),
    "vbd_mesh_edge_adjacency": (
        ctypes.c_int,
        [c_int32_p, ctypes.c_int32, c_int32_p, c_int32_p, c_int32_p, c_int32_p, c_int32_p],
    ),
    "vbd_mesh_vertex_csr": (
        ctypes.c_int,
        [c_int32_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, ctypes.c_int32, c_int32_p, c_int32_p],
    ),
    "vbd_mesh_edge_adjacency_device": (
        ctypes.c_int,
        [_VP, ctypes.c_int32, _VP, _VP, _VP, c_int32_p, c_int32_p, _VP],
    ),
    "vbd_mesh_vertex_csr_device": (
        ctypes.c_int,
        [_VP, ctypes.c_int32, ctypes.c_int32, c_int32_p, ctypes.c_int32, _VP, _VP, c_int32_p, _VP],
    ),
    "vbd_trimesh_graph_edges_device": (
        ctypes.c_int,
        [ctypes.c_int32, _VP, ctypes.c_int64, _VP, ctypes.c_int64, _VP, ctypes.POINTER(ctypes.c_int64), _VP],
    ),
}

_lib = None


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Load (building in-tree first if needed) the CUDA library; raises if it cannot."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() and build_if_missing and os.environ.get("VBD_NO_BUILD") != "1":
        from . import build as _build

        _build.build()
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m newton_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class VbdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[vbd error {code}] {message}")
        self.code = code


def check(code: int) -> None:
    if code != VBD_OK:
        msg = load().vbd_last_error()
        raise VbdError(code, msg.decode() if msg else "")


def ptr(arr) -> ctypes.c_void_p | None:
    """Address of a torch tensor / numpy array (None -> NULL)."""
    if arr is None:
        return None
    if isinstance(arr, np.ndarray):
        return ctypes.c_void_p(arr.ctypes.data)
    return ctypes.c_void_p(arr.data_ptr())


def as_i32p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(c_int32_p)


def as_f32p(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(c_float_p)


def color_graph(num_nodes: int, edges: np.ndarray, algorithm: int = 0, balance: bool = True, target_ratio: float = 1.1):
    """Color an undirected graph with the library's host coloring (vbd_color_graph)."""
    lib = load()
    edges = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1, 2))
    colors = np.empty(num_nodes, dtype=np.int32)
    nc = ctypes.c_int32(0)
    check(
        lib.vbd_color_graph(
            num_nodes,
            edges.shape[0],
            as_i32p(edges) if edges.size else None,
            algorithm,
            1 if balance else 0,
            float(target_ratio),
            as_i32p(colors) if num_nodes else None,
            ctypes.byref(nc),
        )
    )
    return colors, int(nc.value)


def mesh_edge_adjacency(tris: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """(edge_indices [ne,4], edge_tri [ne,2], tri_edge [nt,3], non-manifold sides) of a triangle
    mesh (vbd_mesh_edge_adjacency)."""
    lib = load()
    tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
    nt = tris.shape[0]
    edges = np.empty((3 * nt, 4), np.int32)
    edge_tri = np.empty((3 * nt, 2), np.int32)
    tri_edge = np.empty((nt, 3), np.int32)
    ne, bad = ctypes.c_int32(0), ctypes.c_int32(0)
    if nt:
        check(lib.vbd_mesh_edge_adjacency(as_i32p(tris), nt, as_i32p(edges), as_i32p(edge_tri), as_i32p(tri_edge),
                                          ctypes.byref(ne), ctypes.byref(bad)))
    return edges[: ne.value].copy(), edge_tri[: ne.value].copy(), tri_edge, bad.value


def mesh_vertex_csr(entries: np.ndarray, slot_of, particle_count: int) -> tuple[np.ndarray, np.ndarray]:
    """(values, offsets) of the per-vertex (element, slot) CSR (vbd_mesh_vertex_csr)."""
    lib = load()
    entries = np.ascontiguousarray(np.asarray(entries, dtype=np.int32))
    n_el, per = entries.shape
    slots = np.ascontiguousarray(np.asarray(slot_of, dtype=np.int32).reshape(-1))
    n_rec = int(np.count_nonzero(entries != -1))
    values = np.empty(max(2 * n_rec, 2), np.int32)
    offsets = np.zeros(particle_count + 1, np.int32)
    check(lib.vbd_mesh_vertex_csr(as_i32p(entries), n_el, per, as_i32p(slots), int(particle_count), as_i32p(values),
                                  as_i32p(offsets)))
    return values[: 2 * n_rec].copy(), offsets


def trimesh_graph_edges(num_nodes: int, tris: np.ndarray, bend: np.ndarray | None) -> np.ndarray:
    """Canonical conflict-graph edges of triangles + bending hinges (vbd_trimesh_graph_edges)."""
    lib = load()
    tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
    bend = np.ascontiguousarray(np.asarray(bend if bend is not None else np.empty((0, 4)), dtype=np.int32)
                                .reshape(-1, 4))
    cap = 3 * tris.shape[0] + 6 * bend.shape[0]
    out = np.empty((max(cap, 1), 2), np.int32)
    n = ctypes.c_int64(0)
    check(lib.vbd_trimesh_graph_edges(int(num_nodes), as_i32p(tris) if tris.size else None, tris.shape[0],
                                      as_i32p(bend) if bend.size else None, bend.shape[0], as_i32p(out),
                                      ctypes.byref(n)))
    return out[: n.value].copy()


def canonical_edges(num_nodes: int, pairs: np.ndarray) -> np.ndarray:
    """Unique (min, max) vertex pairs in lexicographic order (vbd_coloring_graph_edges)."""
    lib = load()
    pairs = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    out = np.empty_like(pairs)
    n = ctypes.c_int64(0)
    if pairs.shape[0] == 0:
        return out
    check(lib.vbd_coloring_graph_edges(int(num_nodes), pairs.shape[0], as_i32p(pairs), as_i32p(out), ctypes.byref(n)))
    return out[: n.value].copy()


# ---- the set-up tables on the GPU (same tables as the host functions above) ----------------------
def _dev_call(device):
    import torch

    dev = torch.device(device)
    return torch, dev, ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def mesh_edge_adjacency_device(tris: np.ndarray, device) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """mesh_edge_adjacency computed on ``device`` (vbd_mesh_edge_adjacency_device)."""
    lib = load()
    torch, dev, st = _dev_call(device)
    tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
    nt = tris.shape[0]
    if nt == 0:
        return np.empty((0, 4), np.int32), np.empty((0, 2), np.int32), np.empty((0, 3), np.int32), 0
    d_tris = torch.from_numpy(tris).to(dev)
    d_edges = torch.empty((3 * nt, 4), dtype=torch.int32, device=dev)
    d_edge_tri = torch.empty((3 * nt, 2), dtype=torch.int32, device=dev)
    d_tri_edge = torch.empty((nt, 3), dtype=torch.int32, device=dev)
    ne, bad = ctypes.c_int32(0), ctypes.c_int32(0)
    check(lib.vbd_mesh_edge_adjacency_device(ptr(d_tris), nt, ptr(d_edges), ptr(d_edge_tri), ptr(d_tri_edge),
                                             ctypes.byref(ne), ctypes.byref(bad), st))
    n = ne.value
    return d_edges[:n].cpu().numpy(), d_edge_tri[:n].cpu().numpy(), d_tri_edge.cpu().numpy(), bad.value


def mesh_vertex_csr_device(entries: np.ndarray, slot_of, particle_count: int, device) -> tuple[np.ndarray, np.ndarray]:
    """mesh_vertex_csr computed on ``device`` (vbd_mesh_vertex_csr_device)."""
    lib = load()
    torch, dev, st = _dev_call(device)
    entries = np.ascontiguousarray(np.asarray(entries, dtype=np.int32))
    n_el, per = entries.shape
    slots = np.ascontiguousarray(np.asarray(slot_of, dtype=np.int32).reshape(-1))
    d_entries = torch.from_numpy(entries).to(dev)
    d_values = torch.empty(max(2 * n_el * per, 2), dtype=torch.int32, device=dev)
    d_offsets = torch.empty(particle_count + 1, dtype=torch.int32, device=dev)
    n_rec = ctypes.c_int32(0)
    check(lib.vbd_mesh_vertex_csr_device(ptr(d_entries), n_el, per, as_i32p(slots), int(particle_count),
                                         ptr(d_values), ptr(d_offsets), ctypes.byref(n_rec), st))
    return d_values[: 2 * n_rec.value].cpu().numpy(), d_offsets.cpu().numpy()


def trimesh_graph_edges_device(num_nodes: int, tris: np.ndarray, bend: np.ndarray | None, device) -> np.ndarray:
    """trimesh_graph_edges computed on ``device`` (vbd_trimesh_graph_edges_device)."""
    lib = load()
    torch, dev, st = _dev_call(device)
    tris = np.ascontiguousarray(np.asarray(tris, dtype=np.int32).reshape(-1, 3))
    bend = np.ascontiguousarray(np.asarray(bend if bend is not None else np.empty((0, 4)), dtype=np.int32)
                                .reshape(-1, 4))
    cap = 3 * tris.shape[0] + 6 * bend.shape[0]
    if cap == 0:
        return np.empty((0, 2), np.int32)
    d_tris = torch.from_numpy(tris).to(dev) if tris.size else None
    d_bend = torch.from_numpy(bend).to(dev) if bend.size else None
    d_out = torch.empty((cap, 2), dtype=torch.int32, device=dev)
    n = ctypes.c_int64(0)
    check(lib.vbd_trimesh_graph_edges_device(int(num_nodes), ptr(d_tris), tris.shape[0], ptr(d_bend),
                                             bend.shape[0], ptr(d_out), ctypes.byref(n), st))
    return d_out[: n.value].cpu().numpy()
