"""ctypes binding of libipcb200.so (include/ipcb.h).

The library is required: there is no CPU fallback.  Importing this module
loads it; any call that launches work needs a CUDA device and raises if the
library is missing or a call reports an error.
"""
from __future__ import annotations

import contextlib
import ctypes
import gc
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libipcb200.so")

c_int, c_float, c_double, c_size_t, c_void_p = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p
P = c_void_p


class Soup(ctypes.Structure):
    _fields_ = [("n_verts", c_int), ("n_edges", c_int), ("n_tris", c_int), ("fp64", c_int),
                ("x", P), ("xcs", P), ("edges", P), ("triangles", P), ("body", P)]


class Contacts(ctypes.Structure):
    _fields_ = [("a1a2b1b2", P), ("e0e1", P), ("l0", P), ("alpha", P), ("lam", P), ("cnt", P),
                ("capacity", c_int)]


class Lbvh(ctypes.Structure):
    _fields_ = [("n", c_int), ("capacity", c_int), ("nodes", P), ("parent", P), ("sorted", P), ("keys", P),
                ("flags", P), ("wide", P)]


class Bodies(ctypes.Structure):
    _fields_ = [("n_bodies", c_int), ("local_lower", P), ("local_upper", P), ("edge_off", P), ("edge_ids", P),
                ("tri_off", P), ("tri_ids", P), ("vert_off", P), ("vert_ids", P), ("edge_wide", P), ("tri_wide", P),
                ("max_edges", c_int), ("max_tris", c_int), ("max_verts", c_int), ("frames", P), ("motion", P)]


class Abd(ctypes.Structure):
    _fields_ = [("n_bodies", c_int), ("fp64", c_int), ("q", P), ("q0", P), ("q_tilde", P), ("qdot", P), ("dx", P),
                ("mass", P), ("volume", P), ("stiffness", P), ("fixed", P)]


class Terms(ctypes.Structure):
    _fields_ = [("fp64", c_int), ("x", P), ("xcs", P), ("ee", Contacts), ("pt", Contacts), ("kappa", c_double),
                ("c_rows", P), ("c_cols", P), ("c_vals", P), ("c_mask", P), ("material", c_int), ("tets", P),
                ("n_tets", c_int), ("Bm", P), ("W", P), ("mu", c_double), ("lam", c_double), ("t_rows", P),
                ("t_cols", P), ("t_vals", P), ("force", P), ("queue", P), ("ee_ws", P), ("pt_ws", P),
                ("abd", Abd), ("body_row0", c_int), ("h2", c_double), ("a_rows", P), ("a_cols", P), ("a_vals", P),
                ("a_grad", P)]


class LsState(ctypes.Structure):
    _fields_ = [("E0", c_double), ("E1", c_double), ("alpha", c_double), ("ub", c_double), ("eps", c_double),
                ("alpha_accepted", c_double), ("it", c_int), ("max_it", c_int), ("accepted", c_int), ("done", c_int),
                ("overflow", c_int), ("max_ee", c_int), ("max_pt", c_int), ("refused", c_int)]


class AlSet(ctypes.Structure):
    _fields_ = [("table_size", c_int), ("capacity", c_int), ("cell_start", P), ("a1a2b1b2", P), ("e0e1", P),
                ("l0", P), ("alpha", P), ("lam", P), ("gamma", P), ("slack", P), ("mollifier", P), ("d0", P),
                ("distance_type", P), ("grad", P)]


class Mixed(ctypes.Structure):
    _fields_ = [("fp64", c_int), ("n_fem", c_int), ("n_verts", c_int), ("n_bodies", c_int), ("body", P),
                ("fixed", P), ("rest", P)]


class Graph(ctypes.Structure):
    _fields_ = [("n", c_int), ("nnz", c_int), ("n_lower", c_int), ("offsets", P), ("columns", P), ("rows", P),
                ("rev", P), ("diag", P), ("lower", P)]


class Tape(ctypes.Structure):
    _fields_ = [("h", P), ("e", P), ("m", P), ("a", P), ("u", P), ("proj", P), ("training", c_int)]


class PcgState(ctypes.Structure):
    _fields_ = [("rz", c_double), ("rz_new", c_double), ("pAp", c_double), ("rr", c_double), ("bb", c_double),
                ("tol2", c_double), ("last_rr", c_double), ("it", c_int), ("done", c_int), ("maxiter", c_int),
                ("status", c_int), ("arrived", c_int)]


class Pcg(ctypes.Structure):
    _fields_ = [("n", c_int), ("fp64", c_int), ("precond", c_int), ("offsets", P), ("columns", P), ("values", P),
                ("dinv", P), ("g_offsets", P), ("g_columns", P), ("diag", P), ("g", P), ("scale", P), ("b", P),
                ("x", P), ("r", P), ("z", P), ("p", P), ("q", P), ("t", P), ("state", P), ("n_point", c_int),
                ("n_groups", c_int), ("dinv_group", P), ("x0", P)]


SP, CP, BP = ctypes.POINTER(Soup), ctypes.POINTER(Contacts), ctypes.POINTER(Lbvh)
BD = ctypes.POINTER(Bodies)
AB = ctypes.POINTER(Abd)
MX = ctypes.POINTER(Mixed)
GP, TP = ctypes.POINTER(Graph), ctypes.POINTER(Tape)

# name -> (restype, argtypes); every symbol here is declared in include/ipcb.h
SIGNATURES = {
    "ipcb_version": (c_int, []),
    "ipcb_last_error": (ctypes.c_char_p, []),
    "ipcb_sort_workspace_u32": (c_size_t, [c_int]),
    "ipcb_sort_workspace_u64": (c_size_t, [c_int]),
    "ipcb_sort_pairs_u32": (c_int, [P, P, c_int, c_int, P, c_size_t, P]),
    "ipcb_sort_pairs_u64": (c_int, [P, P, c_int, c_int, P, c_size_t, P]),
    "ipcb_lbvh_bytes": (c_size_t, [c_int]),
    "ipcb_lbvh_bind": (c_int, [BP, P, c_int]),
    "ipcb_lbvh_build_workspace": (c_size_t, [c_int]),
    "ipcb_lbvh_build": (c_int, [BP, P, P, c_int, P, c_size_t, P]),
    "ipcb_lbvh_refit": (c_int, [BP, P, P, P]),
    "ipcb_lbvh_build_noalloc_scratch_bytes": (c_size_t, []),
    "ipcb_lbvh_build_noalloc": (c_int, [BP, P, P, c_int, P]),
    "ipcb_pack_positions": (c_int, [SP, P, P]),
    "ipcb_edge_aabbs": (c_int, [SP, P, c_float, P, P, P]),
    "ipcb_triangle_aabbs": (c_int, [SP, P, c_float, P, P, P]),
    "ipcb_add_dx": (c_int, [SP, P, P, P]),
    "ipcb_swept_edge_aabbs": (c_int, [SP, P, c_double, P, P, P]),
    "ipcb_swept_triangle_aabbs": (c_int, [SP, P, c_double, P, P, P]),
    "ipcb_dcd_ee": (c_int, [SP, P, BP, c_float, c_float, c_int, CP, P, P]),
    "ipcb_dcd_pt": (c_int, [SP, P, BP, c_float, c_float, c_int, P, CP, P, P]),
    "ipcb_dcd_ee_range": (c_int, [SP, P, BP, c_float, c_float, c_int, c_int, c_int, CP, P, P]),
    "ipcb_dcd_pt_range": (c_int, [SP, P, BP, c_float, c_float, c_int, P, c_int, c_int, CP, P, P]),
    "ipcb_contact_hessian": (c_int, [c_int, SP, CP, c_int, c_int, c_double, P, P, P, P, P, P]),
    "ipcb_contact_hessian_after": (c_int, [c_int, SP, CP, c_int, c_int, P, c_double, P, P, P, P, P, P]),
    "ipcb_contact_hessian_workspace": (c_size_t, [c_int]),
    "ipcb_edge_triangle_crossings": (c_int, [SP, BP, P, P, c_int, P, P]),
    "ipcb_contact_hessian_sorted": (c_int, [c_int, SP, CP, c_int, c_int, P, c_double, P, P, P, P, P, P, c_size_t, P]),
    "ipcb_contact_energy": (c_int, [c_int, SP, CP, c_int, c_double, P, P]),
    "ipcb_toi_workspace": (c_size_t, [c_int]),
    "ipcb_edge_edge_toi": (c_int, [SP, P, BP, P, P, c_int, P, P, P, c_size_t, P]),
    "ipcb_point_triangle_toi": (c_int, [SP, P, BP, c_double, c_int, P, P, P, c_size_t, P]),
    "ipcb_edge_edge_toi_range": (c_int, [SP, P, BP, P, P, c_int, c_int, c_int, P, P, P, c_size_t, P]),
    "ipcb_point_triangle_toi_range": (c_int, [SP, P, BP, c_double, c_int, c_int, c_int, P, P, P, c_size_t, P]),
    "ipcb_collision_time": (c_int, [c_int, c_int, P, P, P, P, P]),
    "ipcb_cubic_roots": (c_int, [c_int, P, c_double, c_double, P, P, P, P]),
    "ipcb_mpnn_param_count": (c_int, []),
    "ipcb_mpnn_packed_count": (c_int, []),
    "ipcb_mpnn_pack": (c_int, [P, P, P]),
    "ipcb_mpnn_graph_workspace": (c_size_t, [c_int]),
    "ipcb_mpnn_graph": (c_int, [GP, P, P, c_size_t, P]),
    "ipcb_mpnn_features": (c_int, [GP, c_int, P, P, P, P, P, P, P]),
    "ipcb_mpnn_forward": (c_int, [GP, P, P, P, P, P, TP, P, P, P]),
    "ipcb_fsai_normalize": (c_int, [GP, P, P, P, P, P, P, P, P]),
    "ipcb_mpnn_loss_grad": (c_int, [GP, P, P, P, P, P, c_double, P]),
    "ipcb_mpnn_backward_workspace": (c_size_t, [c_int, c_int, c_int]),
    "ipcb_mpnn_backward": (c_int, [GP, P, P, P, P, TP, P, P, P, P, c_size_t, P]),
    "ipcb_adam": (c_int, [c_int, P, P, P, P, c_float, c_float, c_float, c_float, c_int, P]),
    "ipcb_fsai_apply": (c_int, [GP, P, P, c_int, P, P, P, P]),
    "ipcb_pcg_start": (c_int, [ctypes.POINTER(Pcg), c_double, c_int, P]),
    "ipcb_pcg_iterate": (c_int, [ctypes.POINTER(Pcg), c_int, P]),
    "ipcb_block_jacobi": (c_int, [c_int, P, P, P, P, c_int, P, P, P]),
    "ipcb_group_jacobi": (c_int, [c_int, c_int, P, P, P, c_int, P, P, P]),
    "ipcb_fsai_mirror": (c_int, [GP, P, P, P]),
    "ipcb_terms_launch": (c_int, [ctypes.POINTER(Terms), c_int, c_int, c_int, c_int, P]),
    "ipcb_bsr_slots": (c_int, [c_int, P, P, c_int, P, P, P, P]),
    "ipcb_bsr_union_workspace": (c_size_t, [c_int]),
    "ipcb_bsr_union": (c_int, [c_int, P, P, P, P, P, P, P, P, P, c_int, P, P, P, c_size_t, P]),
    "ipcb_newton_values": (c_int, [c_int, P, c_int, P, P, P, P, P, P, P, c_double, P, P, c_double, P, P]),
    "ipcb_abi_hash": (ctypes.c_char_p, []),
    "ipcb_ls_inertia": (c_int, [c_int, c_int, P, P, P, P, c_double, P, P, P, c_double, P, P]),
    "ipcb_ls_begin": (c_int, [P, P, c_int, P, P, c_double, c_double, c_int, CP, CP, P]),
    "ipcb_ls_trial": (c_int, [P, c_int, c_int, P, P, P, P, P]),
    "ipcb_ls_accept": (c_int, [P, P, c_double, CP, CP, ctypes.c_ulonglong, P]),
    "ipcb_ls_finish": (c_int, [P, c_int, c_int, P, P, P]),
    "ipcb_acc_fold": (c_int, [P, P, c_int, P]),
    "ipcb_graph_while_begin": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(ctypes.c_ulonglong), P]),
    "ipcb_graph_while_end": (c_int, [c_void_p, P]),
    "ipcb_graph_launch": (c_int, [c_void_p, P]),
    "ipcb_graph_destroy": (None, [c_void_p]),
    "ipcb_edge_edge_intersections": (c_int, [SP, P, BP, P, P, c_int, c_double, P, CP, P, P, c_size_t, P]),
    "ipcb_point_triangle_intersections": (c_int, [SP, P, BP, c_double, c_int, c_double, P, CP, P, P, c_size_t, P]),
    "ipcb_al_vertex_toi": (c_int, [c_int, CP, c_int, P, P]),
    "ipcb_al_workspace": (c_size_t, [c_int]),
    "ipcb_al_create": (c_int, [c_int, ctypes.POINTER(AlSet), CP, c_int, P, P, c_size_t, P]),
    "ipcb_al_merge": (c_int, [c_int, ctypes.POINTER(AlSet), ctypes.POINTER(AlSet), ctypes.POINTER(AlSet), c_int, c_int,
                              P, c_size_t, P]),
    "ipcb_abd_map": (c_int, [c_int, c_int, P, P, P, P, P]),
    "ipcb_abd_step_from": (c_int, [c_int, c_int, P, P, c_double, P, P]),
    "ipcb_abd_prepare_tilde": (c_int, [AB, c_double, P, P, P, P]),
    "ipcb_abd_update_velocity": (c_int, [AB, c_double, P]),
    "ipcb_abd_body_system": (c_int, [AB, c_double, P, P, P, P, P]),
    "ipcb_abd_body_energy": (c_int, [AB, c_double, P, P]),
    "ipcb_abd_reduce_force": (c_int, [AB, c_int, P, P, P, P, P]),
    "ipcb_abd_add_contact_gradient": (c_int, [c_int, c_int, P, P, c_double, P]),
    "ipcb_abd_reduce_hessian": (c_int, [AB, c_int, P, P, P, P, P, c_double, P, P, P, P]),
    "ipcb_abd_pattern_workspace": (c_size_t, [c_int]),
    "ipcb_abd_pattern": (c_int, [c_int, P, P, c_int, P, P, P, P, P, c_int, P, P, P, P, P, c_size_t, P]),
    "ipcb_abd_assemble": (c_int, [AB, c_double, c_int, c_int, P, P, P, P, P, P, P, P, P, P, c_int, P, P, c_int, P, P,
                                  P, P]),
    "ipcb_mixed_map": (c_int, [MX, P, P, P]),
    "ipcb_mixed_reduce_force": (c_int, [MX, P, c_double, P, P]),
    "ipcb_mixed_hessian_workspace": (c_size_t, [c_int]),
    "ipcb_mixed_reduce_hessian": (c_int, [MX, c_int, P, P, P, P, c_double, c_int, P, P, P, P, P, P, c_size_t, P]),
    "ipcb_mixed_pins": (c_int, [MX, P, P, P, P, c_double, P, P, P, P, P, P]),
    "ipcb_body_pairs": (c_int, [BD, c_int, P, c_double, P, c_int, P, P, P]),
    "ipcb_fixed_dcd_ee": (c_int, [SP, P, BD, P, c_int, c_float, CP, P, P]),
    "ipcb_fixed_dcd_pt": (c_int, [SP, P, BD, P, c_int, c_float, CP, P, P]),
    "ipcb_body_pairs_swept": (c_int, [BD, c_int, P, P, c_double, P, c_int, P, P, P]),
    "ipcb_fixed_edge_edge_toi": (c_int, [SP, P, BD, P, P, c_int, c_double, P, P, P, c_size_t, P]),
    "ipcb_fixed_point_triangle_toi": (c_int, [SP, P, BD, P, c_int, c_double, P, P, P, c_size_t, P]),
    "ipcb_umma_gemm_bf16": (c_int, [c_int, c_int, c_int, P, P, P, P, P]),
    "ipcb_tet_rest": (c_int, [c_int, P, P, c_int, P, P, P]),
    "ipcb_tet_hessian": (c_int, [c_int, c_int, P, P, c_int, P, P, c_double, c_double, P, P, P, P, P]),
    "ipcb_tet_energy": (c_int, [c_int, c_int, P, P, c_int, P, P, c_double, c_double, P, P]),
    "ipcb_bsr_workspace": (c_size_t, [c_int, c_int, c_int]),
    "ipcb_bsr_from_triplets": (c_int, [c_int, c_int, c_int, P, P, P, c_int, P, P, P, P, P, c_size_t, P]),
    "ipcb_bsr_mv": (c_int, [c_int, P, P, P, c_int, P, P, c_double, c_double, P]),
    "ipcb_contact_bsr_workspace": (c_size_t, [c_int, c_int]),
    "ipcb_contact_bsr": (c_int, [CP, c_int, CP, c_int, c_int, P, P, c_int, P, P, P, P, P, P, c_size_t, P]),
}


@contextlib.contextmanager
def no_collection():
    """Garbage collection off for a CUDA graph capture: an object collected
    inside it (an earlier solver's graph, a tensor whose allocator queries
    events) must not touch the capturing stream."""
    was_on = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was_on:
            gc.enable()


class NativeError(RuntimeError):
    pass


_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        header = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ipcb.h")
        if os.path.exists(header):
            import hashlib

            with open(header, "rb") as f:
                want = hashlib.sha1(f.read()).hexdigest()[:16]
            have = L.ipcb_abi_hash().decode()
            if have != want:
                raise NativeError(f"{LIB_PATH} was built against another include/ipcb.h ({have} != {want}): "
                                  "rebuild it (`python -c 'import __graft_entry__ as g; g.build()'`)")
        _lib = L
    return _lib


def call(name: str, *args):
    """Invoke a C-ABI entry point; raise on a non-zero return code."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        msg = lib().ipcb_last_error()
        raise NativeError(f"{name} returned {rc}: {msg.decode() if msg else ''}")
    return rc


def size(name: str, *args) -> int:
    return int(getattr(lib(), name)(*args))


def ptr(t) -> int:
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else t.data_ptr()


def stream_handle(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)
