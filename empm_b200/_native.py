"""ctypes binding of libempm_b200.so (include/empm_b200.h).

The library is built in-tree by ``empm_b200.build`` (nvcc, sm_100a). Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libempm_b200.so")

EMPM_OK = 0
ROLLOUT_GRAPH, ROLLOUT_RESUME, ROLLOUT_KEEP = 1, 2, 4
EMPM_ERR_INVALID, EMPM_ERR_CUDA, EMPM_ERR_OOM, EMPM_ERR_UNSUPPORTED = -1, -2, -3, -4
EMPM_MAX_COLLIDERS = 16
EMPM_MAX_MODIFIERS = 8
EMPM_STATUS_NAN, EMPM_STATUS_CFL, EMPM_STATUS_OUT_OF_BAND = 1, 2, 4

COLL_SURFACE, COLL_GEOMETRY, COLL_GRID_VELOCITY, COLL_CUBOID_VELOCITY, COLL_BOUNDING_BOX, COLL_GRID_MASK = 1, 2, 3, 4, 5, 6
SHAPE_CUBE, SHAPE_SPHERE, SHAPE_CYLINDER, SHAPE_HALFSPACE = 1, 2, 3, 4
GATE_OFF, GATE_APPLY, GATE_ZERO_ALL = 0, 1, 2
OPT_SORT_EVERY, OPT_P2G_MODE, OPT_G2P_TILE, OPT_TILE_CAP, OPT_SEG_CAP, OPT_ADJ_STORE = 1, 2, 3, 4, 5, 6
OPT_FUSE = 7
OPT_SEGMENT_GRAPH = 8
MOD_IMPULSE, MOD_IMPULSE_MASK, MOD_SET_VELOCITY, MOD_ROTATION, MOD_MOVER = 1, 2, 3, 4, 5
MOD_SET_VELOCITY_LAYERED = 6

F3 = ctypes.c_float * 3


class EmpmModelParams(ctypes.Structure):
    _fields_ = [
        ("n_grid", ctypes.c_int), ("grid_lim", ctypes.c_float), ("material", ctypes.c_int),
        ("gravity", F3), ("rpic_damping", ctypes.c_float), ("grid_v_damping_scale", ctypes.c_float),
        ("softening", ctypes.c_float), ("hardening", ctypes.c_float), ("xi", ctypes.c_float),
        ("plastic_viscosity", ctypes.c_float), ("alpha", ctypes.c_float),
    ]


class EmpmCollider(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("gate", ctypes.c_int), ("shape", ctypes.c_int), ("surface_type", ctypes.c_int),
        ("point", F3), ("normal", F3), ("size", F3), ("velocity", F3), ("rot_axis", F3),
        ("angular_velocity", ctypes.c_float), ("radius", ctypes.c_float), ("half_height", ctypes.c_float),
        ("friction", ctypes.c_float), ("mask", ctypes.c_void_p),
    ]


class EmpmModifier(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("gate", ctypes.c_int), ("vec", F3), ("point", F3), ("normal", F3),
        ("axis1", F3), ("axis2", F3), ("scale", ctypes.c_float * 2), ("mask", ctypes.c_void_p),
    ]


class EmpmStep(ctypes.Structure):
    _fields_ = [
        ("time", ctypes.c_float), ("dt", ctypes.c_float), ("n_colliders", ctypes.c_int), ("n_modifiers", ctypes.c_int),
        ("hold", ctypes.c_int), ("reserved", ctypes.c_int),
        ("colliders", EmpmCollider * EMPM_MAX_COLLIDERS), ("modifiers", EmpmModifier * EMPM_MAX_MODIFIERS),
    ]


class EmpmParticles(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("v", ctypes.c_void_p), ("C", ctypes.c_void_p), ("F", ctypes.c_void_p)]


class EmpmMaterial(ctypes.Structure):
    _fields_ = [
        ("vol", ctypes.c_void_p), ("mu", ctypes.c_void_p), ("lam", ctypes.c_void_p),
        ("yield_stress", ctypes.c_void_p), ("selection", ctypes.c_void_p), ("F_elastic", ctypes.c_void_p),
    ]


class EmpmMaterialGrad(ctypes.Structure):
    _fields_ = [("mu", ctypes.c_void_p), ("lam", ctypes.c_void_p), ("yield_stress", ctypes.c_void_p),
                ("mass", ctypes.c_void_p)]


class EmpmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"empm error {code}: {message}")
        self.code = code


_lib = None


def lib():
    """Load libempm_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m empm_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback for the MPM substep.")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    I = ctypes.c_int
    sig = {
        "empm_version": ([], I),
        "empm_ctx_create": ([ctypes.POINTER(EmpmModelParams), I, I, ctypes.POINTER(P)], I),
        "empm_ctx_destroy": ([P], I),
        "empm_ctx_set_params": ([P, ctypes.POINTER(EmpmModelParams)], I),
        "empm_prepare": ([P, P, P, P, P, P, P, P, I, P], I),
        "empm_pack_particles": ([P, P, P, P, P, I, ctypes.POINTER(EmpmParticles), I, P], I),
        "empm_unpack_particles": ([ctypes.POINTER(EmpmParticles), P, P, P, P, I, P], I),
        "empm_substep": ([P, ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmParticles),
                          ctypes.POINTER(EmpmMaterial), ctypes.POINTER(EmpmStep), P], I),
        "empm_substep_inplace": ([P, ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmMaterial),
                                  ctypes.POINTER(EmpmStep), P, P], I),
        "empm_rollout": ([P, ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmParticles),
                          ctypes.POINTER(EmpmMaterial), P, I, I, I, P], I),
        "empm_rollout_ex": ([P, ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmParticles),
                          ctypes.POINTER(EmpmMaterial), P, I, I, I, P], I),
        "empm_batch_create": ([P, P, I, I, ctypes.POINTER(P)], I),
        "empm_batch_set_params": ([P, I, ctypes.POINTER(EmpmModelParams)], I),
        "empm_batch_info": ([P, ctypes.POINTER(I), P, P], I),
        "empm_batch_reserve": ([P, I, ctypes.c_longlong, I], I),
        "empm_batch_reconfigure": ([P, P, P, I, P], I),
        "empm_substep_noalloc": ([ctypes.POINTER(EmpmModelParams), ctypes.POINTER(EmpmParticles),
                                  ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmMaterial),
                                  ctypes.POINTER(EmpmStep), I, P, P], I),
        "empm_read_status": ([P, ctypes.POINTER(ctypes.c_uint32), P], I),
        "empm_last_error": ([P, ctypes.c_char_p, I], I),
        "empm_debug_stress": ([ctypes.POINTER(EmpmModelParams), P, P, P, P, ctypes.c_float, P, P, I, P], I),
        "empm_adjoint_segment": ([P, ctypes.POINTER(EmpmParticles), P, P, P, ctypes.POINTER(EmpmMaterial), P, I,
                                  ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmMaterialGrad), P], I),
        "empm_prepare_adjoint": ([P, P, P, P, P, P, P, P, P, I, P], I),
        "empm_segment_bytes": ([P, I, I, ctypes.POINTER(ctypes.c_size_t)], I),
        "empm_segment_create": ([P, I, I, ctypes.POINTER(P)], I),
        "empm_segment_blocks": ([P, ctypes.POINTER(I), ctypes.POINTER(I), P], I),
        "empm_segment_destroy": ([P], I),
        "empm_segment_forward": ([P, P, ctypes.POINTER(EmpmParticles), P, P, P, ctypes.POINTER(EmpmMaterial), P, I,
                                  ctypes.POINTER(EmpmParticles), P], I),
        "empm_segment_reverse": ([P, P, ctypes.POINTER(EmpmParticles), ctypes.POINTER(EmpmMaterialGrad), P], I),
        "empm_chamfer": ([P, P, I, I, P, P, I, I, I, P, P, P, P, P], I),
        "empm_restart_F": ([P, ctypes.POINTER(EmpmParticles), P, P, P, P], I),
        "empm_chamfer_backward": ([P, P, I, P, P, I, I, P, P, P, P, P, P, P], I),
        "empm_debug_stress_adjoint": ([ctypes.POINTER(EmpmModelParams), P, P, P, P, ctypes.c_float, P, P, P, P, P,
                                       P, I, P], I),
        "empm_knn": ([P, I, P, I, I, I, P, I, P, P], I),
        "empm_idw_weights": ([P, I, P, I, P, I, I, P, P, P], I),
        "empm_lbs_bones": ([P, P, I, P, I, I, I, P, P, P, P], I),
        "empm_lbs_blend": ([P, I, P, P, I, P, I, I, P, P, P, P, P, P], I),
        "empm_lbs_blend_dense": ([P, I, P, P, I, P, P, P, P, P], I),
        "empm_rotation_to_quat": ([P, I, I, P, P], I),
        "empm_ctx_grid": ([P, ctypes.POINTER(P), ctypes.POINTER(P)], I),
        "empm_ctx_timing": ([P, I, I], I),
        "empm_ctx_set_option": ([P, I, I], I),
        "empm_ctx_kernel_times": ([P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(I)], I),
        "empm_ctx_adjoint_kernel_times": ([P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(I)], I),
        "empm_ctx_fused_kernel_times": ([P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(I)], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def kernel_times(L, ctx) -> dict:
    """Per-kernel CUDA-event times of a context's stream-path launches:
    {kernel: (total_ms, launches)} for stress_p2g, grid_update, g2p and the
    fused g2p2g."""
    ms = (ctypes.c_float * 3)()
    cnt = (ctypes.c_int * 3)()
    check(L.empm_ctx_kernel_times(ctx, ms, cnt), ctx)
    out = {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("stress_p2g", "grid_update", "g2p"))}
    fms, fcnt = ctypes.c_float(), ctypes.c_int()
    check(L.empm_ctx_fused_kernel_times(ctx, ctypes.byref(fms), ctypes.byref(fcnt)), ctx)
    out["g2p2g"] = (float(fms.value), int(fcnt.value))
    return out


def last_error(ctx=None) -> str:
    buf = ctypes.create_string_buffer(512)
    lib().empm_last_error(ctx, buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int, ctx=None) -> None:
    if rc != EMPM_OK:
        raise EmpmError(rc, last_error(ctx))


def header_symbols():
    """Function names declared in include/empm_b200.h."""
    import re

    path = os.path.join(os.path.dirname(_HERE), "include", "empm_b200.h")
    src = open(path).read()
    return sorted(set(re.findall(r"^\s*int\s+(empm_\w+)\s*\(", src, flags=re.M)))


def grid_dense_index(G: int):
    """Blocked-layout address of every node (i, j, k) of a G^3 grid, as a
    [G, G, G] int64 numpy array (see empm_ctx_grid)."""
    import numpy as np

    nb = (G + 3) // 4
    i, j, k = np.meshgrid(np.arange(G), np.arange(G), np.arange(G), indexing="ij")
    blk = ((i >> 2) * nb + (j >> 2)) * nb + (k >> 2)
    return (blk << 6) | ((i & 3) << 4) | ((j & 3) << 2) | (k & 3)
