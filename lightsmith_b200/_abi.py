"""ctypes binding of the C ABI in ``include/lsfdtd.h`` (``liblsfdtd.so``, built in-tree by ``build.py``).

The structures mirror the header field by field. Loading fails loudly when the library is missing: there is
no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblsfdtd.so")

F32, F64 = 0, 1
OK, EINVAL, ECUDA, EUNSUPPORTED, ERANGE, ETIMEOUT, ENONFINITE = 0, 1, 2, 3, 4, 5, 6
MAX_MEDIA, MAX_POLES = 4, 6
ABI_VERSION = 2

vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64
f64 = C.c_double


class GridDesc(C.Structure):
    _fields_ = [("shape", i32 * 3), ("precision", i32), ("is_complex", i32), ("periodic", i32 * 3),
                ("spacing", f64 * 3), ("dt", f64), ("bloch", f64 * 3), ("dft_stride", i32),
                ("E", vp), ("H", vp), ("cbE", vp * 3), ("step", vp), ("energy", vp), ("E_alt", vp), ("H_alt", vp),
                ("mirror", i32 * 3)]


class OffdiagDesc(C.Structure):
    _fields_ = [("e", vp), ("h", vp), ("w", vp), ("n", i64), ("width", i32)]


class TensorDesc(C.Structure):
    _fields_ = [("idx", vp), ("n_nodes", i64), ("vn", vp), ("scale", vp), ("normal", vp), ("n_vert", i64),
                ("t_pos", vp), ("t_v", vp), ("t_vc", vp), ("t_g", vp), ("t_nc", vp), ("t_conj", vp), ("frac", vp),
                ("n_tslots", i64), ("p_pos", vp), ("p_node", vp), ("p_medium", vp), ("n_pslots", i64),
                ("n_media", i32), ("n_poles", i32 * MAX_MEDIA), ("eps_inf", f64 * MAX_MEDIA),
                ("c1", (f64 * MAX_POLES) * MAX_MEDIA), ("c2", (f64 * MAX_POLES) * MAX_MEDIA),
                ("c3", (f64 * MAX_POLES) * MAX_MEDIA), ("state", vp)]


class PmlDesc(C.Structure):
    _fields_ = [("axis", i32), ("cells_lo", i32), ("cells_hi", i32), ("b", vp * 2), ("c", vp * 2), ("k", vp * 2),
                ("psi", ((vp * 2) * 3) * 2), ("psi_alt", (vp * 2) * 3)]


class GroupDesc(C.Structure):
    _fields_ = [("n", i64), ("idx", vp), ("mixed", i32), ("has_h", i32), ("has_a", i32), ("n_media", i32),
                ("n_poles", i32 * MAX_MEDIA), ("c1", (f64 * MAX_POLES) * MAX_MEDIA),
                ("c2", (f64 * MAX_POLES) * MAX_MEDIA), ("c3", (f64 * MAX_POLES) * MAX_MEDIA),
                ("inv_eps_inf", f64 * MAX_MEDIA), ("h0", vp), ("inv_a", vp), ("w", vp), ("frac", vp), ("state", vp)]


class Csr(C.Structure):
    _fields_ = [("n_nodes", i64), ("nodes", vp), ("offsets", vp), ("n_entries", i64)]


class TableSourceDesc(C.Structure):
    _fields_ = [("table", vp), ("table_len", i64), ("inc_table", vp), ("inc_len", i64), ("m", i32), ("cmax", i64),
                ("pts", Csr * 2), ("base", vp * 2), ("i0", vp * 2), ("u0", vp * 2), ("coef", vp * 2),
                ("inc_base", vp), ("inc_i0", vp), ("inc_u0", vp), ("view", vp)]


class DipoleDesc(C.Structure):
    _fields_ = [("n", i32), ("idx", vp), ("coef", vp), ("wave", vp), ("wave_len", i64)]


class LineSourceDesc(C.Structure):
    _fields_ = [("M", i32), ("m_src", i32), ("ca", vp), ("cb", vp), ("da", vp), ("db", vp), ("wave", vp),
                ("wave_len", i64), ("E_line", vp), ("H_line", vp), ("pts", Csr * 2), ("i0", vp * 2), ("w", vp * 2),
                ("coef", vp * 2)]


class ColumnSourceDesc(C.Structure):
    _fields_ = [("column", vp), ("k_src", i32), ("k_launch", i32), ("phase", vp), ("amp", (f64 * 2) * 2),
                ("wave", vp), ("wave_len", i64), ("cE", f64), ("cH", f64)]


class ModeSourceDesc(C.Structure):
    _fields_ = [("n_h", i32), ("r_e", i32), ("h_idx", vp), ("mH", vp), ("tab_E", vp), ("len_E", i64),
                ("n_e", i32), ("r_h", i32), ("e_idx", vp), ("mE", vp), ("tab_H", vp), ("len_H", i64)]


class MonitorDesc(C.Structure):
    _fields_ = [("n_freq", i32), ("omega", vp), ("n_e", i64), ("e_idx", vp), ("n_h", i64), ("h_idx1", vp),
                ("h_idx2", vp), ("acc_e", vp), ("acc_h", vp), ("energy", i32), ("space", i32), ("E_src", vp),
                ("H_src", vp)]


# every exported symbol of include/lsfdtd.h with its ctypes signature
class AdjointDesc(C.Structure):
    # psi_bar: C's [buffer][E, H][axis][component][side], flat: (((b * 2 + f) * 3 + d) * 3 + c) * 2 + side
    _fields_ = [("Eb", vp), ("Hb", vp), ("psi_bar", vp * 72), ("box_lo", i32 * 3), ("box_hi", i32 * 3),
                ("hist", vp), ("hist_slots", i32), ("grad", vp), ("e_idx", vp), ("ge", vp), ("n_e", i64),
                ("h_idx1", vp), ("h_idx2", vp), ("gh", vp), ("n_h", i64), ("omega", vp), ("n_freq", i32),
                ("n_groups", i32), ("group_bar", vp * 8), ("od_h", vp), ("od_ptr", vp), ("od_e", vp), ("od_w", vp),
                ("od_rows", i64), ("tm_bar", vp), ("tm_work", vp), ("tm_vs_ptr", vp), ("tm_vs_idx", vp),
                ("tm_nd_ptr", vp), ("tm_nd_src", vp), ("inj_e_tgt", vp), ("inj_e_ptr", vp), ("inj_e_src", vp),
                ("inj_n_e", i64), ("inj_h_tgt", vp), ("inj_h_ptr", vp), ("inj_h_src", vp), ("inj_n_h", i64),
                ("inj_work", vp)]


# the GPU voxeliser's descriptors (lsfdtd_vox_* in include/lsfdtd.h)
VOX_MAX_REGIONS = 8
VOX_MAX_MEDIA = 16


class VoxParticle(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_regions", C.c_int32), ("pos", C.c_double * 3), ("a", C.c_double),
                ("b", C.c_double), ("radii", C.c_double * VOX_MAX_REGIONS), ("slot", C.c_int32 * VOX_MAX_REGIONS)]


class VoxScene(C.Structure):
    _fields_ = [("n_particles", C.c_int32), ("particles", C.c_void_p), ("has_substrate", C.c_int32),
                ("z_int", C.c_double), ("sub_slot", C.c_int32), ("origin", C.c_double * 3), ("dx", C.c_double * 3),
                ("shape", C.c_int32 * 3), ("roi_lo", C.c_int32 * 3), ("roi_hi", C.c_int32 * 3)]


class VoxMedia(C.Structure):
    _fields_ = [("n", C.c_int32), ("samples", C.c_int32), ("mode", C.c_int32), ("eps_inf", C.c_double * VOX_MAX_MEDIA),
                ("dispersive", C.c_int8 * VOX_MAX_MEDIA), ("background", C.c_int8 * VOX_MAX_MEDIA)]


class VoxCells(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("frac", "nhat", "w", "part", "has_disp", "inv", "od")]


SIGNATURES = {
    "lsfdtd_abi_version": (i32, []),
    "lsfdtd_last_error": (C.c_char_p, []),
    "lsfdtd_cpml_slab": (i32, [C.POINTER(i32), C.POINTER(i32), i32, i32, i32, i32, i32, i32, C.POINTER(i32),
                               C.POINTER(i32)]),
    "lsfdtd_group_state_len": (i64, [i32, i32, C.POINTER(i32)]),
    "lsfdtd_engine_create": (i32, [C.POINTER(GridDesc), C.POINTER(vp)]),
    "lsfdtd_engine_destroy": (i32, [vp]),
    "lsfdtd_engine_set_pml": (i32, [vp, C.POINTER(PmlDesc)]),
    "lsfdtd_engine_add_group": (i32, [vp, C.POINTER(GroupDesc)]),
    "lsfdtd_engine_add_offdiag": (i32, [vp, C.POINTER(OffdiagDesc)]),
    "lsfdtd_engine_add_tensor": (i32, [vp, C.POINTER(TensorDesc)]),
    "lsfdtd_tensor_state_len": (i64, [i64, i64, i64, i64, i32, C.POINTER(i32)]),
    "lsfdtd_engine_add_table_source": (i32, [vp, C.POINTER(TableSourceDesc)]),
    "lsfdtd_engine_add_dipole": (i32, [vp, C.POINTER(DipoleDesc)]),
    "lsfdtd_engine_add_line_source": (i32, [vp, C.POINTER(LineSourceDesc)]),
    "lsfdtd_engine_add_column_source": (i32, [vp, C.POINTER(ColumnSourceDesc)]),
    "lsfdtd_engine_add_mode_source": (i32, [vp, C.POINTER(ModeSourceDesc)]),
    "lsfdtd_engine_add_monitor": (i32, [vp, C.POINTER(MonitorDesc)]),
    "lsfdtd_engine_scratch_bytes": (i32, [vp, C.POINTER(C.c_size_t)]),
    "lsfdtd_engine_set_scratch": (i32, [vp, vp, C.c_size_t]),
    "lsfdtd_engine_step": (i32, [vp, i32, vp]),
    "lsfdtd_engine_sample": (i32, [vp, vp]),
    "lsfdtd_engine_chunk": (i32, [vp, i32, i32, vp]),
    "lsfdtd_engine_chunk_timed": (i32, [vp, i32, vp, C.POINTER(f64), C.POINTER(i64)]),
    "lsfdtd_engine_buffer": (i32, [vp]),
    "lsfdtd_engine_status": (i32, [vp, vp, C.POINTER(i32)]),
    "lsfdtd_engine_clear_status": (i32, [vp, vp]),
    "lsfdtd_batch_create_shaped": (i32, [vp, i32, vp, i32, i32, vp]),
    "lsfdtd_engine_set_table_boxes": (i32, [vp, i32, i32, vp, vp, i64, vp]),
    "lsfdtd_engine_set_wait_budget": (i32, [vp, C.c_int64]),
    "lsfdtd_engine_set_clean_split": (i32, [vp, i32]),
    "lsfdtd_engine_set_copy_engine": (i32, [vp, i32]),
    "lsfdtd_engine_uses_tma": (i32, [vp]),
    "lsfdtd_engine_fused": (i32, [vp]),
    "lsfdtd_engine_set_tuning": (i32, [vp, i32, i32, i32, i32]),
    "lsfdtd_engine_steps": (i64, [vp]),
    "lsfdtd_engine_launches_per_chunk": (i64, [vp]),
    "lsfdtd_dft_sample_noalloc": (i32, [C.POINTER(MonitorDesc), i32, i32, vp, f64, vp, vp]),
    "lsfdtd_batch_create": (i32, [C.POINTER(vp), i32, C.POINTER(i64), C.POINTER(vp)]),
    "lsfdtd_batch_destroy": (i32, [vp]),
    "lsfdtd_batch_scratch_bytes": (i32, [vp, C.POINTER(C.c_size_t)]),
    "lsfdtd_batch_set_scratch": (i32, [vp, vp, C.c_size_t]),
    "lsfdtd_batch_run": (i32, [vp, i32, i32, i32, vp]),
    "lsfdtd_batch_ctas": (i32, [vp]),
    "lsfdtd_engine_set_steps": (i32, [vp, i64]),
    "lsfdtd_adjoint_create": (i32, [vp, C.POINTER(AdjointDesc), C.POINTER(vp)]),
    "lsfdtd_adjoint_destroy": (i32, [vp]),
    "lsfdtd_adjoint_record": (i32, [vp, i32, vp]),
    "lsfdtd_adjoint_step": (i32, [vp, i64, i32, vp]),
    "lsfdtd_vox_lattice": (i32, [vp, vp, vp]),
    "lsfdtd_vox_classify": (i32, [vp, vp, i32, i32, vp, vp]),
    "lsfdtd_vox_supersample": (i32, [vp, vp, i32, vp, i64, VoxCells, vp]),
}

_lib = None


class LsfdtdError(RuntimeError):
    pass


def lib():
    """The loaded library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"lightsmith-b200: {LIB_PATH} is missing; build it with "
                              "`python -c 'import lightsmith_b200.build as b; b.build()'` (needs nvcc)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.lsfdtd_abi_version() != ABI_VERSION:
            raise ImportError(f"{LIB_PATH} has ABI {L.lsfdtd_abi_version()}, this binding expects {ABI_VERSION}; "
                              "rebuild it")
        _lib = L
    return _lib


def check(code: int, what: str) -> None:
    if code != OK:
        msg = lib().lsfdtd_last_error().decode(errors="replace")
        raise LsfdtdError(f"{what} failed (code {code}): {msg}")
