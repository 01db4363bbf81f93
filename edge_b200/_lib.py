"""ctypes bindings of ``libedge_b200.so`` (the C ABI of include/edge_b200.h)."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libedge_b200.so")

_lib = None

vp = C.c_void_p
i32, i64, u64, dbl = C.c_int32, C.c_int64, C.c_uint64, C.c_double


class Cfg(C.Structure):
    _fields_ = [("order", C.c_int), ("n_runs", C.c_int), ("n_rms", C.c_int),
                ("precision", C.c_int), ("stream", vp), ("device", C.c_int)]


_SIGS = {
    "edge_mesh_box": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, dbl, u64, C.c_int, C.c_int, vp]),
    "edge_mesh_from_arrays": (C.c_int, [i64, vp, i64, vp, i64, vp, vp, C.c_int, C.c_int, vp, vp]),
    "edge_mesh_sizes": (C.c_int, [vp, vp, vp, vp]),
    "edge_mesh_arrays": (C.c_int, [vp] * 15),
    "edge_mesh_free": (None, [vp]),
    "edge_setup_star": (C.c_int, [vp] * 5),
    "edge_setup_star_anelastic": (C.c_int, [vp, vp]),
    "edge_setup_flux_solvers": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp]),
    "edge_setup_frequencies": (C.c_int, [C.c_int, dbl, dbl, vp]),
    "edge_setup_attenuation": (C.c_int, [C.c_int, dbl, dbl, i64, vp, vp, vp, vp, vp, vp]),
    "edge_setup_anelastic_coeffs": (C.c_int, [C.c_int, dbl, vp, vp]),
    "edge_setup_elastic_lame": (C.c_int, [C.c_int, dbl, vp, vp, vp, dbl, dbl, vp, vp]),
    "edge_setup_dt_cfl": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "edge_setup_dt_cfl_el": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "edge_setup_time_groups": (C.c_int, [vp, vp, C.c_int, dbl, vp, vp]),
    "edge_setup_locate": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_int]),
    "edge_setup_eval_basis": (C.c_int, [C.c_int, vp, vp]),
    "edge_setup_trafo": (C.c_int, [vp] * 5),
    "edge_setup_fs_pair": (C.c_int, [dbl] * 6 + [vp, vp, vp, C.c_int, vp, vp, vp, vp]),
    "edge_b200_create": (C.c_int, [vp, i64, vp]),
    "edge_b200_kernel_config": (C.c_int, [vp, vp]),
    "edge_b200_set_fused": (C.c_int, [vp, C.c_int]),
    "edge_b200_batch_create": (C.c_int, [vp, C.c_int, vp, vp, vp]),
    "edge_b200_batch_set_active": (C.c_int, [vp, vp]),
    "edge_b200_batch_step": (C.c_int, [vp, C.c_int]),
    "edge_b200_batch_sync": (C.c_int, [vp, vp]),
    "edge_b200_batch_last_error": (C.c_char_p, [vp]),
    "edge_b200_batch_destroy": (C.c_int, [vp]),
    "edge_b200_autotune": (C.c_int, [vp, dbl, vp]),
    "edge_b200_destroy": (C.c_int, [vp]),
    "edge_b200_upload_mesh": (C.c_int, [vp] * 5),
    "edge_b200_upload_element_data": (C.c_int, [vp] * 7),
    "edge_b200_upload_dofs": (C.c_int, [vp] * 3),
    "edge_b200_download_dofs": (C.c_int, [vp] * 3),
    "edge_b200_download_tdofs": (C.c_int, [vp] * 2),
    "edge_b200_upload_dofs_async": (C.c_int, [vp] * 3),
    "edge_b200_download_dofs_async": (C.c_int, [vp] * 3),
    "edge_b200_join_transfers": (C.c_int, [vp, C.c_int]),
    "edge_b200_keep_tdofs": (C.c_int, [vp, C.c_int]),
    "edge_b200_set_run_dofs": (C.c_int, [vp, C.c_int, vp, vp]),
    "edge_b200_copy_run": (C.c_int, [vp, C.c_int, vp, C.c_int]),
    "edge_b200_share_element_data": (C.c_int, [vp, vp]),
    "edge_b200_rewind_receivers": (C.c_int, [vp, dbl]),
    "edge_b200_set_sources": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]),
    "edge_b200_set_receivers": (C.c_int, [vp, C.c_int, vp, vp, dbl, dbl, C.c_int]),
    "edge_b200_step": (C.c_int, [vp, dbl, dbl, C.c_int]),
    "edge_b200_upload_geometry": (C.c_int, [vp, vp]),
    "edge_b200_wavefield": (C.c_int, [vp, vp]),
    "edge_b200_error_norms": (C.c_int, [vp, dbl, C.c_int, vp, C.c_int, vp, vp, vp, vp, vp, vp]),
    "edge_b200_set_owned": (C.c_int, [vp, i64]),
    "edge_b200_set_group_dt": (C.c_int, [vp, vp]),
    "edge_b200_set_source_clocks": (C.c_int, [vp, vp, vp]),
    "edge_b200_set_active_elements": (C.c_int, [vp, i64]),
    "edge_b200_set_send_count": (C.c_int, [vp, i64]),
    "edge_b200_step_phase": (C.c_int, [vp, dbl, dbl, C.c_int]),
    "edge_b200_face_block_bytes": (i64, [vp]),
    "edge_b200_pack_faces": (C.c_int, [vp, C.c_int, vp, vp]),
    "edge_b200_unpack_faces": (C.c_int, [vp, C.c_int, vp, vp]),
    "edge_b200_set_time_groups": (C.c_int, [vp, C.c_int, vp]),
    "edge_b200_step_lts": (C.c_int, [vp, dbl, dbl, C.c_int]),
    "edge_b200_read_receivers": (C.c_int, [vp, vp, vp, vp]),
    "edge_b200_sync": (C.c_int, [vp]),
    "edge_b200_device_dofs": (C.c_int, [vp, vp, vp, vp]),
    "edge_b200_last_launches": (i64, [vp]),
    "edge_b200_last_error": (C.c_char_p, [vp]),
    "edge_b200_set_timing": (C.c_int, [vp, C.c_int]),
    "edge_b200_kernel_times": (C.c_int, [vp, vp, vp]),
    "edge_b200_step_noalloc": (C.c_int, [vp, i64, dbl, C.c_int] + [vp] * 12),
}

# every symbol include/edge_b200.h declares
EXPORTED = tuple(_SIGS)


def lib():
    """Loads the in-tree library; fails loudly when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `python -m edge_b200.build` (or "
                               "__graft_entry__.build()) first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    """Raw data pointer of a numpy array (None passes NULL)."""
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)


def check(rc, what=""):
    if rc != 0:
        names = {-1: "EINVAL", -2: "ENOMEM", -3: "EDEVICE", -4: "ETIMEOUT", -5: "ENOTSUP",
                 -6: "EMESH", -7: "ENOTFOUND", -8: "EOVERFLOW"}
        raise RuntimeError(f"{what} failed: {names.get(rc, rc)}")
    return rc
