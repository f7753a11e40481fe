"""ctypes declarations of the C ABI (include/cuplast.h, include/cuplast_host.h).

The library is the in-tree build cudaplasticity_b200/libcuplast.so. There is no
fallback: importing this module fails loudly when the library is missing.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcuplast.so")

CP_OK = 0
CP_ERR_INVALID = 1
CP_ERR_CUDA = 2
CP_ERR_NOMEM = 3
CP_ERR_NOT_CONVERGED = 4
CP_ERR_BREAKDOWN = 5
CP_ERR_MESH = 6
CP_ERR_UNSUPPORTED = 7
CP_ERR_BUSY = 8
CP_ERR_NO_DEVICE = 9
CP_ERR_CANCELLED = 10
CP_ERR_TIMEOUT = 11

CP_PLANE_STRESS, CP_PLANE_STRAIN = 0, 1
CP_DIAGRAM_ELASTIC, CP_DIAGRAM_LINEAR, CP_DIAGRAM_POWER, CP_DIAGRAM_HOLLOMON, CP_DIAGRAM_PIECEWISE = range(5)
CP_PREC_FP64, CP_PREC_MIXED, CP_PREC_FLOAT_BOOST = 0, 1, 2
CP_MAX_PW = 16

c_int, c_double, c_ll, c_p = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
P_int = ctypes.POINTER(ctypes.c_int)
P_double = ctypes.POINTER(ctypes.c_double)
P_ubyte = ctypes.POINTER(ctypes.c_ubyte)
P_ll = ctypes.POINTER(ctypes.c_longlong)


class cp_material(ctypes.Structure):
    _fields_ = [("E", c_double), ("nu", c_double), ("h", c_double), ("rho", c_double), ("plane", c_int),
                ("diagram", c_int), ("sigma_t", c_double), ("k_t", c_double), ("a", c_double), ("m", c_double),
                ("eps0", c_double), ("n", c_double), ("n_points", c_int), ("pw_eps", c_double * CP_MAX_PW),
                ("pw_sig", c_double * CP_MAX_PW)]


class cp_mesh_view(ctypes.Structure):
    _fields_ = [("node_count", c_int), ("node_xy", P_double), ("count3", c_int), ("elem3", P_int),
                ("count4", c_int), ("elem4", P_int), ("count8", c_int), ("elem8", P_int)]


class cp_solve_opts(ctypes.Structure):
    _fields_ = [("precision", c_int), ("cg_tol", c_double), ("outer_tol", c_double), ("max_outer", c_int),
                ("max_cg", c_ll), ("levels", c_int), ("aitken", c_int), ("inner_tol", c_double),
                ("adaptive_cg", c_int), ("precond", c_int), ("predict", c_int), ("recycle", c_int)]


class cp_solve_report(ctypes.Structure):
    _fields_ = [("status", c_int), ("outer_iters", c_int), ("cg_iters", c_ll), ("fp64_spmv", c_ll),
                ("rel_err", c_double), ("cg_rel_res", c_double), ("seconds", c_double), ("levels_done", c_int),
                ("kernel_launches", c_ll)]


class cp_batch_opts(ctypes.Structure):
    _fields_ = [("max_instances", c_int), ("cg_per_trip", c_int), ("elem_per_trip", c_int), ("max_width", c_int),
                ("cg_blocks_per_sm", c_int)]


CP_BATCH_RUN_ALL, CP_BATCH_RUN_ANY_DONE = 0, 1


class cp_server_opts(ctypes.Structure):
    _fields_ = [("device", c_int), ("hbm_reserve", c_double), ("max_bytes", ctypes.c_size_t),
                ("max_inflight", c_int), ("trip_quantum", c_ll), ("batch", cp_batch_opts), ("fp64_lanes", c_int)]


class cp_server_stats(ctypes.Structure):
    _fields_ = [("submitted", c_ll), ("admitted", c_ll), ("completed", c_ll), ("failed", c_ll), ("rejected", c_ll),
                ("inflight", c_ll), ("pending", c_ll), ("runs", c_ll), ("trips", c_ll), ("busy_seconds", c_double),
                ("peak_bytes", ctypes.c_size_t)]

# name -> (restype, argtypes)
_SIGS = {
    "cp_version": (ctypes.c_char_p, []),
    "cp_status_string": (ctypes.c_char_p, [c_int]),
    "cp_device_count": (c_int, [P_int]),
    "cp_context_create": (c_int, [c_int, ctypes.POINTER(c_p)]),
    "cp_context_destroy": (c_int, [c_p]),
    "cp_context_last_error": (ctypes.c_char_p, [c_p]),
    "cp_instance_last_error": (ctypes.c_char_p, [c_p]),
    "cp_context_synchronize": (c_int, [c_p]),
    "cp_instance_create": (c_int, [c_p, ctypes.POINTER(cp_mesh_view), ctypes.POINTER(cp_material),
                                   ctypes.POINTER(c_p)]),
    "cp_instance_destroy": (c_int, [c_p]),
    "cp_instance_footprint": (c_int, [ctypes.POINTER(cp_mesh_view), c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "cp_instance_sizes": (c_int, [c_p, P_int, P_int, P_ll, P_ll]),
    "cp_instance_set_loads": (c_int, [c_p, P_double, P_ubyte, P_double]),
    "cp_instance_reset_state": (c_int, [c_p]),
    "cp_instance_set_level": (c_int, [c_p, c_double]),
    "cp_assemble": (c_int, [c_p, c_int]),
    "cp_cg_solve": (c_int, [c_p, c_double, c_ll, P_ll, P_double]),
    "cp_secant_update": (c_int, [c_p, P_double]),
    "cp_plastic_strains": (c_int, [c_p]),
    "cp_solve_opts_default": (None, [ctypes.POINTER(cp_solve_opts)]),
    "cp_solve": (c_int, [c_p, ctypes.POINTER(cp_solve_opts), ctypes.POINTER(cp_solve_report)]),
    "cp_bench_cg": (c_int, [c_p, c_int, c_int, c_int, P_double, P_double, P_double, P_double]),
    "cp_secant_update_noalloc": (c_int, [c_p, ctypes.POINTER(cp_material), c_int, c_p, c_int, c_p, c_p, c_p, c_p,
                                         c_p, c_p, P_double]),
    "cp_batch_opts_default": (None, [ctypes.POINTER(cp_batch_opts)]),
    "cp_batch_create": (c_int, [c_p, ctypes.POINTER(cp_batch_opts), ctypes.POINTER(c_p)]),
    "cp_batch_destroy": (c_int, [c_p]),
    "cp_batch_add": (c_int, [c_p, c_p, ctypes.POINTER(cp_solve_opts), P_int]),
    "cp_batch_launch": (c_int, [c_p, c_int, c_ll]),
    "cp_batch_wait": (c_int, [c_p, P_int, P_int]),
    "cp_batch_interrupt": (c_int, [c_p]),
    "cp_batch_run": (c_int, [c_p, c_int, c_ll, P_int, P_int]),
    "cp_batch_harvest": (c_int, [c_p, c_int, P_int, ctypes.POINTER(c_p), ctypes.POINTER(cp_solve_report), P_int]),
    "cp_batch_set_tile": (c_int, [c_p, c_int, c_int]),
    "cp_batch_get_tile": (c_int, [c_p, c_int, P_int]),
    "cp_batch_autotune": (c_int, [c_p, P_double]),
    "cp_batch_stats": (c_int, [c_p, P_ll, P_ll, P_ll]),
    "cp_batch_last_run_ms": (c_int, [c_p, P_double]),
    "cp_batch_progress": (c_int, [c_p, c_int, P_int, P_int, ctypes.POINTER(cp_solve_report)]),
    "cp_server_opts_default": (None, [ctypes.POINTER(cp_server_opts)]),
    "cp_server_create": (c_int, [ctypes.POINTER(cp_server_opts), ctypes.POINTER(c_p)]),
    "cp_server_destroy": (c_int, [c_p]),
    "cp_server_submit": (c_int, [c_p, ctypes.POINTER(cp_mesh_view), ctypes.POINTER(cp_material), P_double, P_ubyte,
                                 P_double, ctypes.POINTER(cp_solve_opts), P_ll]),
    "cp_server_wait": (c_int, [c_p, c_ll, c_double, ctypes.POINTER(c_p), ctypes.POINTER(cp_solve_report),
                               P_double]),
    "cp_server_get_stats": (c_int, [c_p, ctypes.POINTER(cp_server_stats)]),
    "cp_get_csr": (c_int, [c_p, P_int, P_int, P_int, P_int, P_double]),
    "cp_get_slot_map": (c_int, [c_p, P_int]),
    "cp_get_field": (c_int, [c_p, ctypes.c_char_p, P_double]),
    "cp_set_field": (c_int, [c_p, ctypes.c_char_p, P_double]),
    # host helpers
    "cpx_mesh_create": (c_int, [ctypes.POINTER(c_p)]),
    "cpx_mesh_destroy": (c_int, [c_p]),
    "cpx_mesh_gen_rect": (c_int, [c_p, c_double, c_double, c_double, c_double, c_int, c_int, c_int]),
    "cpx_mesh_gen_rect_with_hole": (c_int, [c_p, c_double, c_double, c_double, c_double, c_double, c_int, c_int,
                                            c_int, c_int]),
    "cpx_mesh_gen_ring": (c_int, [c_p, c_double, c_double, c_int, c_int, c_int]),
    "cpx_mesh_split_t3": (c_int, [c_p]),
    "cpx_mesh_load_inp": (c_int, [c_p, ctypes.c_char_p]),
    "cp_bench_assemble": (c_int, [c_p, c_int, c_int, P_double, P_double]),
    "cp_bench_cg_fused": (c_int, [c_p, c_int, c_int, P_double, P_double]),
    "cp_bench_mg": (c_int, [c_p, c_int, P_double, P_double]),
    "cpx_mesh_renum_by_direction": (c_int, [c_p, c_double, c_double]),
    "cpx_mesh_smooth_ring": (c_int, [c_p, c_int]),
    "cpx_mesh_quality": (c_int, [c_p, P_double, P_double, P_double]),
    "cpx_mesh_set": (c_int, [c_p, c_int, P_double, c_int, P_int, c_int, P_int, c_int, P_int, P_int, c_int, P_int]),
    "cpx_mesh_counts": (c_int, [c_p, P_int, P_int, P_int, P_int, P_int, P_int]),
    "cpx_mesh_get": (c_int, [c_p, P_double, P_int, P_int, P_int, P_int, P_int]),
    "cpx_mesh_max_index_diff": (c_int, [c_p, P_int]),
    "cpx_loads_create": (c_int, [ctypes.POINTER(c_p)]),
    "cpx_loads_destroy": (c_int, [c_p]),
    "cpx_loads_set_force": (c_int, [c_p, c_int, c_double, c_double, c_int]),
    "cpx_loads_set_displacement": (c_int, [c_p, c_int, c_double, c_double, c_int, c_int]),
    "cpx_loads_fix_border": (c_int, [c_p, c_int]),
    "cpx_loads_fix_border_vert": (c_int, [c_p, c_int]),
    "cpx_loads_fix_border_hor": (c_int, [c_p, c_int]),
    "cpx_loads_fix_vert_axis": (c_int, [c_p, c_double]),
    "cpx_loads_fix_hor_axis": (c_int, [c_p, c_double]),
    "cpx_loads_fix_point": (c_int, [c_p, c_double, c_double]),
    "cpx_loads_set_displ_point": (c_int, [c_p, c_double, c_double, c_double, c_double]),
    "cpx_loads_set_force_point": (c_int, [c_p, c_double, c_double, c_double, c_double]),
    "cpx_loads_set_gravity": (c_int, [c_p, c_double, c_double, c_double]),
    "cpx_loads_set_rotation": (c_int, [c_p, c_double, c_double, c_double]),
    "cpx_loads_fix_dof": (c_int, [c_p, c_int]),
    "cpx_loads_build": (c_int, [c_p, c_p, c_double, c_double, P_double, P_ubyte, P_double]),
    "cpx_amg_build": (c_int, [c_int, P_int, P_int, P_double, P_ubyte, c_int, c_int, ctypes.POINTER(c_p)]),
    "cpx_amg_level_parts": (c_int, [c_p, c_int, P_int, P_int]),
    "cpx_amg_destroy": (c_int, [c_p]),
    "cpx_amg_levels": (c_int, [c_p, P_int]),
    "cpx_amg_level_sizes": (c_int, [c_p, c_int, P_int, P_int, P_int, P_int]),
    "cpx_amg_level_get": (c_int, [c_p, c_int, P_int, P_int, P_int, P_double]),
    "cpx_amg_galerkin": (c_int, [c_p, c_int, P_double, P_double]),
    "cpx_amg_device_maps": (c_int, [c_p, c_int, P_int, P_int, P_int, P_int, P_int, P_int, P_int, P_int]),
    "cpx_recycle_solve": (c_int, [P_double, c_int, P_double]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cudaplasticity_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGS)
