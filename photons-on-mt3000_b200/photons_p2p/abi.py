"""ctypes declarations of the C ABI in include/photons_p2p.h."""
import ctypes

P2P_OK = 0
P2P_ERR_ARG = 1
P2P_ERR_CUDA = 2
P2P_ERR_STATE = 3
P2P_ERR_NOMEM = 4
P2P_ERR_RANGE = 5
P2P_ERR_CAPACITY = 6

SOFT_CLAMP = 0
SOFT_PLUMMER = 1

FORM_PLAIN_FP64 = 0
FORM_SPLIT = 1
FORM_NAIVE_FP32 = 2
FORM_KAHAN_FP32 = 3

VARIANT_AUTO = 0
VARIANT_SINK_LANES = 1
VARIANT_SOURCE_LANES = 2
VARIANT_SOURCE_LANES_X2 = 3
VARIANT_SOURCE_LANES_X2_S16 = 4
VARIANT_SINK_LANES_X2 = 5
VARIANT_SINK_REGS = 6
VARIANT_SINK_REGS8 = 7

FORM_NAMES = {
    FORM_PLAIN_FP64: "plain_fp64",
    FORM_SPLIT: "split_fp32_fp64",
    FORM_NAIVE_FP32: "naive_fp32",
    FORM_KAHAN_FP32: "kahan_fp32",
}


class Params(ctypes.Structure):
    _fields_ = [
        ("form", ctypes.c_int),
        ("soft_mode", ctypes.c_int),
        ("soften", ctypes.c_double),
        ("split_radius", ctypes.c_double),
        ("x_cut", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("warps_per_block", ctypes.c_int),
        ("stage_sources", ctypes.c_int),
        ("blocks_per_sm", ctypes.c_int),
        ("kernel_variant", ctypes.c_int),
        ("poly_tol", ctypes.c_double),
        ("warps_per_leaf", ctypes.c_int),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("slots", ctypes.c_int),
        ("max_pack", ctypes.c_int),
        ("full_grid", ctypes.c_int),
        ("hbm_bytes", ctypes.c_size_t),
        ("rows_per_particle", ctypes.c_double),
        ("particles_per_leaf", ctypes.c_double),
        ("batch_window_ms", ctypes.c_double),
        ("min_pack_pairs", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("requests_done", ctypes.c_int64),
        ("launches", ctypes.c_int64),
        ("boxes_launched", ctypes.c_int64),
        ("builds", ctypes.c_int64),
        ("evictions", ctypes.c_int64),
        ("pairs", ctypes.c_int64),
        ("kernel_ms", ctypes.c_double),
        ("build_ms", ctypes.c_double),
        ("resident_boxes", ctypes.c_int),
        ("resident_bytes", ctypes.c_size_t),
        ("capacity_bytes", ctypes.c_size_t),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double

class WalkTree(ctypes.Structure):
    """p2p_walk_tree: the kd-tree in device memory (pointers as integers)."""
    _fields_ = [
        ("nnode", ctypes.c_int),
        ("nleaf", ctypes.c_int),
        ("son", ctypes.c_void_p),
        ("node_first", ctypes.c_void_p),
        ("node_center", ctypes.c_void_p),
        ("node_width", ctypes.c_void_p),
        ("leaf_center", ctypes.c_void_p),
        ("leaf_width", ctypes.c_void_p),
        ("leaf_active", ctypes.c_void_p),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "p2p_params_default": (None, [ctypes.POINTER(Params)]),
    "p2p_status_string": (ctypes.c_char_p, [_i]),
    "p2p_last_error": (ctypes.c_char_p, []),
    "p2p_version": (_i, []),
    "p2p_device_count": (_i, [ctypes.POINTER(_i)]),
    "p2p_session_create": (_i, [_i, ctypes.POINTER(_vp)]),
    "p2p_session_destroy": (_i, [_vp]),
    "p2p_session_set_params": (_i, [_vp, ctypes.POINTER(Params)]),
    "p2p_session_get_params": (_i, [_vp, ctypes.POINTER(Params)]),
    "p2p_session_stream": (_vp, [_vp]),
    "p2p_session_poly_degree": (_i, [_vp]),
    "p2p_session_poly_error": (_d, [_vp]),
    "p2p_pass_begin": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp]),
    "p2p_pass_begin_update": (_i, [_vp, _i, _vp, _i, _vp, _vp, _vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "p2p_pass_begin_device": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp]),
    "p2p_pass_submit": (_i, [_vp, _i64, _vp, _vp]),
    "p2p_pass_submit_device": (_i, [_vp, _i64, _vp, _vp]),
    "p2p_pass_end": (_i, [_vp, ctypes.POINTER(_d)]),
    "p2p_pass_accumulate": (_i, [_vp, _vp]),
    "p2p_pass_result": (_i, [_vp, _vp]),
    "p2p_pass_result_device": (_i, [_vp, ctypes.POINTER(_vp)]),
    "p2p_pass_submit_walk": (_i, [_vp, ctypes.POINTER(WalkTree), _d, _d, ctypes.POINTER(_i64)]),
    "p2p_pass_rows": (_i, [_vp, _vp, _vp]),
    "p2p_session_synchronize": (_i, [_vp]),
    "p2p_pass_pair_count": (_i, [_vp, ctypes.POINTER(_i64)]),
    "p2p_pass_evaluated_pairs": (_i, [_vp, ctypes.POINTER(_i64)]),
    "p2p_pass_run_device": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp, _i64, _vp, _vp]),
    "p2p_kernel_launch_count": (_i64, []),
    "p2p_session_last_kernel_ms": (_i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "p2p_measure_fp32_peak": (_i, [_vp, ctypes.POINTER(_d)]),
    "p2p_measure_fp64_peak": (_i, [_vp, ctypes.POINTER(_d)]),
    "p2p_pass_noalloc": (_i, [ctypes.POINTER(Params), _i, _vp, _i, _vp, _vp, _i64, _vp, _vp, _vp, _vp]),
    "p2p_server_config_default": (None, [ctypes.POINTER(ServerConfig)]),
    "p2p_server_create": (_i, [_i, ctypes.POINTER(Params), ctypes.POINTER(ServerConfig),
                               ctypes.POINTER(_vp)]),
    "p2p_server_destroy": (_i, [_vp]),
    "p2p_server_add_box": (_i, [_vp, _d, _d, _i, _vp, _i, _vp, _vp, _i64, _vp, _vp, _i, _vp,
                                ctypes.POINTER(_i)]),
    "p2p_server_preload": (_i, [_vp, _i]),
    "p2p_server_box_bytes": (_i, [_vp, _i, ctypes.POINTER(ctypes.c_size_t)]),
    "p2p_server_submit": (_i, [_vp, _i, _vp, ctypes.POINTER(_i64)]),
    "p2p_server_wait": (_i, [_vp, _i64, ctypes.POINTER(_d)]),
    "p2p_server_query": (_i, [_vp, _i64, ctypes.POINTER(_i), ctypes.POINTER(_d)]),
    "p2p_server_drain": (_i, [_vp]),
    "p2p_server_set_batching": (_i, [_vp, _d, _d]),
    "p2p_server_get_stats": (_i, [_vp, ctypes.POINTER(ServerStats)]),
    "p2p_dtree_build": (_i, [_vp, _i, _vp, _vp, _i, _d, ctypes.POINTER(_vp)]),
    "p2p_dtree_free": (_i, [_vp]),
    "p2p_dtree_rebuild": (_i, [_vp, _vp, _i, _vp, _vp, _i, _d]),
    "p2p_dtree_counts": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                              ctypes.POINTER(ctypes.c_float)]),
    "p2p_dtree_device_arrays": (_i, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                     ctypes.POINTER(_vp)]),
    "p2p_dtree_walk_tree": (_i, [_vp, ctypes.POINTER(WalkTree)]),
    "p2p_dtree_download": (_i, [_vp] + [_vp] * 11),
    "p2p_dtree_unpermute": (_i, [_vp, _vp, _vp, _vp]),
    "p2p_fmm_create": (_i, [_vp, ctypes.POINTER(_vp)]),
    "p2p_fmm_destroy": (_i, [_vp]),
    "p2p_fmm_far": (_i, [_vp, ctypes.POINTER(WalkTree), _i, _vp, _vp, _vp] + [_d] * 5 + [_vp]),
    "p2p_fmm_stats": (_i, [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                           ctypes.POINTER(_i), ctypes.POINTER(ctypes.c_float)]),
    "p2p_fmm_download": (_i, [_vp, _vp, _vp]),
    "p2p_pm_create": (_i, [_vp, _i, _d, _d, ctypes.POINTER(_vp)]),
    "p2p_pm_destroy": (_i, [_vp]),
    "p2p_pm_forces": (_i, [_vp, _i, _vp, _vp, _d, _vp]),
    "p2p_pm_timings": (_i, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "p2p_pm_download": (_i, [_vp, _vp, _vp]),
    "p2p_host_alloc": (_i, [ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "p2p_host_free": (_i, [_vp]),
}


def declare(lib):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def header_symbols(header_path):
    """Function names declared in a C header (for the export test)."""
    import re

    text = open(header_path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
    names = re.findall(r"\b([a-zA-Z_][a-zA-Z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "sizeof")))
