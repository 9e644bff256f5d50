"""ctypes loaders for the package's native libraries.

The CUDA library is required: there is no CPU fallback for the P2P pass, and
loading fails loudly when libphotons_p2p.so has not been built.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}

_i32p = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


def lib_path(name):
    return os.path.join(_HERE, name)


def _load(name):
    if name in _libs:
        return _libs[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{name} is not built ({path}); run `python photons-on-mt3000_b200/build.py`")
    lib = ctypes.CDLL(path)
    _libs[name] = lib
    return lib


def lists():
    lib = _load("libphotons_lists.so")
    if not getattr(lib, "_typed", False):
        lib.p2p_make_ghosts.restype = ctypes.c_int64
        lib.p2p_make_ghosts.argtypes = [ctypes.c_int, _f64p, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _f64p, ctypes.c_int64, _i32p]
        lib.p2p_tree_build.restype = _vp
        lib.p2p_tree_build.argtypes = [ctypes.c_int, _f64p, _i32p, ctypes.c_int, ctypes.c_double,
                                       _i32p]
        lib.p2p_tree_free.argtypes = [_vp]
        lib.p2p_tree_nleaf.argtypes = [_vp]
        lib.p2p_tree_nleaf.restype = ctypes.c_int
        lib.p2p_tree_nnode.argtypes = [_vp]
        lib.p2p_tree_nnode.restype = ctypes.c_int
        lib.p2p_tree_leaves.argtypes = [_vp, _i32p, _i32p, _i32p, _f64p, _f64p]
        lib.p2p_tree_nodes.argtypes = [_vp, _i32p, _i32p, _f64p, _f64p]
        lib.p2p_tree_walk.restype = ctypes.c_int64
        lib.p2p_tree_walk.argtypes = [_vp, ctypes.c_double, ctypes.c_double]
        lib.p2p_tree_tasks.argtypes = [_vp, _i32p, _i32p]
        lib.p2p_tree_walk_masked.restype = ctypes.c_int64
        lib.p2p_tree_walk_masked.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        lib.p2p_lists_num_threads.restype = ctypes.c_int
        lib._typed = True
    return lib


def core():
    """libphotons_p2p.so with its C ABI (include/photons_p2p.h) typed."""
    lib = _load("libphotons_p2p.so")
    if getattr(lib, "_typed", False):
        return lib
    from . import abi
    abi.declare(lib)
    lib._typed = True
    return lib
