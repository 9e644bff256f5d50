"""The C-ABI libraries load and export every symbol their headers declare.
No GPU compute is called here."""
import ctypes
import os
import subprocess

import pytest

from photons_p2p import _native, abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(REPO, "include")
REF = os.path.join(REPO, "oracle", "_ref")


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_core_exports_every_header_symbol():
    lib = _native.lib_path("libphotons_p2p.so")
    syms = exported(lib)
    declared = abi.header_symbols(os.path.join(INCLUDE, "photons_p2p.h"))
    assert declared, "no declarations parsed"
    missing = [s for s in declared if s not in syms]
    assert not missing, missing
    # the ctypes table covers the same functions
    assert set(abi.SIGNATURES) == set(declared)


def test_core_loads_and_answers_without_gpu():
    lib = _native.core()
    assert lib.p2p_version() >= 10000
    assert lib.p2p_status_string(abi.P2P_ERR_RANGE) == b"input index out of range"
    p = abi.Params()
    lib.p2p_params_default(ctypes.byref(p))
    assert p.form == abi.FORM_PLAIN_FP64 and p.soft_mode == abi.SOFT_CLAMP and p.x_cut == 2.8125
    n = ctypes.c_int(-1)
    assert lib.p2p_device_count(ctypes.byref(n)) == abi.P2P_OK
    assert n.value >= 0


def test_null_arguments_are_rejected():
    lib = _native.core()
    assert lib.p2p_session_create(0, None) == abi.P2P_ERR_ARG
    assert lib.p2p_session_set_params(None, None) == abi.P2P_ERR_ARG
    assert lib.p2p_pass_end(None, None) == abi.P2P_ERR_ARG
    assert lib.p2p_pass_submit_walk(None, None, 1.0, 0.0, None) == abi.P2P_ERR_ARG
    assert lib.p2p_pass_rows(None, None, None) == abi.P2P_ERR_ARG
    assert b"null" in lib.p2p_last_error()


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_walk.so")),
                    reason="reference walk harness not built")
def test_reference_walk_library_loads():
    ctypes.CDLL(os.path.join(REF, "libref_walk.so"), mode=ctypes.RTLD_LOCAL)
    ctypes.CDLL(os.path.join(REF, "libref_pair.so"), mode=ctypes.RTLD_LOCAL)


def test_lists_library_loads():
    lib = _native.lists()
    assert lib.p2p_lists_num_threads() >= 1


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libref_dropin_dp.so")),
                    reason="drop-in harness (reference walk + B200 gpu_entry) not built")
@pytest.mark.parametrize("variant", ["dp", "sp", "act"])
def test_dropin_exports_legacy_entry_points(variant):
    syms = exported(os.path.join(REF, f"libref_dropin_{variant}.so"))
    declared = abi.header_symbols(os.path.join(INCLUDE, "photons_gpu_entry.h"))
    assert {"task_compute_p2p_gpu", "task_compute_p2p_act_gpu", "p2ppack_compute_act_gpu"} <= set(declared)
    missing = [s for s in declared if s not in syms]
    assert not missing, missing
    # every symbol resolves at load time (no GPU call is made by loading)
    ctypes.CDLL(os.path.join(REF, f"libref_dropin_{variant}.so"), mode=ctypes.RTLD_LOCAL)
