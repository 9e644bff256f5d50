"""The allocation-free entry point p2p_pass_noalloc, called through the C ABI.

It is meant for host codes that cannot have a library call cudaMalloc or
cudaFree while they run (a simulation that reserves the GPU's memory for its
own pool, a process under a fixed device-memory quota, a code whose other
streams must not be stalled by cudaFree's device-wide synchronisation; the
call itself blocks its host thread until its own stream has finished the
pass). Its scratch is a fixed
static device array, so two calls in a row must give the same forces as the
session entry point (p2p_pass_run_device), within the same tolerances the
parity tests use. This file is collected last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err
from photons_p2p import _native, abi, workloads as W
from photons_p2p.p2p import Session, params_for

pytestmark = pytest.mark.gpu

SPLIT_RMS = 1e-5
SPLIT_MAX = 1e-3
PLAIN_MAX = 1e-12


def _device_inputs(torch, tl):
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
            for a in (tl.pos, tl.leaf_ipart, tl.leaf_npart, tl.task_t, tl.task_s)]


def _session_result(prm, tl, d):
    with Session(0, prm) as s:
        s.run_device(tl.npart, d[0].data_ptr(), tl.nleaf, d[1].data_ptr(), d[2].data_ptr(),
                     tl.ntask, d[3].data_ptr(), d[4].data_ptr())
        s.end()
        out = np.zeros((3, tl.npart))
        s.accumulate(out)
    return out


@pytest.mark.parametrize("form", [abi.FORM_SPLIT, abi.FORM_PLAIN_FP64])
def test_noalloc_matches_session_entry_point(gpu, form):
    torch = pytest.importorskip("torch")
    lib = _native.core()
    cfg = W.ref_dropin_config(32, 64, 32)
    pos = W.lattice_gaussian(32, 0.2, W.rng(1))
    tl = W.prepare(pos, cfg)
    prm = params_for(cfg, form, 1.0 / pos.shape[1])
    d = _device_inputs(torch, tl)
    torch.cuda.synchronize()
    ref = _session_result(prm, tl, d)
    d_acc = torch.empty(3 * tl.npart, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d_acc.fill_(np.nan)  # the entry point must overwrite every element
        torch.cuda.synchronize()
        st = lib.p2p_pass_noalloc(ctypes.byref(prm), tl.npart, d[0].data_ptr(), tl.nleaf,
                                  d[1].data_ptr(), d[2].data_ptr(), tl.ntask, d[3].data_ptr(),
                                  d[4].data_ptr(), d_acc.data_ptr(), stream)
        assert st == abi.P2P_OK, (call, st, lib.p2p_status_string(st))
        got = d_acc.cpu().numpy().reshape(3, tl.npart)
        local = tl.tag == 1
        rms, mx = rel_err(got, ref, local)
        if form == abi.FORM_PLAIN_FP64:
            assert mx <= PLAIN_MAX, (call, rms, mx)
        else:
            assert rms <= SPLIT_RMS and mx <= SPLIT_MAX, (call, rms, mx)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    """Beyond P2P_NOALLOC_SCRATCH_BYTES the call returns P2P_ERR_CAPACITY on the
    host, before any work is queued (the small buffers are never read)."""
    torch = pytest.importorskip("torch")
    lib = _native.core()
    prm = abi.Params()
    lib.p2p_params_default(ctypes.byref(prm))
    prm.form = abi.FORM_SPLIT
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    ints = torch.zeros(16, dtype=torch.int32, device="cuda")
    npart = 8_000_000  # 16 B per particle of scratch alone exceeds 64 MiB
    st = lib.p2p_pass_noalloc(ctypes.byref(prm), npart, small.data_ptr(), 1, ints.data_ptr(),
                              ints.data_ptr(), 1, ints.data_ptr(), ints.data_ptr(), small.data_ptr(),
                              None)
    assert st == abi.P2P_ERR_CAPACITY
