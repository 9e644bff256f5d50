import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "photons-on-mt3000_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    """Build whatever native pieces are missing (no-op when present)."""
    import build as pkg_build

    lib_dir = os.path.join(PKG, "photons_p2p")
    if not os.path.exists(os.path.join(lib_dir, "libphotons_lists.so")):
        pkg_build.build_lists()
    if not os.path.exists(os.path.join(lib_dir, "libphotons_p2p.so")):
        pkg_build.build_cuda()
    from oracle import oracle

    oracle.build()


_ensure_built()


def gpu_count():
    from photons_p2p import _native
    import ctypes

    n = ctypes.c_int(0)
    try:
        _native.core().p2p_device_count(ctypes.byref(n))
    except Exception:
        return 0
    return n.value


@pytest.fixture(scope="session")
def gpu():
    if gpu_count() < 1:
        pytest.fail("this test needs a CUDA GPU and none is visible")
    return 0


def rel_err(got, ref, mask=None):
    """Per-particle relative error |a - b| / |b| of (3, n) force arrays."""
    import numpy as np

    num = np.linalg.norm(got - ref, axis=0)
    den = np.linalg.norm(ref, axis=0)
    if mask is not None:
        num, den = num[mask], den[mask]
    keep = den > 0
    r = num[keep] / den[keep]
    return float(np.sqrt(np.mean(r ** 2))) if r.size else 0.0, float(r.max()) if r.size else 0.0
