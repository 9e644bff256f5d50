"""Build recipe for the native libraries of the package.

    libphotons_p2p.so    CUDA P2P pass for sm_100a + its C ABI (csrc/*.cu); the PM
                         long-range force links cuFFT for its two FFTs
    libphotons_lists.so  host tree build / interaction-list walk (host/*.cpp)

Both land in photons_p2p/ next to the Python bindings, so a snapshot of the
repository carries them. Run `python photons-on-mt3000_b200/build.py`
(add --force to rebuild). nvcc cross-compiles sm_100a without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "photons_p2p")
INCLUDE = os.path.join(REPO, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CUDA_SOURCES = ["p2p_core.cu", "p2p_noalloc.cu", "p2p_pair_sink_lanes.cu", "p2p_pair_source_lanes.cu",
                "p2p_pair_source_lanes_x2.cu", "p2p_pair_source_lanes_x2_kahan.cu",
                "p2p_pair_source_lanes_x2_f32.cu", "p2p_pair_plain.cu", "p2p_server.cu", "p2p_pair_sink_lanes_x2.cu",
                "p2p_pair_sink_regs.cu", "p2p_tree.cu", "p2p_pm.cu", "p2p_fmm.cu"]
CUDA_HEADERS = ["p2p_kernels.cuh", "p2p_pass_kernels.cuh", "p2p_pair_kernels.cuh",
                "p2p_device_common.cuh", "p2p_launch.h", "p2p_internal.h", "p2p_fit.h",
                "p2p_pair_x2_impl.h", "p2p_csr.h", "p2p_args.h", "p2p_host_shared.h", "p2p_walk_kernels.cuh",
                "p2p_pair_sreg.cuh", "p2p_tree_kernels.cuh"]
HOST_SOURCES = ["p2p_lists.cpp"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_lists(force=False):
    target = os.path.join(OUT, "libphotons_lists.so")
    srcs = [os.path.join(HERE, "host", s) for s in HOST_SOURCES]
    if force or _stale(target, srcs + [__file__]):
        _run(["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-std=c++17", "-fPIC", "-fopenmp", "-shared",
              "-o", target] + srcs)
    return target


def build_cuda(force=False, extra=()):
    """Each .cu compiles to an object in parallel, then one shared link."""
    from concurrent.futures import ThreadPoolExecutor

    target = os.path.join(OUT, "libphotons_p2p.so")
    srcs = [os.path.join(HERE, "csrc", s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(HERE, "csrc", h) for h in CUDA_HEADERS] + [
        os.path.join(INCLUDE, "photons_p2p.h"), __file__]
    if not (force or _stale(target, deps)):
        return target
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = GENCODE + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                       "-I", INCLUDE] + list(extra)
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]
    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        list(ex.map(lambda so: _run([NVCC] + flags + ["-c", so[0], "-o", so[1]]), zip(srcs, objs)))
    cudalib = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
    _run([NVCC] + GENCODE + ["--shared", "-o", target] + objs +
         ["-L", cudalib, "-lcufft", "-Xlinker", "-rpath," + cudalib])
    return target


def build(force=False):
    os.makedirs(OUT, exist_ok=True)
    return [build_lists(force), build_cuda(force)]


if __name__ == "__main__":
    build(force="--force" in sys.argv)
