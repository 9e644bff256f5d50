// Launcher of the sink-lanes mapping of the FP32 pair kernel (pair_split_kernel),
// every (softening, masses, accumulation, coefficient count) instance.
#include "p2p_launch.h"
#include "p2p_pair_kernels.cuh"

namespace p2p {
namespace {

constexpr int kMaxSmemBytes = 227 * 1024;

template <int SOFT, bool MASSES, int ACC>
PairLaunchResult by_ncoef(const PairLaunch &L, const PairArgs &a) {
    const size_t smem = pair_smem_split(L.warps, L.stage, false);
    switch (L.ncoef) {
        case 9: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 9>, smem, a);
        case 11: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 11>, smem, a);
        case 13: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 13>, smem, a);
        case 15: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 15>, smem, a);
        case 17: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 17>, smem, a);
        case 21: return launch_persistent(L, pair_split_kernel<SOFT, MASSES, ACC, 21>, smem, a);
        default: {
            PairLaunchResult r;
            r.cuda = cudaErrorInvalidValue;
            return r;
        }
    }
}

template <int SOFT, bool MASSES>
PairLaunchResult by_acc(const PairLaunch &L, const PairArgs &a) {
    switch (L.acc) {
        case ACC_KAHAN: return by_ncoef<SOFT, MASSES, ACC_KAHAN>(L, a);
        case ACC_F32: return by_ncoef<SOFT, MASSES, ACC_F32>(L, a);
        default: return by_ncoef<SOFT, MASSES, ACC_F64>(L, a);
    }
}

template <int SOFT, bool MASSES, int ACC>
cudaError_t allow_acc() {
    const void *ks[] = {(const void *)pair_split_kernel<SOFT, MASSES, ACC, 9>, (const void *)pair_split_kernel<SOFT, MASSES, ACC, 11>,
                        (const void *)pair_split_kernel<SOFT, MASSES, ACC, 13>, (const void *)pair_split_kernel<SOFT, MASSES, ACC, 15>,
                        (const void *)pair_split_kernel<SOFT, MASSES, ACC, 17>, (const void *)pair_split_kernel<SOFT, MASSES, ACC, 21>};
    cudaError_t e = cudaSuccess;
    for (const void *k : ks)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemBytes);
    return e;
}

template <int SOFT, bool MASSES>
cudaError_t allow_masses() {
    cudaError_t e = allow_acc<SOFT, MASSES, ACC_F64>();
    if (e == cudaSuccess) e = allow_acc<SOFT, MASSES, ACC_KAHAN>();
    if (e == cudaSuccess) e = allow_acc<SOFT, MASSES, ACC_F32>();
    return e;
}

}  // namespace

PairLaunchResult launch_pair_sink_lanes(const PairLaunch &L, const PairArgs &a) {
    if (L.soft_mode == SOFT_CLAMP)
        return L.masses ? by_acc<SOFT_CLAMP, true>(L, a) : by_acc<SOFT_CLAMP, false>(L, a);
    return L.masses ? by_acc<SOFT_PLUMMER, true>(L, a) : by_acc<SOFT_PLUMMER, false>(L, a);
}

cudaError_t allow_smem_sink_lanes() {
    cudaError_t e = allow_masses<SOFT_CLAMP, false>();
    if (e == cudaSuccess) e = allow_masses<SOFT_CLAMP, true>();
    if (e == cudaSuccess) e = allow_masses<SOFT_PLUMMER, false>();
    if (e == cudaSuccess) e = allow_masses<SOFT_PLUMMER, true>();
    return e;
}

}  // namespace p2p
