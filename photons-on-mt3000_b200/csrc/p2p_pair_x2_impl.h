// Launch helpers of the packed source-lane kernel for one accumulation mode.
// Each p2p_pair_source_lanes_x2*.cu instantiates one mode so the instances
// compile in parallel.
#pragma once

#include "p2p_launch.h"
#include "p2p_pair_kernels.cuh"

namespace p2p {
namespace x2_impl {

template <int SOFT, bool MASSES, int ACC, int NP>
PairLaunchResult by_ncoef(const PairLaunch &L, const PairArgs &a) {
    const size_t smem = pair_smem_x2(L.warps, L.stage);
    switch (L.ncoef) {
        case 9: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 9, NP>, smem, a);
        case 11: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 11, NP>, smem, a);
        case 13: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 13, NP>, smem, a);
        case 15: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 15, NP>, smem, a);
        case 17: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 17, NP>, smem, a);
        case 21: return launch_persistent(L, pair_split_src2_kernel<SOFT, MASSES, ACC, 21, NP>, smem, a);
        default: {
            PairLaunchResult r;
            r.cuda = cudaErrorInvalidValue;
            return r;
        }
    }
}

template <int SOFT, bool MASSES, int ACC>
PairLaunchResult by_tile(const PairLaunch &L, const PairArgs &a) {
    return L.sink_pairs == 8 ? by_ncoef<SOFT, MASSES, ACC, 8>(L, a) : by_ncoef<SOFT, MASSES, ACC, 16>(L, a);
}

template <int ACC>
PairLaunchResult launch(const PairLaunch &L, const PairArgs &a) {
    if (L.soft_mode == SOFT_CLAMP)
        return L.masses ? by_tile<SOFT_CLAMP, true, ACC>(L, a) : by_tile<SOFT_CLAMP, false, ACC>(L, a);
    return L.masses ? by_tile<SOFT_PLUMMER, true, ACC>(L, a) : by_tile<SOFT_PLUMMER, false, ACC>(L, a);
}

template <int SOFT, bool MASSES, int ACC, int NP>
cudaError_t allow_tile() {
    const void *ks[] = {(const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 9, NP>,
                        (const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 11, NP>,
                        (const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 13, NP>,
                        (const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 15, NP>,
                        (const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 17, NP>,
                        (const void *)pair_split_src2_kernel<SOFT, MASSES, ACC, 21, NP>};
    cudaError_t e = cudaSuccess;
    for (const void *k : ks)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    return e;
}

template <int SOFT, bool MASSES, int ACC>
cudaError_t allow_one() {
    cudaError_t e = allow_tile<SOFT, MASSES, ACC, 16>();
    if (e == cudaSuccess) e = allow_tile<SOFT, MASSES, ACC, 8>();
    return e;
}

template <int ACC>
cudaError_t allow() {
    cudaError_t e = allow_one<SOFT_CLAMP, false, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_CLAMP, true, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, false, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, true, ACC>();
    return e;
}

}  // namespace x2_impl

// one function pair per accumulation mode (p2p_pair_source_lanes_x2{,_kahan,_f32}.cu)
PairLaunchResult launch_x2_f64(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_x2_kahan(const PairLaunch &L, const PairArgs &a);
PairLaunchResult launch_x2_f32(const PairLaunch &L, const PairArgs &a);
cudaError_t allow_x2_f64();
cudaError_t allow_x2_kahan();
cudaError_t allow_x2_f32();

}  // namespace p2p
