// Launcher of the FP64 drop-in pair kernel (pair_plain_kernel).
#include "p2p_launch.h"
#include "p2p_pair_kernels.cuh"

namespace p2p {

PairLaunchResult launch_pair_plain(const PairLaunch &L, const PairArgs &a) {
    const size_t smem = pair_smem_plain(L.warps, L.stage);
    if (L.soft_mode == SOFT_CLAMP)
        return L.masses ? launch_persistent(L, pair_plain_kernel<SOFT_CLAMP, true>, smem, a)
                        : launch_persistent(L, pair_plain_kernel<SOFT_CLAMP, false>, smem, a);
    return L.masses ? launch_persistent(L, pair_plain_kernel<SOFT_PLUMMER, true>, smem, a)
                    : launch_persistent(L, pair_plain_kernel<SOFT_PLUMMER, false>, smem, a);
}

cudaError_t allow_smem_plain() {
    const void *ks[] = {(const void *)pair_plain_kernel<SOFT_CLAMP, false>,
                        (const void *)pair_plain_kernel<SOFT_CLAMP, true>,
                        (const void *)pair_plain_kernel<SOFT_PLUMMER, false>,
                        (const void *)pair_plain_kernel<SOFT_PLUMMER, true>};
    cudaError_t e = cudaSuccess;
    for (const void *k : ks)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    return e;
}

}  // namespace p2p
