// Launcher of the sink-register mapping of the FP32 pair kernel
// (pair_sreg_kernel), all accumulation modes.
#include "p2p_launch.h"
#include "p2p_pair_sreg.cuh"

namespace p2p {
namespace {

template <int SOFT, bool MASSES, int ACC>
PairLaunchResult by_ncoef(const PairLaunch &L0, const PairArgs &a) {
    PairLaunch L = L0;
    L.stage = sreg_stage(L0.stage);  // the kernel's stage capacity (at least one staging group)
    const size_t smem = pair_smem_sreg(L.warps, L.stage);
    switch (L.ncoef) {
        case 9: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 9, P2P_SREG_SPL>, smem, a);
        case 11: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 11, P2P_SREG_SPL>, smem, a);
        case 13: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 13, P2P_SREG_SPL>, smem, a);
        case 15: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 15, P2P_SREG_SPL>, smem, a);
        case 17: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 17, P2P_SREG_SPL>, smem, a);
        case 21: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 21, P2P_SREG_SPL>, smem, a);
        default: {
            PairLaunchResult r;
            r.cuda = cudaErrorInvalidValue;
            return r;
        }
    }
}

template <int ACC>
PairLaunchResult by_soft(const PairLaunch &L, const PairArgs &a) {
    if (L.soft_mode == SOFT_CLAMP)
        return L.masses ? by_ncoef<SOFT_CLAMP, true, ACC>(L, a) : by_ncoef<SOFT_CLAMP, false, ACC>(L, a);
    return L.masses ? by_ncoef<SOFT_PLUMMER, true, ACC>(L, a) : by_ncoef<SOFT_PLUMMER, false, ACC>(L, a);
}

template <int SOFT, bool MASSES, int ACC>
cudaError_t allow_one() {
    const void *ks[] = {(const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 9, P2P_SREG_SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 11, P2P_SREG_SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 13, P2P_SREG_SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 15, P2P_SREG_SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 17, P2P_SREG_SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 21, P2P_SREG_SPL>};
    cudaError_t e = cudaSuccess;
    for (const void *k : ks) {
        // the opt-in limit covers static and dynamic shared memory together
        cudaFuncAttributes fa;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     227 * 1024 - (int)fa.sharedSizeBytes);
    }
    return e;
}

template <int ACC>
cudaError_t allow_acc() {
    cudaError_t e = allow_one<SOFT_CLAMP, false, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_CLAMP, true, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, false, ACC>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, true, ACC>();
    return e;
}

}  // namespace

PairLaunchResult launch_pair_sink_regs(const PairLaunch &L, const PairArgs &a) {
    switch (L.acc) {
        case ACC_KAHAN: return by_soft<ACC_KAHAN>(L, a);
        case ACC_F32: return by_soft<ACC_F32>(L, a);
        default: return by_soft<ACC_F64>(L, a);
    }
}

cudaError_t allow_smem_sink_regs() {
    cudaError_t e = allow_acc<ACC_F64>();
    if (e == cudaSuccess) e = allow_acc<ACC_KAHAN>();
    if (e == cudaSuccess) e = allow_acc<ACC_F32>();
    return e;
}

}  // namespace p2p
