// Launcher of the sink-register mapping of the FP32 pair kernel
// (pair_sreg_kernel), all accumulation modes.
#include "p2p_launch.h"
#include "p2p_pair_sreg.cuh"

namespace p2p {
namespace {

template <int SOFT, bool MASSES, int ACC, int SPL>
PairLaunchResult by_ncoef(const PairLaunch &L0, const PairArgs &a) {
    PairLaunch L = L0;
    L.stage = sreg_stage(L0.stage);  // the kernel's stage capacity (at least one staging group)
    const size_t smem = pair_smem_sreg(L.warps, L.stage, SPL);
    switch (L.ncoef) {
        case 9: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 9, SPL>, smem, a);
        case 11: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 11, SPL>, smem, a);
        case 13: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 13, SPL>, smem, a);
        case 15: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 15, SPL>, smem, a);
        case 17: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 17, SPL>, smem, a);
        case 21: return launch_persistent(L, pair_sreg_kernel<SOFT, MASSES, ACC, 21, SPL>, smem, a);
        default: {
            PairLaunchResult r;
            r.cuda = cudaErrorInvalidValue;
            return r;
        }
    }
}

template <int ACC, int SPL>
PairLaunchResult by_soft(const PairLaunch &L, const PairArgs &a) {
    if (L.soft_mode == SOFT_CLAMP)
        return L.masses ? by_ncoef<SOFT_CLAMP, true, ACC, SPL>(L, a) : by_ncoef<SOFT_CLAMP, false, ACC, SPL>(L, a);
    return L.masses ? by_ncoef<SOFT_PLUMMER, true, ACC, SPL>(L, a) : by_ncoef<SOFT_PLUMMER, false, ACC, SPL>(L, a);
}

template <int SPL>
PairLaunchResult by_acc(const PairLaunch &L, const PairArgs &a) {
    switch (L.acc) {
        case ACC_KAHAN: return by_soft<ACC_KAHAN, SPL>(L, a);
        case ACC_F32: return by_soft<ACC_F32, SPL>(L, a);
        default: return by_soft<ACC_F64, SPL>(L, a);
    }
}

template <int SOFT, bool MASSES, int ACC, int SPL>
cudaError_t allow_one() {
    const void *ks[] = {(const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 9, SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 11, SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 13, SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 15, SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 17, SPL>,
                        (const void *)pair_sreg_kernel<SOFT, MASSES, ACC, 21, SPL>};
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

template <int ACC, int SPL>
cudaError_t allow_acc() {
    cudaError_t e = allow_one<SOFT_CLAMP, false, ACC, SPL>();
    if (e == cudaSuccess) e = allow_one<SOFT_CLAMP, true, ACC, SPL>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, false, ACC, SPL>();
    if (e == cudaSuccess) e = allow_one<SOFT_PLUMMER, true, ACC, SPL>();
    return e;
}

}  // namespace

PairLaunchResult launch_pair_sink_regs(const PairLaunch &L, const PairArgs &a) {
    return L.sreg_spl == 8 ? by_acc<8>(L, a) : by_acc<4>(L, a);
}

cudaError_t allow_smem_sink_regs() {
    cudaError_t e = cudaSuccess;
    for (int spl : {4, 8}) {
        if (e == cudaSuccess) e = spl == 4 ? allow_acc<ACC_F64, 4>() : allow_acc<ACC_F64, 8>();
        if (e == cudaSuccess) e = spl == 4 ? allow_acc<ACC_KAHAN, 4>() : allow_acc<ACC_KAHAN, 8>();
        if (e == cudaSuccess) e = spl == 4 ? allow_acc<ACC_F32, 4>() : allow_acc<ACC_F32, 8>();
    }
    return e;
}

}  // namespace p2p
