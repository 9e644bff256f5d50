// Launcher of the packed (f32x2) source-lane mapping of the FP32 pair kernel
// (pair_split_src2_kernel), FP64 accumulation; dispatches the other
// accumulation modes to their own translation units.
#include "p2p_pair_x2_impl.h"

namespace p2p {

PairLaunchResult launch_x2_f64(const PairLaunch &L, const PairArgs &a) { return x2_impl::launch<ACC_F64>(L, a); }
cudaError_t allow_x2_f64() { return x2_impl::allow<ACC_F64>(); }

PairLaunchResult launch_pair_source_lanes_x2(const PairLaunch &L, const PairArgs &a) {
    switch (L.acc) {
        case ACC_KAHAN: return launch_x2_kahan(L, a);
        case ACC_F32: return launch_x2_f32(L, a);
        default: return launch_x2_f64(L, a);
    }
}

cudaError_t allow_smem_source_lanes_x2() {
    cudaError_t e = allow_x2_f64();
    if (e == cudaSuccess) e = allow_x2_kahan();
    if (e == cudaSuccess) e = allow_x2_f32();
    return e;
}

}  // namespace p2p
