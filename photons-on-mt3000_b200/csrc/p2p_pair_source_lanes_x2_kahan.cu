// Packed source-lane pair kernel, Kahan-compensated FP32 accumulation.
#include "p2p_pair_x2_impl.h"

namespace p2p {

PairLaunchResult launch_x2_kahan(const PairLaunch &L, const PairArgs &a) { return x2_impl::launch<ACC_KAHAN>(L, a); }
cudaError_t allow_x2_kahan() { return x2_impl::allow<ACC_KAHAN>(); }

}  // namespace p2p
