// Packed source-lane pair kernel, plain FP32 accumulation.
#include "p2p_pair_x2_impl.h"

namespace p2p {

PairLaunchResult launch_x2_f32(const PairLaunch &L, const PairArgs &a) { return x2_impl::launch<ACC_F32>(L, a); }
cudaError_t allow_x2_f32() { return x2_impl::allow<ACC_F32>(); }

}  // namespace p2p
