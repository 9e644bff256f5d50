// Host services of libphotons_p2p shared across its translation units
// (defined in p2p_core.cu).
#pragma once

#include <cuda_runtime.h>

#include "photons_p2p.h"

namespace p2p {
// Records msg as p2p_last_error() of the calling thread; returns status.
int report_error(int status, const char *msg);
// P2P_OK or P2P_ERR_ARG (with the message recorded) for a parameter set.
int check_params(const p2p_params *p);
// Adds to p2p_kernel_launch_count().
void count_launches(int n);
// Opts every pair kernel into large dynamic shared memory on the current device.
cudaError_t allow_large_smem();
// The CUDA device of a session.
int session_device(const p2p_session *s);
// Device scratch the session keeps between calls: slot k holds at least
// bytes (grown when smaller, after the session's stream has drained;
// nullptr with p2p_last_error set when allocation fails). Freed with the
// session. Callers number their temporaries in request order, so repeated
// calls of the same size allocate nothing.
void *session_scratch(p2p_session *s, int slot, size_t bytes);
}  // namespace p2p
