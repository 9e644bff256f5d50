// Device code of the P2P pass for sm_100a.
//
// Pass structure on the device (one chunk of the interaction list):
//   prep        one warp per leaf: FP64 frame centre (bounding-box midpoint of
//               the leaf's particles) and FP32 coordinates relative to it,
//               scaled by c = 1/(2 r_s); the FP64 form keeps FP64 positions.
//   csr_count   sink histogram of the (sink, source) list + pair count
//   scan        exclusive scan of the histogram -> row offsets (int64)
//   csr_scatter sources grouped by sink row
//   pair kernel persistent, one warp per sink row taken from an atomic work
//               counter; the row's source leaves are staged in shared memory
//               in the sink's frame, every lane owns a sink particle (or a
//               share of one, for rows with <= 16 sink particles) and streams
//               the staged sources.
//
// The reference builds the same CSR with thrust::sort_by_key /
// reduce_by_key / exclusive_scan (src/gpu_entry.cu:132-138) and runs
// P2P_kernel3 with one CTA per sink leaf (src/gpu_kernel.impl.h:439-524).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "p2p_internal.h"

#include "p2p_pass_kernels.cuh"
#include "p2p_pair_kernels.cuh"
