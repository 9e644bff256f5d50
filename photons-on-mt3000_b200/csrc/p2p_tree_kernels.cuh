// Device kd-tree build: the caller-side tree of the P2P pass (PhotoNs'
// build_kdtree / center_kdtree, src/fmm.c:69-122,231-327) built on the GPU
// with the same nodes, leaves, numbering and particle order.
//
// The reference splits a node of n particles at the mean of its coordinate
// on axis depth % 3 (sampled every max(1, n / 1e5)-th particle, summed in
// order) with an in-place two-pointer partition (bksort_inplace,
// src/fmm.c:69-122). That partition has a parallel form, used here: with nS
// the number of particles not above the mean, the k-th particle above the
// mean among the first nS slots swaps with the k-th particle not above it
// counted from the right among the last n - nS slots; the left child takes
// nS particles, or n - 1 when none lies above the mean; a node of two
// particles splits at their midpoint, swapping them when the first is above
// the second. Nodes are split level by level while they hold more than
// kTreeSmall particles (the mean by one thread, the partition by tiles of
// the node's slots); smaller subtrees are built whole by one block each in
// shared memory. Nodes and leaves get build-order ids as they are made; the
// pre-order ids of the reference (son[0]'s subtree first, leaves numbered
// apart from nodes) and the node boxes follow from two passes over depths.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace p2p {

constexpr int kTreeSmall = 2048;       // subtrees up to this size are built by one block
constexpr int kTreeTile = 2048;        // slots per tile of the level-wide partition
constexpr int kTreeThreads = 256;
constexpr int kTreeMaxStack = kTreeSmall;

// Status bits of the tree build.
enum : int {
    TB_NODE_CAP = 1,   // more nodes than the build's node capacity
    TB_LEAF_CAP = 2,   // more leaves than the leaf capacity
    TB_NUMBERING = 4,  // a pre-order id out of range (inconsistent records; nothing written)
};

// Build-order records (structure of arrays) of nodes and leaves.
struct TreeRec {
    // nodes
    double *split;
    int *son;      // 2 per node: build id of a leaf l -> 2l, of a node k -> 2k+1
    int *depth;
    int *nn, *nl;  // nodes and leaves in the node's subtree (itself included)
    int *pre;      // pre-order id
    int *first;    // pre-order id of the subtree's first leaf
    double *box;   // 6 per node: left[3], right[3]
    int node_cap;
    // leaves
    int *lipart, *lnpart, *lid;  // particle range, pre-order leaf id
    int leaf_cap;
    int *counters;  // [0] nodes made, [1] leaves made, [2] status bits, [3] max depth
};

// Particles being partitioned: SoA coordinates and original indices.
struct TreeParts {
    double *x, *y, *z;
    int *id;
};

__device__ __forceinline__ double tree_coord(const TreeParts &P, int axis, int i) {
    return axis == 0 ? P.x[i] : (axis == 1 ? P.y[i] : P.z[i]);
}

__device__ __forceinline__ void tree_swap(TreeParts &P, int i, int j) {
    const double tx = P.x[i], ty = P.y[i], tz = P.z[i];
    const int ti = P.id[i];
    P.x[i] = P.x[j]; P.y[i] = P.y[j]; P.z[i] = P.z[j]; P.id[i] = P.id[j];
    P.x[j] = tx; P.y[j] = ty; P.z[j] = tz; P.id[j] = ti;
}

// The reference's split value of a node of length >= 3: the sampled mean,
// summed in slot order (src/fmm.c:88-97).
__device__ __forceinline__ double tree_mean(const double *c, int length) {
    int mul = 1;
    if (length > 100000) mul = length / 100000;
    double mean = 0.0;
    for (int n = 0; n < length; n += mul) mean = __dadd_rn(mean, c[n]);
    mean = __ddiv_rn(mean, (double)length);
    return __dmul_rn(mean, (double)mul);
}

// -------------------------------------------------------------- inputs ---

// Copies the positions into the work arrays, ids = slot, and per-block
// min / max of the float-rounded coordinates (particle_combine's bounds,
// src/gravity.c:69-121).
__global__ void tree_init_kernel(const double *__restrict__ pos, int n, TreeParts P,
                                 float *__restrict__ block_lo, float *__restrict__ block_hi) {
    __shared__ float slo[3][kTreeThreads], shi[3][kTreeThreads];
    float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double c[3] = {pos[i], pos[(size_t)n + i], pos[2 * (size_t)n + i]};
        P.x[i] = c[0];
        P.y[i] = c[1];
        P.z[i] = c[2];
        P.id[i] = i;
        for (int d = 0; d < 3; ++d) {
            const float f = (float)c[d];
            lo[d] = fminf(lo[d], f);
            hi[d] = fmaxf(hi[d], f);
        }
    }
    for (int d = 0; d < 3; ++d) {
        slo[d][threadIdx.x] = lo[d];
        shi[d][threadIdx.x] = hi[d];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int d = 0; d < 3; ++d) {
                slo[d][threadIdx.x] = fminf(slo[d][threadIdx.x], slo[d][threadIdx.x + s]);
                shi[d][threadIdx.x] = fmaxf(shi[d][threadIdx.x], shi[d][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) {
            block_lo[3 * blockIdx.x + d] = slo[d][0];
            block_hi[3 * blockIdx.x + d] = shi[d][0];
        }
}

// The root box: boxL = min(boxsize, min float coordinate) - 1e-6 boxsize,
// boxH = max(0, max float coordinate) + 1e-6 boxsize, per axis (one thread).
__global__ void tree_root_box_kernel(const float *__restrict__ block_lo, const float *__restrict__ block_hi,
                                     int nblocks, double boxsize, TreeRec R, int root) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int d = 0; d < 3; ++d) {
        double lo = boxsize, hi = 0.0;
        for (int b = 0; b < nblocks; ++b) {
            const double l = (double)block_lo[3 * b + d], h = (double)block_hi[3 * b + d];
            if (lo > l) lo = l;
            if (hi < h) hi = h;
        }
        const double margin = __dmul_rn(0.000001, boxsize);
        R.box[6 * (size_t)root + d] = __dsub_rn(lo, margin);
        R.box[6 * (size_t)root + 3 + d] = __dadd_rn(hi, margin);
    }
}

// ---------------------------------------------------- level-wide split ---

// A node split level-wide: its slots, axis, and (after the count) the number
// of its particles not above the mean.
struct TreeSeg {
    int ipart, length, axis, node;
    double mean;
    int nsmall, nbig;
};

// One block per segment: the split value. The samples are gathered into
// shared memory by the whole block, a chunk at a time, and summed in slot
// order by one thread (the reference's rounding sequence, tree_mean).
constexpr int kTreeMeanChunk = 4096;
__global__ void __launch_bounds__(kTreeThreads) tree_seg_mean_kernel(TreeSeg *segs, TreeParts P, TreeRec R) {
    __shared__ double buf[kTreeMeanChunk];
    const TreeSeg g = segs[blockIdx.x];
    const double *c = (g.axis == 0 ? P.x : (g.axis == 1 ? P.y : P.z)) + g.ipart;
    int mul = 1;
    if (g.length > 100000) mul = g.length / 100000;
    const int nsamp = (g.length + mul - 1) / mul;  // slots 0, mul, 2 mul, ... < length
    double mean = 0.0;
    for (int s0 = 0; s0 < nsamp; s0 += kTreeMeanChunk) {
        const int ns = min(kTreeMeanChunk, nsamp - s0);
        for (int i = threadIdx.x; i < ns; i += blockDim.x) buf[i] = c[(size_t)(s0 + i) * mul];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int i = 0; i < ns; ++i) mean = __dadd_rn(mean, buf[i]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        mean = __dmul_rn(__ddiv_rn(mean, (double)g.length), (double)mul);
        segs[blockIdx.x].mean = mean;
        R.split[g.node] = mean;
    }
}

// Tiles of kTreeTile slots: tile t covers slots [tile_off[t], +kTreeTile) of
// segment tile_seg[t]; counts the slots not above the mean.
__global__ void __launch_bounds__(kTreeThreads)
tree_tile_count_kernel(const TreeSeg *__restrict__ segs, const int *__restrict__ tile_seg,
                       const int *__restrict__ tile_off, TreeParts P, int *__restrict__ tile_small) {
    __shared__ int red[kTreeThreads / 32];
    const TreeSeg g = segs[tile_seg[blockIdx.x]];
    const int off = tile_off[blockIdx.x];
    const int end = min(g.length, off + kTreeTile);
    const double *c = (g.axis == 0 ? P.x : (g.axis == 1 ? P.y : P.z)) + g.ipart;
    int cnt = 0;
    for (int r = off + threadIdx.x; r < end; r += blockDim.x) cnt += c[r] > g.mean ? 0 : 1;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kTreeThreads / 32; ++w) t += red[w];
        tile_small[blockIdx.x] = t;
    }
}

// Block-wide exclusive prefix of one flag per thread (kTreeThreads threads).
__device__ __forceinline__ int tree_block_prefix(int flag, int *warp_tot, int *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    const int before = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[w] = __popc(m);
    __syncthreads();
    int base = 0, tot = 0;
    for (int q = 0; q < kTreeThreads / 32; ++q) {
        const int v = warp_tot[q];
        if (q < w) base += v;
        tot += v;
    }
    __syncthreads();
    *total = tot;
    return base + before;
}

// The swapped slots not above the mean: map[nsmall + q] = the slot of the
// (q+1)-th particle not above the mean counted from the right among the
// slots [nsmall, length) of the segment (relative slots). tile_pre[t] = slots
// not above the mean before tile t within its segment.
__global__ void __launch_bounds__(kTreeThreads)
tree_tile_map_kernel(const TreeSeg *__restrict__ segs, const int *__restrict__ tile_seg,
                     const int *__restrict__ tile_off, const int *__restrict__ tile_pre, TreeParts P,
                     int *__restrict__ map) {
    __shared__ int warp_tot[kTreeThreads / 32];
    const TreeSeg g = segs[tile_seg[blockIdx.x]];
    const int off = tile_off[blockIdx.x];
    const int end = min(g.length, off + kTreeTile);
    if (end <= g.nsmall) return;  // the whole tile lies in the left part (block-uniform)
    const double *c = (g.axis == 0 ? P.x : (g.axis == 1 ? P.y : P.z)) + g.ipart;
    int small_before = tile_pre[blockIdx.x];
    for (int r0 = off; r0 < end; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;
        const bool small = r < end && !(c[r] > g.mean);
        int tot;
        const int rank = tree_block_prefix(small ? 1 : 0, warp_tot, &tot);
        if (small && r >= g.nsmall) map[g.ipart + g.nsmall + (g.nsmall - (small_before + rank) - 1)] = r;
        small_before += tot;
    }
}

// The swaps: the particle above the mean at slot r < nsmall, the (q+1)-th
// such from the left (q = r minus the slots not above the mean before r),
// with the slot map[nsmall + q]. Only the thread of slot r touches r and its
// partner; flags are read in [0, nsmall) only, which no other thread writes.
__global__ void __launch_bounds__(kTreeThreads)
tree_tile_swap_kernel(const TreeSeg *__restrict__ segs, const int *__restrict__ tile_seg,
                      const int *__restrict__ tile_off, const int *__restrict__ tile_pre, TreeParts P,
                      const int *__restrict__ map) {
    __shared__ int warp_tot[kTreeThreads / 32];
    const TreeSeg g = segs[tile_seg[blockIdx.x]];
    const int off = tile_off[blockIdx.x];
    const int end = min(min(g.length, off + kTreeTile), g.nsmall);
    if (end <= off) return;  // the whole tile lies in the right part (block-uniform)
    const double *c = (g.axis == 0 ? P.x : (g.axis == 1 ? P.y : P.z)) + g.ipart;
    int small_before = tile_pre[blockIdx.x];
    for (int r0 = off; r0 < end; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;
        const bool in = r < end;
        const bool big = in && c[r] > g.mean;
        int tot;
        const int rank = tree_block_prefix(in && !big ? 1 : 0, warp_tot, &tot);
        if (big) {
            const int q = r - (small_before + rank);
            tree_swap(P, g.ipart + r, g.ipart + map[g.ipart + g.nsmall + q]);
        }
        small_before += tot;
    }
}

// ---------------------------------------------------- subtree per block ---

// A subtree to build in one block: slots, axis of its root, depth of its
// root, and where its root's code goes (son[2 * parent + side]).
struct TreeTask {
    int ipart, length, axis, depth, parent, side;
};

struct SmallItem {
    int span;    // slot offset in the task (low 16 bits) and length (high 16 bits)
    int parent;  // build id of the parent node
    short depth;
    char axis, side;
};

// Dynamic shared memory of tree_small_kernel.
constexpr size_t kTreeSmallSmem = (size_t)kTreeSmall * (3 * sizeof(double) + sizeof(int) + sizeof(short)) +
                                  (size_t)kTreeMaxStack * sizeof(SmallItem);

__device__ __forceinline__ int tree_new_leaf(TreeRec &R, int ip, int np) {
    const int l = atomicAdd(&R.counters[1], 1);
    if (l >= R.leaf_cap) {
        atomicOr(&R.counters[2], TB_LEAF_CAP);
        return -1;
    }
    R.lipart[l] = ip;
    R.lnpart[l] = np;
    return l;
}

__device__ __forceinline__ int tree_new_node(TreeRec &R, int depth) {
    const int k = atomicAdd(&R.counters[0], 1);
    if (k >= R.node_cap) {
        atomicOr(&R.counters[2], TB_NODE_CAP);
        return -1;
    }
    R.depth[k] = depth;
    atomicMax(&R.counters[3], depth);
    return k;
}

// One block builds a whole subtree of at most kTreeSmall particles in shared
// memory, node after node from an explicit stack (left child first, as the
// reference recursion), then writes the permuted particles back.
__global__ void __launch_bounds__(kTreeThreads)
tree_small_kernel(const TreeTask *__restrict__ tasks, TreeParts P, TreeRec R, int maxleaf) {
    extern __shared__ double tsm[];
    double *sx = tsm, *sy = sx + kTreeSmall, *sz = sy + kTreeSmall;
    int *sid = reinterpret_cast<int *>(sz + kTreeSmall);
    short *smap = reinterpret_cast<short *>(sid + kTreeSmall);
    SmallItem *stack = reinterpret_cast<SmallItem *>(smap + kTreeSmall);
    __shared__ int warp_tot[kTreeThreads / 32];
    __shared__ int s_top, s_node, s_kpairs;
    __shared__ double s_mean;
    const TreeTask T = tasks[blockIdx.x];
    for (int i = threadIdx.x; i < T.length; i += blockDim.x) {
        sx[i] = P.x[T.ipart + i];
        sy[i] = P.y[T.ipart + i];
        sz[i] = P.z[T.ipart + i];
        sid[i] = P.id[T.ipart + i];
    }
    if (threadIdx.x == 0) {
        SmallItem it;
        it.span = T.length << 16;
        it.parent = T.parent;
        it.depth = (short)T.depth;
        it.axis = (char)T.axis;
        it.side = (char)T.side;
        stack[0] = it;
        s_top = 1;
    }
    __syncthreads();
    while (s_top > 0) {
        const SmallItem it = stack[s_top - 1];
        __syncthreads();
        if (threadIdx.x == 0) {
            s_top -= 1;
            const int k = tree_new_node(R, it.depth);
            s_node = k;
            if (k >= 0 && it.parent >= 0) R.son[2 * it.parent + it.side] = 2 * k + 1;
        }
        __syncthreads();
        const int node = s_node;
        if (node < 0) break;  // node capacity exceeded (status set)
        const int base = it.span & 0xffff, len = it.span >> 16, axis = it.axis;
        double *c = axis == 0 ? sx : (axis == 1 ? sy : sz);
        int nleft;
        if (len < 2) {
            nleft = 0;
            if (threadIdx.x == 0) R.split[node] = 0.0;
        } else if (len == 2) {
            nleft = 1;
            if (threadIdx.x == 0) {
                R.split[node] = __dmul_rn(0.5, __dadd_rn(c[base], c[base + 1]));
                if (c[base] > c[base + 1]) {
                    double t;
                    t = sx[base]; sx[base] = sx[base + 1]; sx[base + 1] = t;
                    t = sy[base]; sy[base] = sy[base + 1]; sy[base + 1] = t;
                    t = sz[base]; sz[base] = sz[base + 1]; sz[base + 1] = t;
                    const int ti = sid[base]; sid[base] = sid[base + 1]; sid[base + 1] = ti;
                }
            }
        } else {
            if (threadIdx.x == 0) {
                s_mean = tree_mean(c + base, len);
                R.split[node] = s_mean;
            }
            __syncthreads();
            const double mean = s_mean;
            // nsmall: slots not above the mean
            int nsmall = 0;
            for (int r0 = 0; r0 < len; r0 += blockDim.x) {
                const int r = r0 + threadIdx.x;
                int tot;
                tree_block_prefix((r < len && !(c[base + r] > mean)) ? 1 : 0, warp_tot, &tot);
                nsmall += tot;
            }
            // positions of the swapped slots by rank; the pairs are the particles
            // above the mean among the first nsmall slots: nsmall minus the
            // slots not above it there (read at slot nsmall)
            if (threadIdx.x == 0) s_kpairs = 0;
            int small_before = 0;
            for (int r0 = 0; r0 < len; r0 += blockDim.x) {
                const int r = r0 + threadIdx.x;
                const bool in = r < len;
                const bool small = in && !(c[base + r] > mean);
                int tot;
                const int rank = tree_block_prefix(small ? 1 : 0, warp_tot, &tot);
                if (in) {
                    const int sb = small_before + rank;
                    if (!small && r < nsmall) smap[r - sb] = (short)r;
                    else if (small && r >= nsmall) smap[nsmall + (nsmall - sb - 1)] = (short)r;
                    if (r == nsmall) s_kpairs = nsmall - sb;
                }
                small_before += tot;
            }
            __syncthreads();
            const int kpairs = s_kpairs;
            __syncthreads();
            for (int q = threadIdx.x; q < kpairs; q += blockDim.x) {
                const int a = base + smap[q], b = base + smap[nsmall + q];
                double t;
                t = sx[a]; sx[a] = sx[b]; sx[b] = t;
                t = sy[a]; sy[a] = sy[b]; sy[b] = t;
                t = sz[a]; sz[a] = sz[b]; sz[b] = t;
                const int ti = sid[a]; sid[a] = sid[b]; sid[b] = ti;
            }
            nleft = (len - nsmall) == 0 ? len - 1 : nsmall;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int np[2] = {nleft, len - nleft};
            const int ip[2] = {base, base + nleft};
            const char naxis = (char)((axis + 1) % 3);
            // the right child is pushed first so the left one is split next
            for (int n = 1; n >= 0; --n) {
                if (np[n] <= maxleaf) {
                    const int l = tree_new_leaf(R, T.ipart + ip[n], np[n]);
                    if (l >= 0) R.son[2 * node + n] = 2 * l;
                } else {
                    SmallItem ch;
                    ch.span = ip[n] | (np[n] << 16);
                    ch.parent = node;
                    ch.depth = (short)(it.depth + 1);
                    ch.axis = naxis;
                    ch.side = (char)n;
                    stack[s_top++] = ch;
                }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < T.length; i += blockDim.x) {
        P.x[T.ipart + i] = sx[i];
        P.y[T.ipart + i] = sy[i];
        P.z[T.ipart + i] = sz[i];
        P.id[T.ipart + i] = sid[i];
    }
}

// ------------------------------------------------- numbering and boxes ---

// Bottom-up, nodes of depth d: subtree node and leaf counts.
__global__ void tree_count_kernel(TreeRec R, int nnode, int d) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnode; k += gridDim.x * blockDim.x) {
        if (R.depth[k] != d) continue;
        int nn = 1, nl = 0;
        for (int n = 0; n < 2; ++n) {
            const int c = R.son[2 * k + n];
            if (c < 0 || ((c & 1) && (c >> 1) >= nnode)) {  // a child never recorded
                atomicOr(&R.counters[2], TB_NUMBERING);
                continue;
            }
            if (c & 1) {
                nn += R.nn[c >> 1];
                nl += R.nl[c >> 1];
            } else {
                nl += 1;
            }
        }
        R.nn[k] = nn;
        R.nl[k] = nl;
    }
}

// Top-down, nodes of depth d (whose pre-order id, first leaf and box are
// set): the children's ids, first leaves and boxes (center_kdtree,
// src/fmm.c:273-327).
__global__ void tree_order_kernel(TreeRec R, int nnode, int d) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnode; k += gridDim.x * blockDim.x) {
        if (R.depth[k] != d) continue;
        const int axis = d % 3;
        const double split = R.split[k];
        const int pre = R.pre[k], first = R.first[k];
        const double *bx = R.box + 6 * (size_t)k;
        const int c0 = R.son[2 * k], c1 = R.son[2 * k + 1];
        const int nodes0 = (c0 & 1) ? R.nn[c0 >> 1] : 0;
        const int leaves0 = (c0 & 1) ? R.nl[c0 >> 1] : 1;
        if ((c0 & 1) && (unsigned)(c0 >> 1) >= (unsigned)nnode) {
            atomicOr(&R.counters[2], TB_NUMBERING);
            continue;
        }
        for (int n = 0; n < 2; ++n) {
            const int c = n == 0 ? c0 : c1;
            if ((c & 1) ? (unsigned)(c >> 1) >= (unsigned)nnode : (unsigned)(c >> 1) >= (unsigned)R.leaf_cap) {
                atomicOr(&R.counters[2], TB_NUMBERING);
                continue;
            }
            const int cpre = n == 0 ? pre + 1 : pre + 1 + nodes0;
            const int cfirst = n == 0 ? first : first + leaves0;
            if (c & 1) {
                const int j = c >> 1;
                R.pre[j] = cpre;
                R.first[j] = cfirst;
                double *cb = R.box + 6 * (size_t)j;
                for (int q = 0; q < 6; ++q) cb[q] = bx[q];
                if (n == 0) cb[3 + axis] = split;  // right[axis] = split
                else cb[axis] = split;             // left[axis] = split
            } else {
                R.lid[c >> 1] = cfirst;
            }
        }
    }
}

// Output tables in pre-order: node child codes in final ids, first leaves,
// centres and widths (AoS); leaf ranges, centres and widths (from the
// parent's box, the split axis cut at the split).
__global__ void tree_emit_kernel(TreeRec R, int nnode, int nleaf, int *__restrict__ son,
                                 int *__restrict__ node_first, double *__restrict__ node_center,
                                 double *__restrict__ node_width, int *__restrict__ leaf_ipart,
                                 int *__restrict__ leaf_npart, double *__restrict__ leaf_center,
                                 double *__restrict__ leaf_width) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnode; k += gridDim.x * blockDim.x) {
        const int pre = R.pre[k];
        if ((unsigned)pre >= (unsigned)nnode) {
            atomicOr(&R.counters[2], TB_NUMBERING);
            continue;
        }
        const int axis = R.depth[k] % 3;
        const double *bx = R.box + 6 * (size_t)k;
        double w[3], ctr[3];
        for (int q = 0; q < 3; ++q) {
            w[q] = __dsub_rn(bx[3 + q], bx[q]);
            ctr[q] = __dmul_rn(0.5, __dadd_rn(bx[3 + q], bx[q]));
            node_center[3 * (size_t)pre + q] = ctr[q];
            node_width[3 * (size_t)pre + q] = w[q];
        }
        node_first[pre] = R.first[k];
        const double split = R.split[k];
        for (int n = 0; n < 2; ++n) {
            const int c = R.son[2 * k + n];
            if (c & 1) {
                son[2 * pre + n] = 2 * R.pre[c >> 1] + 1;
            } else {
                const int l = c >> 1, id = R.lid[l];
                if ((unsigned)l >= (unsigned)R.leaf_cap || (unsigned)id >= (unsigned)nleaf) {
                    atomicOr(&R.counters[2], TB_NUMBERING);
                    continue;
                }
                son[2 * pre + n] = 2 * id;
                leaf_ipart[id] = R.lipart[l];
                leaf_npart[id] = R.lnpart[l];
                for (int q = 0; q < 3; ++q) {
                    leaf_width[3 * (size_t)id + q] = w[q];
                    leaf_center[3 * (size_t)id + q] = ctr[q];
                }
                if (n == 0) {
                    leaf_width[3 * (size_t)id + axis] = __dsub_rn(split, bx[axis]);
                    leaf_center[3 * (size_t)id + axis] = __dmul_rn(0.5, __dadd_rn(bx[axis], split));
                } else {
                    leaf_width[3 * (size_t)id + axis] = __dsub_rn(bx[3 + axis], split);
                    leaf_center[3 * (size_t)id + axis] = __dmul_rn(0.5, __dadd_rn(bx[3 + axis], split));
                }
            }
        }
    }
}

// leaf.active (src/fmm.c:1226-1236): 0 when the leaf holds a local particle
// (tag 1), else -1; one warp per leaf.
__global__ void tree_active_kernel(const int *__restrict__ leaf_ipart, const int *__restrict__ leaf_npart,
                                   int nleaf, const int *__restrict__ id, const int *__restrict__ tag,
                                   int *__restrict__ active) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; l < nleaf; l += nw) {
        const int ip = leaf_ipart[l], np = leaf_npart[l];
        bool any = false;
        for (int q = lane; q < np; q += 32) any = any || (tag ? tag[id[ip + q]] == 1 : true);
        any = __any_sync(0xffffffffu, any);
        if (lane == 0) active[l] = any ? 0 : -1;
    }
}

// A per-particle SoA result in tree order back to input order:
// out[d * n + perm[i]] = in[d * n + i].
__global__ void tree_unpermute_kernel(const double *__restrict__ in, const int *__restrict__ perm, int n,
                                      double *__restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = perm[i];
        if ((unsigned)j >= (unsigned)n) continue;
        out[j] = in[i];
        out[(size_t)n + j] = in[(size_t)n + i];
        out[2 * (size_t)n + j] = in[2 * (size_t)n + i];
    }
}

// Positions in tree order (SoA) from the work arrays.
__global__ void tree_pos_out_kernel(TreeParts P, int n, double *__restrict__ pos) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pos[i] = P.x[i];
        pos[(size_t)n + i] = P.y[i];
        pos[2 * (size_t)n + i] = P.z[i];
    }
}

}  // namespace p2p
