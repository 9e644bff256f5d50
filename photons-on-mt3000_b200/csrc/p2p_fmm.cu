// Far field of the short-range force on the GPU (C ABI p2p_fmm_*): the
// multipole part of PhotoNs' FMM within the cutoff sphere, the complement of
// the P2P pass on the same kd-tree.
//
//   p2m + m2m  every leaf's multipole to octupole order about its box centre
//              (p2m, src/operator.c:14-97), then each node's from its two
//              children's, shifted to its centre (m2m / walk_m2m, :102-199):
//              one thread per leaf, climbing while it is the last of a
//              node's children to finish
//   M2L walk   the reference's dual-tree recursion from (root, root)
//              (walk_task_m2l, src/fmm.c:812-957, with the acceptance test
//              of :409-479) expanded breadth first on the GPU, a level of
//              pending pairs per launch: a pair is accepted as an M2L task,
//              opened into its child pairs, or dropped
//   M2L        each sink (leaf or node), one warp, sums over its tasks in
//              increasing source order the source multipole's contribution
//              to its local expansion with the erfc-truncated kernel's derivatives
//              (m2l with LONGSHORT, src/operator.c:331-475)
//   l2l + l2p  each leaf takes its ancestors' locals down its path from the
//              root (l2l / walk_l2l, :477-606) and, if it holds a local
//              particle, evaluates the gradient at its particles (l2p,
//              :203-262; called for active leaves at src/gravity.c:427-428)
//
// Expansions are 20 coefficients per box in the reference's index order
// (inc/operator.h): 1, x, y, z, xx, xy, xz, yy, yz, zz, xxx, xxy, xxz, xyy,
// xyz, xzz, yyy, yyz, yzz, zzz. Multipole coefficients carry (-1)^n / a!b!c!
// and the locals are the derivatives, so a shift or a contraction is a sum
// over multi-indices with the monomials d^g / g! of the shift (mono below).
//
// The reference's m2l returns early when `abs(r2) <= 1e-15` with the integer
// abs() of <stdlib.h> (src/operator.c:340-344): every task with r2 < 1 in
// the caller's length unit contributes nothing. min_r2 keeps that behaviour
// selectable: 1 reproduces the reference, 1e-15 the evident intent.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "photons_p2p.h"
#include "p2p_host_shared.h"
#include "p2p_internal.h"

// This file's own instances of the scan and walk helpers (private namespace,
// so their non-template kernels do not collide with the session's).
namespace p2p_fmm_kernels {
using namespace ::p2p;
#include "p2p_pass_kernels.cuh"
#include "p2p_walk_kernels.cuh"
}  // namespace p2p_fmm_kernels

#define P2P_API extern "C" __attribute__((visibility("default")))

using namespace p2p;
using namespace p2p_fmm_kernels::p2p;

namespace {

constexpr int kNC = 20;  // coefficients per expansion (octupole)

// Exponents (a, b, c) of coefficient k.
__host__ __device__ constexpr int ex(int k, int d) {
    constexpr int t[kNC][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {1, 0, 1},
                               {0, 2, 0}, {0, 1, 1}, {0, 0, 2}, {3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0},
                               {1, 1, 1}, {1, 0, 2}, {0, 3, 0}, {0, 2, 1}, {0, 1, 2}, {0, 0, 3}};
    return t[k][d];
}
__host__ __device__ constexpr int order(int k) { return ex(k, 0) + ex(k, 1) + ex(k, 2); }
// Index of the coefficient with exponents (a, b, c), a + b + c <= 3; -1 otherwise.
__host__ __device__ constexpr int idx(int a, int b, int c) {
    if (a < 0 || b < 0 || c < 0 || a + b + c > 3) return -1;
    for (int k = 0; k < kNC; ++k)
        if (ex(k, 0) == a && ex(k, 1) == b && ex(k, 2) == c) return k;
    return -1;
}
__host__ __device__ constexpr int sum_idx(int k, int j) {
    return idx(ex(k, 0) + ex(j, 0), ex(k, 1) + ex(j, 1), ex(k, 2) + ex(j, 2));
}
__host__ __device__ constexpr int diff_idx(int k, int j) {  // k - j, -1 unless j <= k componentwise
    return idx(ex(k, 0) - ex(j, 0), ex(k, 1) - ex(j, 1), ex(k, 2) - ex(j, 2));
}

// d^g / g! for every multi-index g.
__device__ __forceinline__ void mono(double dx, double dy, double dz, double *p) {
    const double x2 = dx * dx * 0.5, y2 = dy * dy * 0.5, z2 = dz * dz * 0.5;
    p[0] = 1.0;
    p[1] = dx; p[2] = dy; p[3] = dz;
    p[4] = x2; p[5] = dx * dy; p[6] = dx * dz; p[7] = y2; p[8] = dy * dz; p[9] = z2;
    p[10] = x2 * dx * (1.0 / 3.0); p[11] = x2 * dy; p[12] = x2 * dz; p[13] = dx * y2; p[14] = dx * dy * dz;
    p[15] = dx * z2; p[16] = y2 * dy * (1.0 / 3.0); p[17] = y2 * dz; p[18] = dy * z2; p[19] = z2 * dz * (1.0 / 3.0);
}

// Multipole shift: out[a] += sum_{b <= a} m[b] p[a - b].
__device__ __forceinline__ void shift_m(const double *m, const double *p, double *out) {
#pragma unroll
    for (int a = 0; a < kNC; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < kNC; ++b)
            if (diff_idx(a, b) >= 0) s += m[b] * p[diff_idx(a, b)];
        out[a] += s;
    }
}

// Local shift: out[a] += sum_{b >= a} l[b] p[b - a].
__device__ __forceinline__ void shift_l(const double *l, const double *p, double *out) {
#pragma unroll
    for (int a = 0; a < kNC; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < kNC; ++b)
            if (diff_idx(b, a) >= 0) s += l[b] * p[diff_idx(b, a)];
        out[a] += s;
    }
}

// Derivatives to third order of phi(r) = erfc(r / (2 r_s)) / r at r = (x, y,
// z), the radial factors of m2l's LONGSHORT branch.
__device__ __forceinline__ void kernel_derivs(double x, double y, double z, double r2, double irs, double *D) {
    const double dr = sqrt(r2), ir = 1.0 / dr;
    const double ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir, ir6 = ir4 * ir2, ir7 = ir6 * ir;
    const double irs3 = irs * irs * irs, irs5 = irs3 * irs * irs;
    const double u = 0.5 * dr * irs;
    const double ec = exp(-u * u) * 0.56418958354775628695;  // exp(-u^2) / sqrt(pi)
    const double c = erfc(u);
    const double f0 = ir * c;
    const double f1 = -ir3 * (c + dr * ec * irs);
    const double f2 = 3.0 * ir5 * c + (3.0 * irs * ir4 + 0.5 * ir2 * irs3) * ec;
    const double f3 = -15.0 * ir7 * c - (15.0 * ir6 * irs + 2.5 * ir4 * irs3 + 0.25 * ir2 * irs5) * ec;
    const double v[3] = {x, y, z};
    D[0] = f0;
#pragma unroll
    for (int k = 1; k < kNC; ++k) {
        // the axes of coefficient k as an index list i <= j <= l
        int ax[3], n = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int r = 0; r < ex(k, d); ++r) ax[n++] = d;
        if (order(k) == 1) {
            D[k] = f1 * v[ax[0]];
        } else if (order(k) == 2) {
            D[k] = f2 * v[ax[0]] * v[ax[1]] + (ax[0] == ax[1] ? f1 : 0.0);
        } else {
            double t = 0.0;
            if (ax[1] == ax[2]) t += v[ax[0]];
            if (ax[0] == ax[2]) t += v[ax[1]];
            if (ax[0] == ax[1]) t += v[ax[2]];
            D[k] = f3 * v[ax[0]] * v[ax[1]] * v[ax[2]] + f2 * t;
        }
    }
}

struct FmmArgs {
    WalkArgs w;
    const double *pos;       // 3 * npart SoA, tree order
    const int *leaf_ip, *leaf_np;
    int npart;
    double mass, irs, min_r2;
    int *leaf_parent, *node_parent, *nchild, *arrive;
    double *leafM, *nodeM;   // 20 per box
    double *sinkL;           // 20 per sink: leaves then nodes
    double *leafL;           // 20 per leaf: final locals
    int *status;
};

__device__ __forceinline__ const double *box_center(const WalkArgs &w, int c) { return walk_center(w, c); }
__device__ __forceinline__ int sink_index(const WalkArgs &w, int c) { return (c & 1) ? w.nleaf + (c >> 1) : (c >> 1); }

__global__ void fmm_parent_kernel(FmmArgs f) {
    const WalkArgs &w = f.w;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < w.nnode; k += gridDim.x * blockDim.x) {
        int n = 0;
        for (int s = 0; s < 2; ++s) {
            const int c = w.son[2 * k + s];
            if (c < 0) continue;
            if (!walk_valid(w, c)) {
                atomicOr(f.status, ST_WALK_TREE);
                continue;
            }
            if (c & 1)
                f.node_parent[c >> 1] = k;
            else
                f.leaf_parent[c >> 1] = k;
            ++n;
        }
        f.nchild[k] = n;
        f.arrive[k] = 0;
    }
}

// Multipole of leaf l (p2m), then up the tree while this thread is the last
// of a node's children to arrive: the node's multipole from its children's,
// son[0]'s first.
__global__ void fmm_upward_kernel(FmmArgs f) {
    const WalkArgs &w = f.w;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < w.nleaf; l += gridDim.x * blockDim.x) {
        double M[kNC];
#pragma unroll
        for (int k = 0; k < kNC; ++k) M[k] = 0.0;
        const double *c = w.leaf_center + 3 * (size_t)l;
        const int ip = f.leaf_ip[l], np = f.leaf_np[l];
        const size_t n = (size_t)f.npart;
        for (int i = ip; i < ip + np; ++i) {
            double p[kNC];
            mono(f.pos[i] - c[0], f.pos[n + i] - c[1], f.pos[2 * n + i] - c[2], p);
#pragma unroll
            for (int k = 0; k < kNC; ++k) M[k] += ((order(k) & 1) ? -f.mass : f.mass) * p[k];
        }
#pragma unroll
        for (int k = 0; k < kNC; ++k) f.leafM[(size_t)kNC * l + k] = M[k];
        int node = f.leaf_parent[l], guard = 0;
        while (node >= 0) {
            if (++guard > 4096) {  // deeper than any tree the builders make: a cycle
                atomicOr(f.status, ST_WALK_TREE);
                break;
            }
            __threadfence();
            if (atomicAdd(&f.arrive[node], 1) != f.nchild[node] - 1) break;
            __threadfence();
            double T[kNC];
#pragma unroll
            for (int k = 0; k < kNC; ++k) T[k] = 0.0;
            const double *pc = w.node_center + 3 * (size_t)node;
            for (int s = 0; s < 2; ++s) {
                const int ch = w.son[2 * node + s];
                if (ch < 0 || !walk_valid(w, ch)) continue;
                const double *cc = box_center(w, ch);
                const double *src = (ch & 1) ? f.nodeM + (size_t)kNC * (ch >> 1) : f.leafM + (size_t)kNC * (ch >> 1);
                double m[kNC], p[kNC];
#pragma unroll
                for (int k = 0; k < kNC; ++k) m[k] = __ldcg(src + k);
                mono(pc[0] - cc[0], pc[1] - cc[1], pc[2] - cc[2], p);
                shift_m(m, p, T);
            }
#pragma unroll
            for (int k = 0; k < kNC; ++k) f.nodeM[(size_t)kNC * node + k] = T[k];
            node = f.node_parent[node];
        }
    }
}

// Whether an opened pair's child can lead to a task: two leaves (a P2P pair)
// and a pair beyond the cutoff (acceptance -1) end the recursion with none,
// so they are not written to the next level. Codes outside the tree are
// kept, for the next level to report.
__device__ __forceinline__ bool walk_child_live(const WalkArgs &w, int A, int B) {
    if (A < 0 || B < 0) return false;
    if (!walk_valid(w, A) || !walk_valid(w, B)) return true;
    if (A == B) return (A & 1) != 0;
    if (!(A & 1) && !(B & 1)) return false;
    return walk_acceptance(walk_width(w, A), walk_width(w, B), walk_center(w, A), walk_center(w, B), w.cutoff,
                           w.open_angle) != -1;
}

// One level of the M2L walk: each pending pair is accepted (a task), opened
// into its child pairs, or dropped, as walk_task_m2l decides; children that
// cannot lead to a task are not kept (walk_child_live). Output slots come
// from warp-aggregated atomics; a level whose outputs exceed the buffers
// only counts them (the host grows the buffers and repeats it).
__global__ void fmm_walk_kernel(WalkArgs w, const int2 *__restrict__ in, int nin, int2 *__restrict__ out,
                                long long out_cap, unsigned long long *nout, int2 *__restrict__ tasks,
                                long long task_cap, unsigned long long *ntask, int *status) {
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + threadIdx.x - lane; base < nin; base += stride) {
        const int i = base + lane;
        int2 kids[4];
        int nk = 0, nt = 0;
        int2 task = make_int2(0, 0);
        if (i < nin) {
            const int A = in[i].x, B = in[i].y;
            const bool okA = A >= 0 && walk_valid(w, A), okB = B >= 0 && walk_valid(w, B);
            if ((A >= 0 && !okA) || (B >= 0 && !okB)) atomicOr(status, ST_WALK_TREE);
            if (okA && okB) {
                if (A == B) {
                    if (A & 1) {
                        const int s0 = w.son[2 * (A >> 1)], s1 = w.son[2 * (A >> 1) + 1];
                        kids[0] = make_int2(s0, s0);
                        kids[1] = make_int2(s0, s1);
                        kids[2] = make_int2(s1, s0);
                        kids[3] = make_int2(s1, s1);
                        nk = 4;
                    }
                } else if ((A & 1) || (B & 1)) {
                    const double *wa = walk_width(w, A), *wb = walk_width(w, B);
                    const int flag = walk_acceptance(wa, wb, walk_center(w, A), walk_center(w, B), w.cutoff,
                                                     w.open_angle);
                    if (flag == 1) {
                        task = make_int2(A, B);
                        nt = 1;
                    } else if (flag == 0) {
                        bool openA;
                        if (!(A & 1))
                            openA = false;
                        else if (!(B & 1))
                            openA = true;
                        else  // both nodes: open the one with the larger summed width
                            openA = __dadd_rn(__dadd_rn(wa[0], wa[1]), wa[2]) >
                                    __dadd_rn(__dadd_rn(wb[0], wb[1]), wb[2]);
                        if (openA) {
                            kids[0] = make_int2(w.son[2 * (A >> 1)], B);
                            kids[1] = make_int2(w.son[2 * (A >> 1) + 1], B);
                        } else {
                            kids[0] = make_int2(A, w.son[2 * (B >> 1)]);
                            kids[1] = make_int2(A, w.son[2 * (B >> 1) + 1]);
                        }
                        nk = 2;
                    }
                }
            }
        }
        {  // keep the live children only
            int m = 0;
            for (int c = 0; c < nk; ++c)
                if (walk_child_live(w, kids[c].x, kids[c].y)) kids[m++] = kids[c];
            nk = m;
        }
        // warp-aggregated output slots
        int kin = nk, tin = nt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int a = __shfl_up_sync(kFull, kin, off), b = __shfl_up_sync(kFull, tin, off);
            if (lane >= off) {
                kin += a;
                tin += b;
            }
        }
        unsigned long long kbase = 0, tbase = 0;
        if (lane == 31) {
            kbase = kin ? atomicAdd(nout, (unsigned long long)kin) : 0ull;
            tbase = tin ? atomicAdd(ntask, (unsigned long long)tin) : 0ull;
        }
        kbase = __shfl_sync(kFull, kbase, 31);
        tbase = __shfl_sync(kFull, tbase, 31);
        const long long ko = (long long)kbase + kin - nk, to = (long long)tbase + tin - nt;
        for (int k = 0; k < nk; ++k)
            if (ko + k < out_cap) out[ko + k] = kids[k];
        if (nt && to < task_cap) tasks[to] = task;
    }
}

__global__ void fmm_task_count_kernel(WalkArgs w, const int2 *__restrict__ tasks, long long nt, int *count) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += (long long)gridDim.x * blockDim.x)
        atomicAdd(&count[sink_index(w, tasks[t].x)], 1);
}

__global__ void fmm_task_fill_kernel(WalkArgs w, const int2 *__restrict__ tasks, long long nt,
                                     const int64_t *__restrict__ off, int *fill, int *seg) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += (long long)gridDim.x * blockDim.x) {
        const int s = sink_index(w, tasks[t].x);
        seg[off[s] + atomicAdd(&fill[s], 1)] = tasks[t].y;
    }
}

// M2L: one warp per sink. The sink's source codes are put in increasing
// order (a bitonic sort in shared memory up to kM2LSort codes; above that a
// rank sort from seg into seg2), lane j takes the sorted tasks j, j + 32, ...
// and the lanes' partial locals are summed by a fixed shuffle tree: the same
// order on every run, whatever order the walk emitted the tasks in.
constexpr int kM2LWarps = 4;
constexpr int kM2LSort = 2048;

__global__ void __launch_bounds__(32 * kM2LWarps)
fmm_m2l_kernel(FmmArgs f, const int64_t *__restrict__ off, const int *__restrict__ seg, int *__restrict__ seg2,
               unsigned long long *applied) {
    __shared__ int sbuf[kM2LWarps][kM2LSort];
    const WalkArgs &w = f.w;
    const int lane = threadIdx.x & 31;
    int *buf = sbuf[threadIdx.x >> 5];
    const int nsink = w.nleaf + w.nnode;
    const int nwarp = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsink; s += nwarp) {
        const int64_t a = off[s], e = off[s + 1];
        if (a < 0 || e < a || e > off[nsink]) {  // offsets out of order: record it, skip the sink
            if (lane == 0) atomicOr(f.status, ST_WALK_ROW);
            continue;
        }
        const int k = (int)(e - a);
        const int *src = buf;
        if (k <= kM2LSort) {
            int p = 1;
            while (p < k) p <<= 1;
            for (int i = lane; i < p; i += 32) buf[i] = i < k ? seg[a + i] : INT_MAX;
            __syncwarp();
            for (int size = 2; size <= p; size <<= 1) {
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int i = lane; i < p; i += 32) {
                        const int j = i ^ stride;
                        if (j > i) {
                            const int x = buf[i], y = buf[j];
                            if ((x > y) == ((i & size) == 0)) {
                                buf[i] = y;
                                buf[j] = x;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        } else {
            for (int i = lane; i < k; i += 32) {
                const int v = seg[a + i];
                int r = 0;
                for (int j = 0; j < k; ++j) {
                    const int x = seg[a + j];
                    r += (x < v) || (x == v && j < i);
                }
                seg2[a + r] = v;
            }
            __syncwarp();
            src = seg2 + a;
        }
        double L[kNC];
#pragma unroll
        for (int c = 0; c < kNC; ++c) L[c] = 0.0;
        const int code = s < w.nleaf ? 2 * s : 2 * (s - w.nleaf) + 1;
        const double *cs = box_center(w, code);
        unsigned used = 0;
        for (int t = lane; t < k; t += 32) {
            const int sc = src[t];
            const double *cb = box_center(w, sc);
            const double x = cs[0] - cb[0], y = cs[1] - cb[1], z = cs[2] - cb[2];
            const double r2 = x * x + y * y + z * z;
            if (!(r2 >= f.min_r2)) continue;
            ++used;
            const double *Msrc = (sc & 1) ? f.nodeM + (size_t)kNC * (sc >> 1) : f.leafM + (size_t)kNC * (sc >> 1);
            double m[kNC], D[kNC];
#pragma unroll
            for (int c = 0; c < kNC; ++c) m[c] = Msrc[c];
            kernel_derivs(x, y, z, r2, f.irs, D);
#pragma unroll
            for (int c = 0; c < kNC; ++c) {
                double acc = 0.0;
#pragma unroll
                for (int j = 0; j < kNC; ++j)
                    if (sum_idx(c, j) >= 0) acc += m[j] * D[sum_idx(c, j)];
                L[c] += acc;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int c = 0; c < kNC; ++c) L[c] += __shfl_down_sync(kFull, L[c], o);
            used += __shfl_down_sync(kFull, used, o);
        }
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < kNC; ++c) f.sinkL[(size_t)kNC * s + c] = L[c];
            if (used) atomicAdd(applied, (unsigned long long)used);
        }
        __syncwarp();  // the shared buffer is rewritten by the next sink
    }
}

// Locals down each leaf's path from the root, then the gradient at the
// leaf's particles (active leaves; zero for the others).
__global__ void fmm_downward_kernel(FmmArgs f, double *__restrict__ acc) {
    const WalkArgs &w = f.w;
    const size_t n = (size_t)f.npart;
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < w.nleaf; l += gridDim.x * blockDim.x) {
        double L[kNC];
        int A;
        if (w.nnode > 0) {
            A = 1;  // the root node
#pragma unroll
            for (int k = 0; k < kNC; ++k) L[k] = f.sinkL[(size_t)kNC * w.nleaf + k];
            int guard = 0;
            while ((A & 1) && guard++ < 4096) {
                const int ch = walk_child_toward(w, A, l);
                if (ch < 0 || !walk_valid(w, ch)) {
                    atomicOr(f.status, ST_WALK_TREE);
                    break;
                }
                const double *pc = box_center(w, A), *cc = box_center(w, ch);
                double T[kNC], p[kNC];
                const double *own = f.sinkL + (size_t)kNC * sink_index(w, ch);
#pragma unroll
                for (int k = 0; k < kNC; ++k) T[k] = own[k];
                mono(cc[0] - pc[0], cc[1] - pc[1], cc[2] - pc[2], p);
                shift_l(L, p, T);
#pragma unroll
                for (int k = 0; k < kNC; ++k) L[k] = T[k];
                A = ch;
            }
            if (A != 2 * l) atomicOr(f.status, ST_WALK_TREE);
        } else {
#pragma unroll
            for (int k = 0; k < kNC; ++k) L[k] = f.sinkL[(size_t)kNC * l + k];
        }
#pragma unroll
        for (int k = 0; k < kNC; ++k) f.leafL[(size_t)kNC * l + k] = L[k];
        const int ip = f.leaf_ip[l], np = f.leaf_np[l];
        const bool active = w.leaf_active[l] >= 0;
        const double *c = w.leaf_center + 3 * (size_t)l;
        for (int i = ip; i < ip + np; ++i) {
            double g[3] = {0.0, 0.0, 0.0};
            if (active) {
                double p[kNC];
                mono(f.pos[i] - c[0], f.pos[n + i] - c[1], f.pos[2 * n + i] - c[2], p);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    // d/dx_d of sum_b L[b] x^b / b!: sum over b with b_d >= 1 of L[b] x^(b - e_d) / (b - e_d)!
#pragma unroll
                    for (int b = 1; b < kNC; ++b) {
                        const int r = idx(ex(b, 0) - (d == 0), ex(b, 1) - (d == 1), ex(b, 2) - (d == 2));
                        if (r >= 0) g[d] += L[b] * p[r];
                    }
                }
            }
            acc[i] = g[0];
            acc[n + i] = g[1];
            acc[2 * n + i] = g[2];
        }
    }
}

struct DevBufF {
    void *p = nullptr;
    size_t cap = 0;
};

int grow(DevBufF &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return P2P_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    const size_t want = bytes + bytes / 4;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        return report_error(P2P_ERR_NOMEM, "FMM scratch allocation failed");
    }
    b.cap = want;
    return P2P_OK;
}

int fail_cuda(cudaError_t e, const char *what) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return report_error(P2P_ERR_CUDA, msg);
}

int blocks_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max(1LL, std::min(b, 148LL * 32));
}

}  // namespace

struct p2p_fmm {
    int device = 0;
    cudaStream_t stream = nullptr;
    DevBufF parents, leafM, nodeM, sinkL, leafL, front[2], tasks, counts, off, tiles, seg, seg2, ctrl;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    long long n_m2l = 0, n_applied = 0;
    int levels = 0, nleaf = 0, nnode = 0;
};

#define FMM_TRY(expr)                \
    do {                             \
        int _s = (expr);             \
        if (_s != P2P_OK) return _s; \
    } while (0)
#define FMM_CUDA(expr, what)                        \
    do {                                            \
        cudaError_t _e = (expr);                    \
        if (_e != cudaSuccess) return fail_cuda(_e, what); \
    } while (0)

P2P_API int p2p_fmm_create(p2p_session *s, p2p_fmm **out) {
    if (!s || !out) return report_error(P2P_ERR_ARG, "null argument");
    *out = nullptr;
    FMM_CUDA(cudaSetDevice(session_device(s)), "cudaSetDevice");
    p2p_fmm *f = new p2p_fmm();
    f->device = session_device(s);
    f->stream = (cudaStream_t)p2p_session_stream(s);
    for (cudaEvent_t &e : f->ev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            p2p_fmm_destroy(f);
            return report_error(P2P_ERR_CUDA, "FMM event creation failed");
        }
    }
    *out = f;
    return P2P_OK;
}

P2P_API int p2p_fmm_destroy(p2p_fmm *f) {
    if (!f) return P2P_OK;
    cudaSetDevice(f->device);
    cudaStreamSynchronize(f->stream);
    DevBufF *bufs[] = {&f->parents, &f->leafM, &f->nodeM, &f->sinkL, &f->leafL, &f->front[0], &f->front[1],
                       &f->tasks, &f->counts, &f->off, &f->tiles, &f->seg, &f->seg2, &f->ctrl};
    for (DevBufF *b : bufs)
        if (b->p) cudaFree(b->p);
    for (cudaEvent_t e : f->ev)
        if (e) cudaEventDestroy(e);
    delete f;
    return P2P_OK;
}

P2P_API int p2p_fmm_far(p2p_fmm *f, const p2p_walk_tree *t, int npart, const double *d_pos, const int *d_leaf_ipart,
                        const int *d_leaf_npart, double mass, double split_radius, double cutoff, double open_angle,
                        double min_r2, double *d_acc) {
    if (!f || !t) return report_error(P2P_ERR_ARG, "null argument");
    if (npart < 0 || t->nleaf < 0 || t->nnode < 0) return report_error(P2P_ERR_ARG, "negative size");
    if (npart > 0 && (!d_pos || !d_acc || !d_leaf_ipart || !d_leaf_npart))
        return report_error(P2P_ERR_ARG, "null device array");
    if ((t->nnode > 0 && (!t->son || !t->node_first || !t->node_center || !t->node_width)) ||
        (t->nleaf > 0 && (!t->leaf_center || !t->leaf_width || !t->leaf_active)))
        return report_error(P2P_ERR_ARG, "null tree array");
    if (!(split_radius > 0.0) || !(cutoff >= 0.0) || !(open_angle >= 0.0) || !(min_r2 >= 0.0) ||
        !std::isfinite(mass))
        return report_error(P2P_ERR_ARG, "bad split radius, cutoff, open angle, min_r2 or mass");
    FMM_CUDA(cudaSetDevice(f->device), "cudaSetDevice");
    const int nleaf = t->nleaf, nnode = t->nnode, nsink = nleaf + nnode;
    f->nleaf = nleaf;
    f->nnode = nnode;
    f->n_m2l = f->n_applied = 0;
    f->levels = 0;
    cudaStream_t st = f->stream;
    const int threads = 256;
    FMM_CUDA(cudaEventRecord(f->ev[0], st), "FMM");
    if (nleaf == 0) {
        if (npart) FMM_CUDA(cudaMemsetAsync(d_acc, 0, sizeof(double) * 3 * (size_t)npart, st), "FMM");
        for (int k = 1; k < 5; ++k) FMM_CUDA(cudaEventRecord(f->ev[k], st), "FMM");
        return P2P_OK;
    }
    FMM_TRY(grow(f->parents, sizeof(int) * ((size_t)nleaf + 3 * (size_t)nnode)));
    FMM_TRY(grow(f->leafM, sizeof(double) * kNC * (size_t)nleaf));
    FMM_TRY(grow(f->nodeM, sizeof(double) * kNC * (size_t)std::max(nnode, 1)));
    FMM_TRY(grow(f->sinkL, sizeof(double) * kNC * (size_t)nsink));
    FMM_TRY(grow(f->leafL, sizeof(double) * kNC * (size_t)nleaf));
    FMM_TRY(grow(f->counts, sizeof(int) * 2 * (size_t)nsink));
    FMM_TRY(grow(f->off, sizeof(int64_t) * ((size_t)nsink + 1)));
    FMM_TRY(grow(f->tiles, sizeof(int64_t) * (((size_t)nsink + kScanTile - 1) / kScanTile + 1)));
    FMM_TRY(grow(f->ctrl, 64));
    FmmArgs a;
    a.w.nnode = nnode;
    a.w.nleaf = nleaf;
    a.w.son = t->son;
    a.w.node_first = t->node_first;
    a.w.leaf_active = t->leaf_active;
    a.w.node_center = t->node_center;
    a.w.node_width = t->node_width;
    a.w.leaf_center = t->leaf_center;
    a.w.leaf_width = t->leaf_width;
    a.w.cutoff = cutoff;
    a.w.open_angle = open_angle;
    a.pos = d_pos;
    a.leaf_ip = d_leaf_ipart;
    a.leaf_np = d_leaf_npart;
    a.npart = npart;
    a.mass = mass;
    a.irs = 1.0 / split_radius;
    a.min_r2 = min_r2;
    int *par = (int *)f->parents.p;
    a.leaf_parent = par;
    a.node_parent = par + nleaf;
    a.nchild = par + nleaf + nnode;
    a.arrive = par + nleaf + 2 * nnode;
    a.leafM = (double *)f->leafM.p;
    a.nodeM = (double *)f->nodeM.p;
    a.sinkL = (double *)f->sinkL.p;
    a.leafL = (double *)f->leafL.p;
    unsigned long long *ctrl = (unsigned long long *)f->ctrl.p;  // [0] nout [1] ntask [2] applied [3] status
    a.status = (int *)(ctrl + 3);
    FMM_CUDA(cudaMemsetAsync(ctrl, 0, 64, st), "FMM");
    FMM_CUDA(cudaMemsetAsync(par, 0xff, sizeof(int) * ((size_t)nleaf + nnode), st), "FMM");  // parents -1
    if (nnode) fmm_parent_kernel<<<blocks_for(nnode, threads), threads, 0, st>>>(a);
    fmm_upward_kernel<<<blocks_for(nleaf, threads), threads, 0, st>>>(a);
    FMM_CUDA(cudaEventRecord(f->ev[1], st), "FMM upward");

    // M2L walk, one level per launch
    long long nin = 0, ntask = 0;
    if (nnode) {
        long long fcap = std::max<long long>(4LL * nsink, 1024), tcap = std::max<long long>(4LL * nsink, 1024);
        FMM_TRY(grow(f->front[0], sizeof(int2) * (size_t)fcap));
        FMM_TRY(grow(f->front[1], sizeof(int2) * (size_t)fcap));
        FMM_TRY(grow(f->tasks, sizeof(int2) * (size_t)tcap));
        const int2 root = make_int2(1, 1);
        FMM_CUDA(cudaMemcpyAsync(f->front[0].p, &root, sizeof(int2), cudaMemcpyHostToDevice, st), "FMM walk");
        nin = 1;
        int cur = 0;
        unsigned long long h[2];
        while (nin > 0) {
            if (++f->levels > 4096) return report_error(P2P_ERR_CAPACITY, "FMM walk: too many levels");
            const unsigned long long t0 = (unsigned long long)ntask;
            FMM_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(unsigned long long), st), "FMM walk");
            FMM_CUDA(cudaMemcpyAsync(ctrl + 1, &t0, sizeof(t0), cudaMemcpyHostToDevice, st), "FMM walk");
            fmm_walk_kernel<<<blocks_for(nin, threads), threads, 0, st>>>(
                a.w, (const int2 *)f->front[cur].p, (int)nin, (int2 *)f->front[cur ^ 1].p, fcap, ctrl,
                (int2 *)f->tasks.p, tcap, ctrl + 1, a.status);
            FMM_CUDA(cudaMemcpyAsync(h, ctrl, sizeof(h), cudaMemcpyDeviceToHost, st), "FMM walk");
            FMM_CUDA(cudaStreamSynchronize(st), "FMM walk");
            const long long nout = (long long)h[0], nt = (long long)h[1];
            if (nout > fcap || nt > tcap) {
                // grow and repeat the level (the input frontier is kept)
                if (nout > fcap) {
                    fcap = nout + nout / 2;
                    DevBufF keep = f->front[cur];
                    f->front[cur] = DevBufF();
                    FMM_TRY(grow(f->front[cur], sizeof(int2) * (size_t)fcap));
                    FMM_CUDA(cudaMemcpyAsync(f->front[cur].p, keep.p, sizeof(int2) * (size_t)nin,
                                             cudaMemcpyDeviceToDevice, st), "FMM walk");
                    FMM_CUDA(cudaStreamSynchronize(st), "FMM walk");
                    cudaFree(keep.p);
                    FMM_TRY(grow(f->front[cur ^ 1], sizeof(int2) * (size_t)fcap));
                }
                if (nt > tcap) {
                    tcap = nt + nt / 2;
                    DevBufF keep = f->tasks;
                    f->tasks = DevBufF();
                    FMM_TRY(grow(f->tasks, sizeof(int2) * (size_t)tcap));
                    if (ntask)
                        FMM_CUDA(cudaMemcpyAsync(f->tasks.p, keep.p, sizeof(int2) * (size_t)ntask,
                                                 cudaMemcpyDeviceToDevice, st), "FMM walk");
                    FMM_CUDA(cudaStreamSynchronize(st), "FMM walk");
                    cudaFree(keep.p);
                }
                --f->levels;
                continue;
            }
            ntask = nt;
            nin = nout;
            cur ^= 1;
        }
    }
    f->n_m2l = ntask;
    FMM_CUDA(cudaEventRecord(f->ev[2], st), "FMM walk");

    // M2L: tasks grouped by sink, each sink's sum in increasing source order
    int *count = (int *)f->counts.p, *fill = count + nsink;
    int64_t *off = (int64_t *)f->off.p;
    FMM_TRY(grow(f->seg, sizeof(int) * (size_t)std::max<long long>(ntask, 1)));
    FMM_TRY(grow(f->seg2, sizeof(int) * (size_t)std::max<long long>(ntask, 1)));
    FMM_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * 2 * (size_t)nsink, st), "FMM m2l");
    if (ntask)
        fmm_task_count_kernel<<<blocks_for(ntask, threads), threads, 0, st>>>(a.w, (const int2 *)f->tasks.p, ntask,
                                                                               count);
    const int ntiles = (int)(((int64_t)nsink + kScanTile - 1) / kScanTile);
    int64_t *tiles = (int64_t *)f->tiles.p;
    scan_tiles_kernel<<<ntiles, kScanThreads, 0, st>>>(count, nsink, off, tiles);
    scan_sums_kernel<<<1, kScanThreads, 0, st>>>(tiles, ntiles, off + nsink);
    // one thread per element (the kernel has no grid-stride loop)
    scan_add_kernel<<<(nsink + threads - 1) / threads, threads, 0, st>>>(off, nsink, tiles);
    if (ntask)
        fmm_task_fill_kernel<<<blocks_for(ntask, threads), threads, 0, st>>>(a.w, (const int2 *)f->tasks.p, ntask,
                                                                              off, fill, (int *)f->seg.p);
    fmm_m2l_kernel<<<(int)std::min<long long>(((long long)nsink + kM2LWarps - 1) / kM2LWarps, 148LL * 16),
                     32 * kM2LWarps, 0, st>>>(a, off, (const int *)f->seg.p, (int *)f->seg2.p, ctrl + 2);
    FMM_CUDA(cudaEventRecord(f->ev[3], st), "FMM m2l");
    fmm_downward_kernel<<<blocks_for(nleaf, 128), 128, 0, st>>>(a, d_acc);
    FMM_CUDA(cudaEventRecord(f->ev[4], st), "FMM downward");
    FMM_CUDA(cudaGetLastError(), "FMM launch");
    unsigned long long h2[2];
    FMM_CUDA(cudaMemcpyAsync(h2, ctrl + 2, sizeof(h2), cudaMemcpyDeviceToHost, st), "FMM");
    FMM_CUDA(cudaStreamSynchronize(st), "FMM");
    f->n_applied = (long long)h2[0];
    count_launches(4 + f->levels + (ntask ? 5 : 3));
    if ((int)h2[1] & ST_WALK_TREE) return report_error(P2P_ERR_ARG, "FMM: a child code outside the tree");
    if ((int)h2[1] & ST_WALK_ROW) return report_error(P2P_ERR_STATE, "FMM: M2L task offsets out of order");
    return P2P_OK;
}

P2P_API int p2p_fmm_stats(p2p_fmm *f, int64_t *n_m2l, int64_t *n_applied, int *levels, float *ms) {
    if (!f) return report_error(P2P_ERR_ARG, "null argument");
    if (n_m2l) *n_m2l = f->n_m2l;
    if (n_applied) *n_applied = f->n_applied;
    if (levels) *levels = f->levels;
    if (ms) {
        cudaError_t e = cudaEventSynchronize(f->ev[4]);
        for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventElapsedTime(&ms[k], f->ev[k], f->ev[k + 1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[4], f->ev[0], f->ev[4]);
        if (e != cudaSuccess) return fail_cuda(e, "FMM timings");
    }
    return P2P_OK;
}

P2P_API int p2p_fmm_download(p2p_fmm *f, double *leaf_M, double *leaf_L) {
    if (!f) return report_error(P2P_ERR_ARG, "null argument");
    FMM_CUDA(cudaSetDevice(f->device), "cudaSetDevice");
    FMM_CUDA(cudaStreamSynchronize(f->stream), "FMM download");
    const size_t bytes = sizeof(double) * kNC * (size_t)f->nleaf;
    if (leaf_M && bytes) FMM_CUDA(cudaMemcpy(leaf_M, f->leafM.p, bytes, cudaMemcpyDeviceToHost), "FMM download");
    if (leaf_L && bytes) FMM_CUDA(cudaMemcpy(leaf_L, f->leafL.p, bytes, cudaMemcpyDeviceToHost), "FMM download");
    return P2P_OK;
}
