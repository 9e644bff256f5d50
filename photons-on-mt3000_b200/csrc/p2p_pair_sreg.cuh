// Sink-register pair kernel of the FP32 forms (P2P_VARIANT_SINK_REGS).
//
// A slice of ns <= 8 SPL sink particles of a sink leaf (32 with SPL = 4,
// P2P_VARIANT_SINK_REGS; 64 with SPL = 8, P2P_VARIANT_SINK_REGS8, whose
// 168 registers leave 3 blocks per SM) is split into G = ceil(ns / SPL)
// groups of SPL sinks; lane (g, j) = (lane % G, lane / G), j < J = floor(32 /
// G), keeps group g's sinks in
// registers as SPL / 2 packed sink pairs and takes the staged sources j,
// j + J, j + 2J, ... of the row. A staged source is read as two 16-byte
// shared-memory loads (stored pre-duplicated: (x, x, y, y), (z, z, w,
// index)) and evaluated against the lane's sinks with sm_100's packed FP32
// instructions (pair_split_x2n): no
// per-pair shared loads of sinks, no predicated sink blocks, so the FP32 pipe
// rather than instruction issue bounds the loop.
//
// Staging classifies every source of the row against the bounding box of the
// slice's sinks (in the sink frame, FP32): a source whose lower bound on u
// exceeds uout is dropped (every pair with the slice lies beyond the cutoff:
// the result is the same as evaluating it), one whose upper bound stays below
// uin goes to the front of the stage (no cutoff test), the others to the back
// (cutoff test and cutoff-band flags). The two regions are consumed by
// separate loops, so the test is paid only where it can matter, with no
// per-step vote. Staging takes the row's sources P2P_SREG_ROUNDS x 32 at a
// time and issues all their global loads before it classifies and stores
// any, so the loads' latency is paid once per group. A consume before the
// row's end runs whole iterations only (two sources for every lane) and
// leaves the remainder of each region in place for the next one; the
// per-lane guarded tail runs once, at the end of the slice.
//
// With PairArgs::leaf_warps = W > 1 a sink leaf is W work items, each a
// contiguous share of the row's list entries, whose partial forces are added
// with FP64 atomics (a long row is spread over W warps).
//
// Band pairs (FP32 u within the band around x_cut^2) are re-decided from FP64
// positions by the lane that met them (band_pair), as in the other packed
// kernels. FP32 partials of a consume (at most stage/J sources per lane) are
// added to per-lane accumulators in shared memory (FP64, Kahan FP32 or FP32);
// at the slice's end lane i < ns sums sink i's J phase accumulators in phase
// order. Summation order is fixed: results repeat bit for bit.
#pragma once

#include "p2p_launch.h"
#include "p2p_pair_kernels.cuh"

namespace p2p {

#ifndef P2P_SREG_MINBLOCKS
#define P2P_SREG_MINBLOCKS 4  // resident 128-thread blocks per SM the register budget targets
#endif

// Per-lane accumulators in shared memory: value k of lane l at base[k * 32 + l].
template <int ACC> struct SregAcc;
template <> struct SregAcc<ACC_F64> {
    using T = double;
    using Sum = double;
    __device__ __forceinline__ static void zero(T &v) { v = 0.0; }
    __device__ __forceinline__ static void add(T &v, float x) { v += (double)x; }
    __device__ __forceinline__ static Sum value(const T &v) { return v; }
};
template <> struct SregAcc<ACC_KAHAN> {
    using T = float2;  // running sum, carried rounding error
    using Sum = float;
    __device__ __forceinline__ static void zero(T &v) { v = make_float2(0.f, 0.f); }
    __device__ __forceinline__ static void add(T &v, float x) {
        const float y = x - v.y;
        const float t = v.x + y;
        v.y = (t - v.x) - y;
        v.x = t;
    }
    __device__ __forceinline__ static Sum value(const T &v) { return v.x - v.y; }
};
template <> struct SregAcc<ACC_F32> {
    using T = float;
    using Sum = float;
    __device__ __forceinline__ static void zero(T &v) { v = 0.f; }
    __device__ __forceinline__ static void add(T &v, float x) { v += x; }
    __device__ __forceinline__ static Sum value(const T &v) { return v; }
};

#ifndef P2P_SREG_ROUNDS
#define P2P_SREG_ROUNDS 4  // staging rounds of 32 sources whose loads are in flight together
#endif
constexpr int kSregRounds = P2P_SREG_ROUNDS;
static_assert(32 * kSregRounds <= kSregMinStage, "a staging group must fit in the smallest stage");

// 3 values per sink per lane, at most 8 bytes each
__host__ __device__ constexpr int sreg_acc_bytes(int spl) { return 3 * spl * 32 * 8; }

// Staging context of one warp, kept in shared memory rather than registers
// so that none of it is live while the warp evaluates pairs: the current
// batch of 32 list entries (per lane: its entry's particle range, FP32 frame
// offset, whether it lies wholly inside the cutoff), the sink leaf's frame
// and half-extents, and the bounding box of the sink slice.
struct SregCtx {
    int sip[32], snp[32], ein[32];
    float ox[32], oy[32], oz[32];
    double mcx, mcy, mcz;
    float mhx, mhy, mhz;
    float bcx, bcy, bcz, bhx, bhy, bhz;
};
constexpr int kSregCtxBytes = 1024;
static_assert(sizeof(SregCtx) <= kSregCtxBytes, "staging context");

// Shared memory of one warp: staged sources (32 B each), the lane
// accumulators, the staging context.
__host__ __device__ constexpr size_t sreg_warp_bytes(int cap, int spl) {
    return (size_t)cap * 32 + sreg_acc_bytes(spl) + kSregCtxBytes;
}

// The lane's SPL sinks as SPL / 2 packed pairs and their FP32 partial forces.
template <int SPL>
struct SregLane {
    static constexpr int P = SPL / 2;
    float2 px[P], py[P], pz[P];  // negated coordinates of sinks (SPL g + 2 p, SPL g + 2 p + 1)
    float2 ax[P], ay[P], az[P];  // partials of the pairs
    int sfirst, slast;           // particle index of sink SPL g, and of the slice's last sink
};

// One staged source (pre-duplicated layout) against the lane's sinks.
template <int SOFT, bool MASSES, int NC, bool CHECK, int SPL>
__device__ __forceinline__ void sreg_eval(const float4 A, const float4 B, SregLane<SPL> &L, const PairArgs &a,
                                          const float2 eps2v, const float2 negu0v, bool &amb) {
    const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y);
#pragma unroll
    for (int p = 0; p < SPL / 2; ++p)
        pair_split_x2n<SOFT, MASSES, NC, CHECK>(sx, sy, sz, B.z, L.px[p], L.py[p], L.pz[p], a, eps2v, negu0v,
                                                L.ax[p], L.ay[p], L.az[p], amb);
}

// Re-decides the lane's band pairs with one staged source from FP64 positions.
template <int SOFT, bool MASSES, int NC, int SPL>
__device__ __forceinline__ void sreg_band(const float4 A, const float4 B, SregLane<SPL> &L, const PairArgs &a) {
    const float4 src = make_float4(A.x, A.z, B.x, B.z);
    const int isrc = __float_as_int(B.w);
    float3 cb;
#pragma unroll
    for (int p = 0; p < SPL / 2; ++p) {
        if (band_pair<SOFT, MASSES, NC>(src, L.px[p].x, L.py[p].x, L.pz[p].x, isrc, min(L.sfirst + 2 * p, L.slast),
                                        a, &cb)) {
            L.ax[p].x += cb.x; L.ay[p].x += cb.y; L.az[p].x += cb.z;
        }
        if (band_pair<SOFT, MASSES, NC>(src, L.px[p].y, L.py[p].y, L.pz[p].y, isrc,
                                        min(L.sfirst + 2 * p + 1, L.slast), a, &cb)) {
            L.ax[p].y += cb.x; L.ay[p].y += cb.y; L.az[p].y += cb.z;
        }
    }
}

// Consumes staged sources [base, base + n): lane phase j takes slots
// base + j + k J, two per iteration. Full iterations (every lane busy) run
// without per-lane guards; with tail the last, partial iteration follows,
// guarded per lane. Returns the sources consumed (n with tail, else the
// whole iterations' 2 J k).
template <int SOFT, bool MASSES, int NC, bool CHECK, int SPL>
__device__ __forceinline__ int sreg_region(const float4 *stage, const int base, const int n, const int j, const int J,
                                           const bool owner, const bool tail, SregLane<SPL> &L, const PairArgs &a,
                                           const float2 eps2v, const float2 negu0v) {
    const int step = 2 * J;
    const int full = n / step;
    const float4 *p = stage + 2 * (base + j);
    for (int ib = 0; ib < full; ib += 32) {
        const int nb = min(32, full - ib);
        unsigned ambbits = 0;
#pragma unroll 1
        for (int k = 0; k < nb; ++k) {
            const float4 A0 = p[0], B0 = p[1], A1 = p[2 * J], B1 = p[2 * J + 1];
            p += 2 * step;
            bool amb = false;
            sreg_eval<SOFT, MASSES, NC, CHECK, SPL>(A0, B0, L, a, eps2v, negu0v, amb);
            sreg_eval<SOFT, MASSES, NC, CHECK, SPL>(A1, B1, L, a, eps2v, negu0v, amb);
            if (CHECK) ambbits |= amb ? (1u << k) : 0u;
        }
        if (CHECK && owner) {
            while (ambbits) {  // rare: pairs in the cutoff band
                const int k = __ffs(ambbits) - 1;
                ambbits &= ambbits - 1;
                const int s = base + j + (ib + k) * step;
                sreg_band<SOFT, MASSES, NC, SPL>(stage[2 * s], stage[2 * s + 1], L, a);
                sreg_band<SOFT, MASSES, NC, SPL>(stage[2 * (s + J)], stage[2 * (s + J) + 1], L, a);
            }
        }
    }
    if (!tail) return full * step;
    const int k0 = full * step + j;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = k0 + h * J;
        if (k < n) {
            const int s = base + k;
            const float4 A = stage[2 * s], B = stage[2 * s + 1];
            bool amb = false;
            sreg_eval<SOFT, MASSES, NC, CHECK, SPL>(A, B, L, a, eps2v, negu0v, amb);
            if (CHECK && owner && amb) sreg_band<SOFT, MASSES, NC, SPL>(A, B, L, a);
        }
    }
    return n;
}

// Consumes the stage: the inside region [0, ni) without the cutoff test, the
// test region [cap - nc, cap) with it. With fin both are emptied; otherwise
// whole iterations only, taken from the inside region's top and the test
// region's bottom, so each remainder stays where the next sources join it
// ([0, ni) and [cap - nc, cap) again). The FP32 partials go into the lane's
// shared-memory accumulators.
template <int SOFT, bool MASSES, int ACC, int NC, int SPL>
__device__ __forceinline__ void sreg_consume(const float4 *stage, typename SregAcc<ACC>::T *accs, const int cap,
                                             int &ni, int &nc, const bool fin, const int j, const int J,
                                             const bool owner, SregLane<SPL> &L, const PairArgs &a, const float2 eps2v,
                                             const float2 negu0v) {
    using SA = SregAcc<ACC>;
    const int lane = threadIdx.x & 31;
    __syncwarp();
    const int rin = fin ? 0 : ni % (2 * J);  // inside sources left for the next consume
    sreg_region<SOFT, MASSES, NC, false, SPL>(stage, rin, ni - rin, j, J, owner, fin, L, a, eps2v, negu0v);
    ni = rin;
    nc -= sreg_region<SOFT, MASSES, NC, true, SPL>(stage, cap - nc, nc, j, J, owner, fin, L, a, eps2v, negu0v);
    // sink k = 2 p + half of the lane keeps its three partials at accs[(3 k + d) * 32 + lane]
#pragma unroll
    for (int p = 0; p < SPL / 2; ++p) {
        SA::add(accs[(6 * p + 0) * 32 + lane], L.ax[p].x); SA::add(accs[(6 * p + 1) * 32 + lane], L.ay[p].x);
        SA::add(accs[(6 * p + 2) * 32 + lane], L.az[p].x); SA::add(accs[(6 * p + 3) * 32 + lane], L.ax[p].y);
        SA::add(accs[(6 * p + 4) * 32 + lane], L.ay[p].y); SA::add(accs[(6 * p + 5) * 32 + lane], L.az[p].y);
        L.ax[p] = L.ay[p] = L.az[p] = make_float2(0.f, 0.f);
    }
    __syncwarp();
}

template <int SOFT, bool MASSES, int ACC, int NC, int SPL>
__global__ void __launch_bounds__(128, SPL == 4 ? P2P_SREG_MINBLOCKS : 3)
pair_sreg_kernel(const __grid_constant__ PairArgs a, const int cap) {
    extern __shared__ float4 smem_f4[];
    using SA = SregAcc<ACC>;
    using AT = typename SA::T;
    const int lane = threadIdx.x & 31;
    unsigned char *wbase = reinterpret_cast<unsigned char *>(smem_f4) + (threadIdx.x >> 5) * sreg_warp_bytes(cap, SPL);
    float4 *stage = reinterpret_cast<float4 *>(wbase);
    AT *accs = reinterpret_cast<AT *>(wbase + (size_t)cap * 32);
    SregCtx *ctx = reinterpret_cast<SregCtx *>(wbase + (size_t)cap * 32 + sreg_acc_bytes(SPL));
    const float2 eps2v = make_float2(a.eps2, a.eps2), negu0v = make_float2(-a.u0, -a.u0);
    const unsigned lanes_below = (1u << lane) - 1u;
    unsigned long long evaluated = 0;  // pair interactions of staged sources with real sinks
    constexpr int SLICE = 8 * SPL;     // sinks of a slice: G <= 8 groups, J >= 4 phases
    const int W = a.leaf_warps > 1 ? a.leaf_warps : 1;  // warps sharing a row (work items per leaf)
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf * W) break;
        const int li = item_leaf(a, item / W, lane);
        int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (W > 1) {  // this item's contiguous share of the row's entries
            const int part = item % W;
            const int64_t len = re - rb;
            re = rb + len * (part + 1) / W;
            rb = rb + len * part / W;
        }
        if (rb >= re) continue;
        int ipart, npart;
        {
            const LeafMeta mt = a.leaf[li];
            ipart = mt.ipart;
            npart = mt.npart;
            __syncwarp();  // the previous item's readers are done
            if (lane == 0) {
                ctx->mcx = mt.cx; ctx->mcy = mt.cy; ctx->mcz = mt.cz;
                ctx->mhx = mt.hx; ctx->mhy = mt.hy; ctx->mhz = mt.hz;
            }
        }
        for (int s0 = 0; s0 < npart; s0 += SLICE) {
            const int ns = min(SLICE, npart - s0);
            const int G = (ns + SPL - 1) / SPL;
            const int J = 32 / G;
            const int g = lane % G, jl = lane / G;
            const bool owner = jl < J;
            const int j = owner ? jl : 0;  // lanes past G * J shadow phase 0; their sums are never read
            const int first = ipart + s0;
            SregLane<SPL> L;
            {
                L.sfirst = first + min(SPL * g, ns - 1);
                L.slast = first + ns - 1;
#pragma unroll
                for (int p = 0; p < SPL / 2; ++p) {
                    const float4 q0 = a.pos4[min(L.sfirst + 2 * p, L.slast)];
                    const float4 q1 = a.pos4[min(L.sfirst + 2 * p + 1, L.slast)];
                    L.px[p] = make_float2(-q0.x, -q1.x);
                    L.py[p] = make_float2(-q0.y, -q1.y);
                    L.pz[p] = make_float2(-q0.z, -q1.z);
                    L.ax[p] = L.ay[p] = L.az[p] = make_float2(0.f, 0.f);
                }
            }
            {   // bounding box of the slice's sinks (sink frame), for the source classes
                const float4 q = a.pos4[first + min(lane, ns - 1)];
                float lx = q.x, ly = q.y, lz = q.z, hx = q.x, hy = q.y, hz = q.z;
                for (int sk = lane + 32; sk < ns; sk += 32) {
                    const float4 r = a.pos4[first + sk];
                    lx = fminf(lx, r.x); ly = fminf(ly, r.y); lz = fminf(lz, r.z);
                    hx = fmaxf(hx, r.x); hy = fmaxf(hy, r.y); hz = fmaxf(hz, r.z);
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    lx = fminf(lx, __shfl_xor_sync(kFull, lx, off));
                    ly = fminf(ly, __shfl_xor_sync(kFull, ly, off));
                    lz = fminf(lz, __shfl_xor_sync(kFull, lz, off));
                    hx = fmaxf(hx, __shfl_xor_sync(kFull, hx, off));
                    hy = fmaxf(hy, __shfl_xor_sync(kFull, hy, off));
                    hz = fmaxf(hz, __shfl_xor_sync(kFull, hz, off));
                }
                if (lane == 0) {
                    const float cx = 0.5f * (lx + hx), cy = 0.5f * (ly + hy), cz = 0.5f * (lz + hz);
                    ctx->bcx = cx; ctx->bcy = cy; ctx->bcz = cz;
                    // half-extents rounded up past the FP32 rounding of their own computation
                    ctx->bhx = fmaxf(hx - cx, cx - lx) * (1.0f + 1.0e-6f);
                    ctx->bhy = fmaxf(hy - cy, cy - ly) * (1.0f + 1.0e-6f);
                    ctx->bhz = fmaxf(hz - cz, cz - lz) * (1.0f + 1.0e-6f);
                }
            }
#pragma unroll
            for (int k = 0; k < 3 * SPL; ++k) SA::zero(accs[k * 32 + lane]);
            int ni = 0, nc = 0;
            unsigned staged = 0;
            // The row's entries in batches of 32, each batch's sources in groups of
            // 32 x kSregRounds; one consume site serves the mid-row and final consumes.
            int64_t e0 = rb;
            int done = 0, total = 0, incl = 0;
            for (;;) {
                while (done >= total && e0 < re) {  // next batch of entries
                    const int ne = (int)min((int64_t)32, re - e0);
                    int snp = 0;
                    __syncwarp();  // readers of the previous batch are done
                    if (lane < ne) {
                        const LeafMeta ms = a.leaf[a.row_src[e0 + lane]];
                        LeafMeta mt;
                        mt.cx = ctx->mcx; mt.cy = ctx->mcy; mt.cz = ctx->mcz;
                        mt.hx = ctx->mhx; mt.hy = ctx->mhy; mt.hz = ctx->mhz;
                        float ox, oy, oz;
                        entry_offset(ms, mt, a.cscale, ox, oy, oz);
                        snp = entry_u_min(ms, mt, ox, oy, oz) > a.uout ? 0 : ms.npart;
                        ctx->sip[lane] = ms.ipart;
                        ctx->ein[lane] = entry_u_max(ms, mt, ox, oy, oz, a.eps2) < a.uin ? 1 : 0;
                        ctx->ox[lane] = ox; ctx->oy[lane] = oy; ctx->oz[lane] = oz;
                    }
                    ctx->snp[lane] = snp;
                    incl = snp;  // inclusive prefix sum of the entries' sizes
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1) {
                        const int up = __shfl_up_sync(kFull, incl, off);
                        if (lane >= off) incl += up;
                    }
                    total = __shfl_sync(kFull, incl, 31);
                    done = 0;
                    e0 += 32;
                    __syncwarp();
                }
                const bool end = done >= total;  // every source of the row is staged
                // consume at the row's end, and before a group that might not fit
                // (at most twice: the second consume empties the stage)
                for (bool fin = end; end ? (ni + nc > 0) : (ni + nc > cap - 32 * kSregRounds); fin = true)
                    sreg_consume<SOFT, MASSES, ACC, NC, SPL>(stage, accs, cap, ni, nc, fin, j, J, owner, L, a, eps2v,
                                                             negu0v);
                if (end) break;
                {
                    // every round's source located and its load issued first
                    float4 v[kSregRounds];
                    int vidx[kSregRounds], vin[kSregRounds];
                    float vx[kSregRounds], vy[kSregRounds], vz[kSregRounds];
#pragma unroll
                    for (int r = 0; r < kSregRounds; ++r) {
                        const int t = done + 32 * r + lane;
                        const int gsrc = min(t, total - 1);
                        int e = 0;  // this lane's entry: the first whose inclusive prefix exceeds gsrc
#pragma unroll
                        for (int st = 16; st > 0; st >>= 1) {
                            const int probe = __shfl_sync(kFull, incl, e + st - 1);
                            if (probe <= gsrc) e += st;
                        }
                        const int q = gsrc - (__shfl_sync(kFull, incl, e) - ctx->snp[e]);
                        vidx[r] = ctx->sip[e] + q;
                        vin[r] = ctx->ein[e];
                        vx[r] = ctx->ox[e];
                        vy[r] = ctx->oy[e];
                        vz[r] = ctx->oz[e];
                        v[r] = t < total ? a.pos4[vidx[r]] : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                    const float bcx = ctx->bcx, bcy = ctx->bcy, bcz = ctx->bcz;
                    const float bhx = ctx->bhx, bhy = ctx->bhy, bhz = ctx->bhz;
#pragma unroll
                    for (int r = 0; r < kSregRounds; ++r) {
                        const int t = done + 32 * r + lane;
                        int cls = 0;  // 0 dropped, 1 inside, 2 needs the cutoff test
                        const float4 w = make_float4(v[r].x + vx[r], v[r].y + vy[r], v[r].z + vz[r], v[r].w);
                        if (t < total) {
                            if (vin[r]) {
                                cls = 1;
                            } else {
                                const float dx = fabsf(w.x - bcx), dy = fabsf(w.y - bcy), dz = fabsf(w.z - bcz);
                                const float lx = fmaxf(dx - bhx, 0.f), ly = fmaxf(dy - bhy, 0.f),
                                            lz = fmaxf(dz - bhz, 0.f);
                                const float hx = dx + bhx, hy = dy + bhy, hz = dz + bhz;
                                const float umin = fmaf(lx, lx, fmaf(ly, ly, lz * lz));
                                const float umax = fmaf(hx, hx, fmaf(hy, hy, fmaf(hz, hz, a.eps2)));
                                cls = umin > a.uout ? 0 : (umax < a.uin ? 1 : 2);
                            }
                        }
                        const unsigned mi = __ballot_sync(kFull, cls == 1), mc = __ballot_sync(kFull, cls == 2);
                        if (cls) {
                            const int slot = cls == 1 ? ni + __popc(mi & lanes_below)
                                                      : cap - 1 - (nc + __popc(mc & lanes_below));
                            stage[2 * slot] = make_float4(w.x, w.x, w.y, w.y);
                            stage[2 * slot + 1] = make_float4(w.z, w.z, w.w, __int_as_float(vidx[r]));
                        }
                        ni += __popc(mi);
                        nc += __popc(mc);
                        staged += (unsigned)(__popc(mi) + __popc(mc));
                    }
                }
                done += 32 * kSregRounds;
            }
            __syncwarp();
            for (int sk = lane; sk < ns; sk += 32) {
                const int gg = sk / SPL, sl = sk % SPL;
                typename SA::Sum sx = 0, sy = 0, sz = 0;
                for (int jj = 0; jj < J; ++jj) {
                    const int l = gg + jj * G;
                    sx += SA::value(accs[(sl * 3 + 0) * 32 + l]);
                    sy += SA::value(accs[(sl * 3 + 1) * 32 + l]);
                    sz += SA::value(accs[(sl * 3 + 2) * 32 + l]);
                }
                const int idx = first + sk;
                double *o = a.acc;
                const size_t n = (size_t)a.npart;
                if (W > 1) {  // other warps add their shares of the row to the same sinks
                    atomicAdd(o + idx, (double)sx * a.out_scale);
                    atomicAdd(o + n + idx, (double)sy * a.out_scale);
                    atomicAdd(o + 2 * n + idx, (double)sz * a.out_scale);
                } else {
                    o[idx] += (double)sx * a.out_scale;
                    o[n + idx] += (double)sy * a.out_scale;
                    o[2 * n + idx] += (double)sz * a.out_scale;
                }
            }
            __syncwarp();  // accumulators and stage are rewritten by the next slice
            evaluated += (unsigned long long)staged * (unsigned long long)ns;
        }
    }
    if (a.evaluated && lane == 0 && evaluated) atomicAdd(a.evaluated, evaluated);
}

}  // namespace p2p
