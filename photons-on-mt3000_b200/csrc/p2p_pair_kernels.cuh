// Pair kernels of the P2P pass (templates): FP32 forms in three lane
// mappings and the FP64 drop-in form.
#pragma once

#include <type_traits>

#include "p2p_device_common.cuh"

namespace p2p {

// ------------------------------------------------------------ pair: FP32 ---


struct AccF64 {
    double x = 0.0, y = 0.0, z = 0.0;
    __device__ __forceinline__ void add(float ax, float ay, float az) {
        x += (double)ax;
        y += (double)ay;
        z += (double)az;
    }
    __device__ __forceinline__ void reduce_xor(int from) {
        for (int off = from; off < 32; off <<= 1) {
            x += __shfl_xor_sync(kFull, x, off);
            y += __shfl_xor_sync(kFull, y, off);
            z += __shfl_xor_sync(kFull, z, off);
        }
    }
    __device__ __forceinline__ double vx() const { return x; }
    __device__ __forceinline__ double vy() const { return y; }
    __device__ __forceinline__ double vz() const { return z; }
};

struct AccKahan {
    float x = 0.f, y = 0.f, z = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    __device__ __forceinline__ static void kadd(float &s, float &c, float v) {
        const float yv = v - c;
        const float t = s + yv;
        c = (t - s) - yv;
        s = t;
    }
    __device__ __forceinline__ void add(float ax, float ay, float az) {
        kadd(x, cx, ax);
        kadd(y, cy, ay);
        kadd(z, cz, az);
    }
    __device__ __forceinline__ void reduce_xor(int from) {
        x -= cx; y -= cy; z -= cz;
        cx = cy = cz = 0.f;
        for (int off = from; off < 32; off <<= 1) {
            x += __shfl_xor_sync(kFull, x, off);
            y += __shfl_xor_sync(kFull, y, off);
            z += __shfl_xor_sync(kFull, z, off);
        }
    }
    // compensated value: the running sum minus the carried rounding error
    __device__ __forceinline__ double vx() const { return (double)x - (double)cx; }
    __device__ __forceinline__ double vy() const { return (double)y - (double)cy; }
    __device__ __forceinline__ double vz() const { return (double)z - (double)cz; }
};

struct AccF32 {
    float x = 0.f, y = 0.f, z = 0.f;
    __device__ __forceinline__ void add(float ax, float ay, float az) {
        x += ax;
        y += ay;
        z += az;
    }
    __device__ __forceinline__ void reduce_xor(int from) {
        for (int off = from; off < 32; off <<= 1) {
            x += __shfl_xor_sync(kFull, x, off);
            y += __shfl_xor_sync(kFull, y, off);
            z += __shfl_xor_sync(kFull, z, off);
        }
    }
    __device__ __forceinline__ double vx() const { return x; }
    __device__ __forceinline__ double vy() const { return y; }
    __device__ __forceinline__ double vz() const { return z; }
};

template <int ACC> struct AccSel;
template <> struct AccSel<ACC_F64> { using T = AccF64; };
template <> struct AccSel<ACC_KAHAN> { using T = AccKahan; };
template <> struct AccSel<ACC_F32> { using T = AccF32; };

// One pair in scaled units (lengths times c = 1/(2 r_s)). With u = x^2 the
// squared (softened) separation, the truncated kernel
//     g(x) / r^3,   g(x) = erfc(x) + (2/sqrt(pi)) x exp(-x^2)
// is written as g(x) = 1 - x^3 H(x^2), so that in scaled units
//     f = rinv^3 - H(u),   H(u) = sum coef[k] (u - u0)^k,
// a polynomial directly in u: one MUFU rsqrt, no exp, no divide.
template <int SOFT, bool MASSES, int NC>
__device__ __forceinline__ void pair_split(const float4 s, const float px, const float py,
                                           const float pz, const PairArgs &a, float &ax, float &ay,
                                           float &az) {
    const float dx = s.x - px, dy = s.y - py, dz = s.z - pz;
    float u;
    if (SOFT == SOFT_PLUMMER) {
        u = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, a.eps2)));
    } else {
        u = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), a.eps2);
    }
    const float rinv = rsqrt_approx(u);
    const float t = u - a.u0;
    float h = a.coef[NC - 1];  // -H(u)
#pragma unroll
    for (int k = NC - 2; k >= 0; --k) h = fmaf(h, t, a.coef[k]);
    float f = fmaf(rinv * rinv, rinv, h);
    f = (u <= a.ucut) ? f : 0.0f;
    if (MASSES) f *= s.w;
    ax = fmaf(dx, f, ax);
    ay = fmaf(dy, f, ay);
    az = fmaf(dz, f, az);
}

// Staged sources are consumed in FP32 partial sums of at most kFlush
// sources per lane before they are added into the row accumulator.
constexpr int kFlush = 64;

template <int SOFT, bool MASSES, int NC, class Acc>
__device__ __forceinline__ void consume_split(const float4 *stage, int fill, int sub, int kk,
                                              float px, float py, float pz, const PairArgs &a,
                                              Acc &acc) {
    for (int base = sub; base < fill; base += kk * kFlush) {
        float ax = 0.f, ay = 0.f, az = 0.f;
        const int end = min(fill, base + kk * kFlush);
        int j = base;
        for (; j + 3 * kk < end; j += 4 * kk) {
            const float4 s0 = stage[j], s1 = stage[j + kk], s2 = stage[j + 2 * kk],
                         s3 = stage[j + 3 * kk];
            pair_split<SOFT, MASSES, NC>(s0, px, py, pz, a, ax, ay, az);
            pair_split<SOFT, MASSES, NC>(s1, px, py, pz, a, ax, ay, az);
            pair_split<SOFT, MASSES, NC>(s2, px, py, pz, a, ax, ay, az);
            pair_split<SOFT, MASSES, NC>(s3, px, py, pz, a, ax, ay, az);
        }
        for (; j < end; j += kk) pair_split<SOFT, MASSES, NC>(stage[j], px, py, pz, a, ax, ay, az);
        acc.add(ax, ay, az);
    }
}

// Lanes per sink particle group: 32 sink particles per warp pass, or for
// small slices several lanes share a particle and split its sources.
// Sink leaf of work item `item` (warp-uniform): the item itself in a pass over
// one box; in a packed launch, the item's place in the leaf range of the box
// whose segment holds it (segments start at ascending items, seg_item[0] = 0).
__device__ __forceinline__ int item_leaf(const PairArgs &a, const int item, const int lane) {
    if (a.nseg == 0) return item;
    const unsigned m = __ballot_sync(kFull, lane < a.nseg && a.seg_item[lane] <= item);
    const int k = 31 - __clz(m);
    return a.seg_leaf[k] + (item - a.seg_item[k]);
}

__device__ __forceinline__ int group_size(int ns) { return ns > 16 ? 32 : (ns > 8 ? 16 : 8); }

template <int SOFT, bool MASSES, int ACC, int NC>
__global__ void __launch_bounds__(256)
pair_split_kernel(const __grid_constant__ PairArgs a, const int stage_cap) {
    extern __shared__ float4 smem_f4[];
    using Acc = typename AccSel<ACC>::T;
    const int lane = threadIdx.x & 31;
    float4 *stage = smem_f4 + (threadIdx.x >> 5) * stage_cap;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf) break;
        const int li = item_leaf(a, item, lane);
        const int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (rb >= re) continue;
        const LeafMeta mt = a.leaf[li];
        for (int s0 = 0; s0 < mt.npart; s0 += 32) {
            const int ns = min(32, mt.npart - s0);
            const int gs = group_size(ns);
            const int kk = 32 / gs;
            const int i = lane & (gs - 1), sub = lane / gs;
            const bool act = i < ns;
            const float4 p = act ? a.pos4[mt.ipart + s0 + i] : make_float4(0.f, 0.f, 0.f, 0.f);
            Acc acc;
            int fill = 0;
            for (int64_t e0 = rb; e0 < re; e0 += 32) {
                const int ne = (int)min((int64_t)32, re - e0);
                int sip = 0, snp = 0;
                float ox = 0.f, oy = 0.f, oz = 0.f;
                if (lane < ne) {
                    const LeafMeta ms = a.leaf[a.row_src[e0 + lane]];
                    sip = ms.ipart;
                    snp = ms.npart;
                    ox = (float)((ms.cx - mt.cx) * a.cscale);
                    oy = (float)((ms.cy - mt.cy) * a.cscale);
                    oz = (float)((ms.cz - mt.cz) * a.cscale);
                }
                for (int j = 0; j < ne; ++j) {
                    const int jnp = __shfl_sync(kFull, snp, j);
                    const int jip = __shfl_sync(kFull, sip, j);
                    const float jx = __shfl_sync(kFull, ox, j);
                    const float jy = __shfl_sync(kFull, oy, j);
                    const float jz = __shfl_sync(kFull, oz, j);
                    int q0 = 0;
                    while (q0 < jnp) {
                        if (fill == stage_cap) {
                            __syncwarp();
                            consume_split<SOFT, MASSES, NC>(stage, fill, sub, kk, p.x, p.y, p.z, a, acc);
                            __syncwarp();
                            fill = 0;
                        }
                        const int take = min(jnp - q0, stage_cap - fill);
                        for (int q = lane; q < take; q += 32) {
                            const float4 v = a.pos4[jip + q0 + q];
                            stage[fill + q] = make_float4(v.x + jx, v.y + jy, v.z + jz, v.w);
                        }
                        fill += take;
                        q0 += take;
                    }
                }
            }
            __syncwarp();
            consume_split<SOFT, MASSES, NC>(stage, fill, sub, kk, p.x, p.y, p.z, a, acc);
            __syncwarp();
            acc.reduce_xor(gs);
            if (act && sub == 0) {
                const int idx = mt.ipart + s0 + i;
                a.acc[idx] += acc.vx() * a.out_scale;
                a.acc[(size_t)a.npart + idx] += acc.vy() * a.out_scale;
                a.acc[2 * (size_t)a.npart + idx] += acc.vz() * a.out_scale;
            }
        }
    }
}

// ------------------------------------------- pair: FP32, source lanes ---
//
// Second mapping of the same pass: lanes own staged SOURCES (32 per chunk, so
// every lane is busy whatever the sink leaf size) and loop over the sink
// particles of the row, read as shared-memory broadcasts. Each lane keeps an
// FP32 partial force per sink (registers); every kSrcFlushChunks chunks the
// 32 lanes' partials are folded with a transposing butterfly (31 shuffles per
// component) so that lane i holds sink i's sum, which it adds to its FP64
// (or Kahan / FP32) total.
constexpr int kSinkGroup = 4;        // sinks evaluated per predicated block
#ifndef P2P_FLUSH_CHUNKS
#define P2P_FLUSH_CHUNKS 64
#endif
constexpr int kSrcFlushChunks = P2P_FLUSH_CHUNKS;  // FP32 partial depth per lane, in chunks

template <int K, int N>
__device__ __forceinline__ void butterfly_step(float (&v)[N], const int lane) {
    const bool up = lane & K;
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const float send = up ? v[j] : v[j + K];
        const float keep = up ? v[j + K] : v[j];
        v[j] = keep + __shfl_xor_sync(kFull, send, K);
    }
}

// After the call lane L holds in v[0] the sum over all lanes of v[L % N]
// (N = 32 or 16).
template <int N>
__device__ __forceinline__ void transpose_reduce(float (&v)[N], const int lane) {
    static_assert(N == 32 || N == 16, "32 or 16 values per lane");
    if (N == 32) butterfly_step<16>(v, lane);
    butterfly_step<8>(v, lane);
    butterfly_step<4>(v, lane);
    butterfly_step<2>(v, lane);
    butterfly_step<1>(v, lane);
    if (N == 16) v[0] += __shfl_xor_sync(kFull, v[0], 16);
}

template <int SOFT, bool MASSES, int NC>
__device__ __forceinline__ void consume_src_lanes(const float4 *stage, int fill,
                                                  const float4 *sinks, int ns, int lane,
                                                  const PairArgs &a, float (&ax)[32],
                                                  float (&ay)[32], float (&az)[32]) {
    for (int c = 0; c < fill; c += 32) {
        const float4 src = (c + lane < fill) ? stage[c + lane]
                                             : make_float4(1.0e4f, 1.0e4f, 1.0e4f, 0.0f);
#pragma unroll
        for (int g = 0; g < 32; g += kSinkGroup) {
            if (g < ns) {
#pragma unroll
                for (int q = 0; q < kSinkGroup; ++q) {
                    const float4 p = sinks[g + q];
                    pair_split<SOFT, MASSES, NC>(src, p.x, p.y, p.z, a, ax[g + q], ay[g + q],
                                                 az[g + q]);
                }
            }
        }
    }
}

template <int SOFT, bool MASSES, int ACC, int NC>
__global__ void __launch_bounds__(128, 3)
pair_split_src_kernel(const __grid_constant__ PairArgs a, const int stage_cap) {
    extern __shared__ float4 smem_f4[];
    using Acc = typename AccSel<ACC>::T;
    const int lane = threadIdx.x & 31;
    float4 *sinks = smem_f4 + (threadIdx.x >> 5) * (stage_cap + 32);
    float4 *stage = sinks + 32;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf) break;
        const int li = item_leaf(a, item, lane);
        const int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (rb >= re) continue;
        const LeafMeta mt = a.leaf[li];
        for (int s0 = 0; s0 < mt.npart; s0 += 32) {
            const int ns = min(32, mt.npart - s0);
            // sinks of this slice in their own leaf frame; slots past ns repeat
            // the first sink so padded evaluations stay finite (never stored)
            sinks[lane] = a.pos4[mt.ipart + s0 + (lane < ns ? lane : 0)];
            float ax[32], ay[32], az[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) ax[i] = ay[i] = az[i] = 0.f;
            Acc acc;
            int fill = 0, chunks = 0;
            auto flush = [&]() {
                transpose_reduce(ax, lane);
                transpose_reduce(ay, lane);
                transpose_reduce(az, lane);
                acc.add(ax[0], ay[0], az[0]);
#pragma unroll
                for (int i = 0; i < 32; ++i) ax[i] = ay[i] = az[i] = 0.f;
                chunks = 0;
            };
            auto consume = [&]() {
                __syncwarp();
                consume_src_lanes<SOFT, MASSES, NC>(stage, fill, sinks, ns, lane, a, ax, ay, az);
                __syncwarp();
                chunks += (fill + 31) >> 5;
                fill = 0;
                if (chunks >= kSrcFlushChunks) flush();
            };
            for (int64_t e0 = rb; e0 < re; e0 += 32) {
                const int ne = (int)min((int64_t)32, re - e0);
                int sip = 0, snp = 0;
                float ox = 0.f, oy = 0.f, oz = 0.f;
                if (lane < ne) {
                    const LeafMeta ms = a.leaf[a.row_src[e0 + lane]];
                    sip = ms.ipart;
                    snp = ms.npart;
                    ox = (float)((ms.cx - mt.cx) * a.cscale);
                    oy = (float)((ms.cy - mt.cy) * a.cscale);
                    oz = (float)((ms.cz - mt.cz) * a.cscale);
                }
                for (int j = 0; j < ne; ++j) {
                    const int jnp = __shfl_sync(kFull, snp, j);
                    const int jip = __shfl_sync(kFull, sip, j);
                    const float jx = __shfl_sync(kFull, ox, j);
                    const float jy = __shfl_sync(kFull, oy, j);
                    const float jz = __shfl_sync(kFull, oz, j);
                    int q0 = 0;
                    while (q0 < jnp) {
                        if (fill == stage_cap) consume();
                        const int take = min(jnp - q0, stage_cap - fill);
                        for (int q = lane; q < take; q += 32) {
                            const float4 v = a.pos4[jip + q0 + q];
                            stage[fill + q] = make_float4(v.x + jx, v.y + jy, v.z + jz, v.w);
                        }
                        fill += take;
                        q0 += take;
                    }
                }
            }
            if (fill) consume();
            if (chunks) flush();
            __syncwarp();  // sinks[] is rewritten by the next slice
            if (lane < ns) {
                const int idx = mt.ipart + s0 + lane;
                a.acc[idx] += acc.vx() * a.out_scale;
                a.acc[(size_t)a.npart + idx] += acc.vy() * a.out_scale;
                a.acc[2 * (size_t)a.npart + idx] += acc.vz() * a.out_scale;
            }
        }
    }
}

// ------------------------------------ pair: FP32, source lanes, f32x2 ---
//
// The source-lane mapping with two sinks per instruction: sm_100's packed
// FP32 instructions (FFMA2 / FADD2 / FMUL2) evaluate the pair function for
// sinks i and i+1 against the lane's source at once. Same arithmetic as
// pair_split element by element; half the FP instructions, twice the
// independent work per instruction stream.

// Sink pairs in shared memory, coordinates negated so dx = s + (-p).
struct SinkPair {
    float4 xy;  // (-x_i, -x_{i+1}, -y_i, -y_{i+1})
    float2 z;   // (-z_i, -z_{i+1})
    float2 pad;
};

// Tuning knobs of the packed kernel (compile time).
#ifndef P2P_X2_GROUP
#define P2P_X2_GROUP 4  // packed sink pairs per predicated block in the first half of the tile (8 sinks)
#endif
#ifndef P2P_X2_MINBLOCKS
#define P2P_X2_MINBLOCKS 3  // resident 128-thread blocks per SM the register budget targets
#endif
#ifndef P2P_X2_S16_MINBLOCKS
#define P2P_X2_S16_MINBLOCKS 4  // resident blocks per SM the 16-sink tile's register budget targets
#endif
#ifndef P2P_X2_SINKPAIRS
#define P2P_X2_SINKPAIRS 16  // sink pairs per slice (a slice holds 2x that many sinks)
#endif
#ifndef P2P_X2_TAILGROUP
#define P2P_X2_TAILGROUP 2  // packed sink pairs per predicated block in the second half of the tile
#endif
constexpr int kPairGroup = P2P_X2_GROUP;
constexpr int kTailGroup = P2P_X2_TAILGROUP;

// H(t) for two sinks at once: Horner's rule, one packed FMA per coefficient.
// (Measured alternatives: two scalar Horner chains, Estrin's scheme,
// coefficient pairs held in registers or read as f32x2 parameters.)
template <int NC>
__device__ __forceinline__ float2 poly_x2(const float2 t, const PairArgs &a) {
    float2 h = a.coef2[NC - 1];
#pragma unroll
    for (int k = NC - 2; k >= 0; --k) h = __ffma2_rn(h, t, a.coef2[k]);
    return h;
}

// CHECK = false: every pair is known to be inside the cutoff (no select).
// CHECK = true: pairs beyond the band are dropped, pairs inside the band are
// flagged in amb for an FP64 decision.
// Sink pair given as packed negated coordinates (nx, ny, nz).
template <int SOFT, bool MASSES, int NC, bool CHECK>
__device__ __forceinline__ void pair_split_x2n(const float2 sx, const float2 sy, const float2 sz, const float sw,
                                               const float2 nx, const float2 ny, const float2 nz, const PairArgs &a,
                                               const float2 eps2v, const float2 negu0v, float2 &ax, float2 &ay,
                                               float2 &az, bool &amb) {
    const float2 dx = __fadd2_rn(sx, nx);
    const float2 dy = __fadd2_rn(sy, ny);
    const float2 dz = __fadd2_rn(sz, nz);
    float2 u;
    if (SOFT == SOFT_PLUMMER) {
        u = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2v)));
    } else {
        u = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        u.x = fmaxf(u.x, a.eps2);
        u.y = fmaxf(u.y, a.eps2);
    }
    const float2 r = make_float2(rsqrt_approx(u.x), rsqrt_approx(u.y));
    const float2 t = __fadd2_rn(u, negu0v);
    const float2 h = poly_x2<NC>(t, a);  // -H(u)
    float2 f = __ffma2_rn(__fmul2_rn(r, r), r, h);
    if (CHECK) {
        const bool in_x = u.x <= a.ucut_lo, in_y = u.y <= a.ucut_lo;
        amb |= (!in_x && u.x <= a.ucut_hi) || (!in_y && u.y <= a.ucut_hi);
        f.x = in_x ? f.x : 0.0f;
        f.y = in_y ? f.y : 0.0f;
    }
    if (MASSES) f = __fmul2_rn(f, make_float2(sw, sw));
    ax = __ffma2_rn(dx, f, ax);
    ay = __ffma2_rn(dy, f, ay);
    az = __ffma2_rn(dz, f, az);
}

template <int SOFT, bool MASSES, int NC, bool CHECK>
__device__ __forceinline__ void pair_split_x2(const float2 sx, const float2 sy, const float2 sz,
                                              const float sw, const SinkPair &p,
                                              const PairArgs &a, const float2 eps2v,
                                              const float2 negu0v, float2 &ax, float2 &ay,
                                              float2 &az, bool &amb) {
    pair_split_x2n<SOFT, MASSES, NC, CHECK>(sx, sy, sz, sw, make_float2(p.xy.x, p.xy.y), make_float2(p.xy.z, p.xy.w),
                                            p.z, a, eps2v, negu0v, ax, ay, az, amb);
}

// One pair whose FP32 u fell in the cutoff band: decide inclusion from the
// FP64 positions (as the FP64 form does) and, if it is inside, return its
// FP32 contribution through *contrib.
template <int SOFT, bool MASSES, int NC>
__device__ __forceinline__ bool band_pair(const float4 src, const float psx, const float psy,
                                       const float psz, int isrc, int isink, const PairArgs &a,
                                       float3 *contrib) {
    const float dx = src.x + psx, dy = src.y + psy, dz = src.z + psz;  // sinks are negated
    float u;
    if (SOFT == SOFT_PLUMMER) u = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, a.eps2)));
    else u = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), a.eps2);
    if (!(u > a.ucut_lo && u <= a.ucut_hi)) return false;
    const size_t n = (size_t)a.npart;
    const double ex = a.pos[isrc] - a.pos[isink];
    const double ey = a.pos[n + isrc] - a.pos[n + isink];
    const double ez = a.pos[2 * n + isrc] - a.pos[2 * n + isink];
    double r2 = ex * ex + ey * ey + ez * ez;
    r2 = (SOFT == SOFT_PLUMMER) ? r2 + a.eps2_box : fmax(r2, a.eps2_box);
    if (!(r2 <= a.rcut2)) return false;
    const float rinv = rsqrt_approx(u);
    const float t = u - a.u0;
    float h = a.coef[NC - 1];
#pragma unroll
    for (int k = NC - 2; k >= 0; --k) h = fmaf(h, t, a.coef[k]);
    float f = fmaf(rinv * rinv, rinv, h);
    if (MASSES) f *= src.w;
    *contrib = make_float3(dx * f, dy * f, dz * f);
    return true;
}


// Stages the sources of row entries [rb, re) of sink leaf mt: each source
// leaf's FP32 coordinates shifted into the sink's frame by the FP32-rounded
// FP64 offset of the two frames, with its particle index and, in the sign
// bit, whether its entry can reach the cutoff band (box bound on u >= uin).
// Sources of up to 32 entries are numbered consecutively (a warp prefix sum
// of their sizes) and every lane takes every 32nd of them, finding its entry
// by a binary search over the prefix sums, so a whole stage's global loads
// are in flight together. store(slot, source, index) writes one staged
// source; consume() empties the stage (fill = 0) when it is full.
template <class Store, class Consume>
__device__ __forceinline__ void stage_row_flat(const PairArgs &a, const LeafMeta &mt, const int64_t rb,
                                               const int64_t re, const int lane, const int stage_cap,
                                               int &fill, Store &&store, Consume &&consume) {
    for (int64_t e0 = rb; e0 < re; e0 += 32) {
        const int ne = (int)min((int64_t)32, re - e0);
        int sip = 0, snp = 0, chk = 0;
        float ox = 0.f, oy = 0.f, oz = 0.f;
        if (lane < ne) {
            const LeafMeta ms = a.leaf[a.row_src[e0 + lane]];
            sip = ms.ipart;
            entry_offset(ms, mt, a.cscale, ox, oy, oz);
            // entries wholly beyond the cutoff are not staged (their pairs would
            // all be dropped); the others take the cutoff test unless wholly inside
            snp = entry_u_min(ms, mt, ox, oy, oz) > a.uout ? 0 : ms.npart;
            chk = entry_u_max(ms, mt, ox, oy, oz, a.eps2) < a.uin ? 0 : (int)0x80000000;
        }
        int incl = snp;  // inclusive prefix sum of the entries' sizes
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        int done = 0;
        while (done < total) {
            if (fill == stage_cap) consume();
            const int take = min(total - done, stage_cap - fill);
            for (int t0 = 0; t0 < take; t0 += 32) {
                const int t = t0 + lane;
                const int g = done + min(t, take - 1);  // this lane's source (idle lanes repeat the last)
                // its entry: the first one whose inclusive prefix exceeds g
                int e = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int probe = __shfl_sync(kFull, incl, e + step - 1);
                    if (probe <= g) e += step;
                }
                const int q = g - (__shfl_sync(kFull, incl, e) - __shfl_sync(kFull, snp, e));
                const int jip = __shfl_sync(kFull, sip, e);
                const int jchk = __shfl_sync(kFull, chk, e);
                const float jx = __shfl_sync(kFull, ox, e);
                const float jy = __shfl_sync(kFull, oy, e);
                const float jz = __shfl_sync(kFull, oz, e);
                if (t < take) {
                    const float4 v = a.pos4[jip + q];
                    store(fill + t, make_float4(v.x + jx, v.y + jy, v.z + jz, v.w), (jip + q) | jchk);
                }
            }
            fill += take;
            done += take;
        }
    }
}

// NP sink pairs per slice: 16 (32-sink tile, 3 blocks of 4 warps per SM) or
// 8 (16-sink tile, half the partial registers, 4 blocks per SM).
template <int SOFT, bool MASSES, int ACC, int NC, int NP = P2P_X2_SINKPAIRS>
__global__ void __launch_bounds__(128, NP == 8 ? P2P_X2_S16_MINBLOCKS : P2P_X2_MINBLOCKS)
pair_split_src2_kernel(const __grid_constant__ PairArgs a, const int stage_cap) {
    extern __shared__ float4 smem_f4[];
    using Acc = typename AccSel<ACC>::T;
    const int lane = threadIdx.x & 31;
    // per warp: up to 16 sink pairs (512 B), 32 band corrections (512 B), the
    // staged sources and their particle indices
    constexpr int NS = 2 * NP;
    static_assert(NP == 8 || NP == 16, "8 or 16 sink pairs per slice");
    float4 *region = smem_f4 + (threadIdx.x >> 5) * (stage_cap + 64 + stage_cap / 4);
    SinkPair *sinks = reinterpret_cast<SinkPair *>(region);
    float4 *corr = region + 32;
    float4 *stage = region + 64;
    int *sidx = reinterpret_cast<int *>(stage + stage_cap);
    const float2 eps2v = make_float2(a.eps2, a.eps2), negu0v = make_float2(-a.u0, -a.u0);
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf) break;
        const int li = item_leaf(a, item, lane);
        const int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (rb >= re) continue;
        const LeafMeta mt = a.leaf[li];
        for (int s0 = 0; s0 < mt.npart; s0 += NS) {
            const int ns = min(NS, mt.npart - s0);
            {
                // slots past ns repeat the first sink so padded lanes stay finite
                const float4 q = a.pos4[mt.ipart + s0 + (lane < ns ? lane : 0)];
                float *xy = reinterpret_cast<float *>(&sinks[lane >> 1].xy);
                float *z = reinterpret_cast<float *>(&sinks[lane >> 1].z);
                xy[lane & 1] = -q.x;
                xy[2 + (lane & 1)] = -q.y;
                z[lane & 1] = -q.z;
                corr[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            // packed partials: element .x of pair k is sink 2k, .y sink 2k+1
            float2 ax[NP], ay[NP], az[NP];
#pragma unroll
            for (int i = 0; i < NP; ++i) ax[i] = ay[i] = az[i] = make_float2(0.f, 0.f);
            Acc acc;
            int fill = 0, chunks = 0;
            auto flush = [&]() {
                float vx[NS], vy[NS], vz[NS];
#pragma unroll
                for (int i = 0; i < NP; ++i) {
                    vx[2 * i] = ax[i].x; vx[2 * i + 1] = ax[i].y;
                    vy[2 * i] = ay[i].x; vy[2 * i + 1] = ay[i].y;
                    vz[2 * i] = az[i].x; vz[2 * i + 1] = az[i].y;
                }
                transpose_reduce(vx, lane);
                transpose_reduce(vy, lane);
                transpose_reduce(vz, lane);
                acc.add(vx[0], vy[0], vz[0]);
#pragma unroll
                for (int i = 0; i < NP; ++i) ax[i] = ay[i] = az[i] = make_float2(0.f, 0.f);
                chunks = 0;
            };
            auto consume = [&]() {
                __syncwarp();
                unsigned ambmask = 0;  // chunks of this batch with a pair in the cutoff band
                for (int c = 0, ci = 0; c < fill; c += 32, ++ci) {
                    const int slot = c + lane;
                    const float4 src = slot < fill ? stage[slot]
                                                   : make_float4(1.0e4f, 1.0e4f, 1.0e4f, 0.0f);
                    const float2 sx = make_float2(src.x, src.x), sy = make_float2(src.y, src.y),
                                 sz = make_float2(src.z, src.z);
                    // full chunks whose sources all come from entries inside the
                    // cutoff skip the select and the band test
                    const bool check = __any_sync(kFull, slot >= fill || sidx[slot] < 0);
                    bool amb = false;
                    // sink pairs in blocks of kPairGroup over the first half
                    // of the tile and of kTailGroup over the second, where the
                    // last, partly filled block usually falls (less padding)
#define P2P_X2_SWEEP(CHK)                                                                                     \
    _Pragma("unroll") for (int g = 0; g < NP / 2; g += kPairGroup) {                                         \
        if (2 * g < ns) {                                                                                    \
            _Pragma("unroll") for (int q = 0; q < kPairGroup; ++q)                                           \
                pair_split_x2<SOFT, MASSES, NC, CHK>(sx, sy, sz, src.w, sinks[g + q], a, eps2v, negu0v,       \
                                                     ax[g + q], ay[g + q], az[g + q], amb);                  \
        }                                                                                                    \
    }                                                                                                        \
    _Pragma("unroll") for (int g = NP / 2; g < NP; g += kTailGroup) {                                        \
        if (2 * g < ns) {                                                                                    \
            _Pragma("unroll") for (int q = 0; q < kTailGroup; ++q)                                           \
                pair_split_x2<SOFT, MASSES, NC, CHK>(sx, sy, sz, src.w, sinks[g + q], a, eps2v, negu0v,       \
                                                     ax[g + q], ay[g + q], az[g + q], amb);                  \
        }                                                                                                    \
    }
                    if (check) {
                        P2P_X2_SWEEP(true)
                    } else {
                        P2P_X2_SWEEP(false)
                    }
#undef P2P_X2_SWEEP
                    ambmask |= amb ? (1u << ci) : 0u;
                }
                // rare: pairs within the cutoff band, decided in FP64
                if (__any_sync(kFull, ambmask != 0u)) {
                    while (ambmask) {
                        const int ci = __ffs(ambmask) - 1;
                        ambmask &= ambmask - 1;
                        const int slot = ci * 32 + lane;
                        const float4 src = stage[slot];
                        const int isrc = sidx[slot] & 0x7fffffff;
                        for (int k = 0; k < ns; ++k) {
                            const SinkPair &sp = sinks[k >> 1];
                            const float psx = (k & 1) ? sp.xy.y : sp.xy.x;
                            const float psy = (k & 1) ? sp.xy.w : sp.xy.z;
                            const float psz = (k & 1) ? sp.z.y : sp.z.x;
                            float3 cb;
                            if (band_pair<SOFT, MASSES, NC>(src, psx, psy, psz, isrc, mt.ipart + s0 + k, a,
                                                            &cb)) {
                                atomicAdd(&corr[k].x, cb.x);
                                atomicAdd(&corr[k].y, cb.y);
                                atomicAdd(&corr[k].z, cb.z);
                            }
                        }
                    }
                }
                __syncwarp();
                chunks += (fill + 31) >> 5;
                fill = 0;
                if (chunks >= kSrcFlushChunks) flush();
            };
            stage_row_flat(a, mt, rb, re, lane, stage_cap, fill,
                           [&](int slot, const float4 v, int idx) {
                               stage[slot] = v;
                               sidx[slot] = idx;
                           },
                           consume);
            if (fill) consume();
            if (chunks) flush();
            __syncwarp();  // sinks[] and corr[] are rewritten by the next slice
            if (lane < ns) {
                const float4 cr = corr[lane];
                acc.add(cr.x, cr.y, cr.z);
                const int idx = mt.ipart + s0 + lane;
                a.acc[idx] += acc.vx() * a.out_scale;
                a.acc[(size_t)a.npart + idx] += acc.vy() * a.out_scale;
                a.acc[2 * (size_t)a.npart + idx] += acc.vz() * a.out_scale;
            }
        }
    }
}

// ------------------------------------------- pair: FP32, packed sink lanes ---

// Packed sink-lane mapping (P2P_VARIANT_SINK_LANES_X2). A slice of <= 32
// sinks is held as npairs = ceil(ns / 2) sink pairs; lane = (pair p, phase j)
// with P = npairs lanes per phase and J = floor(32 / P) phases: lane (p, j)
// keeps sink pair p in registers (one f32x2 per coordinate) and takes the
// staged sources j, j + J, j + 2J, ... (sources are staged pre-duplicated,
// (x, x, y, y) (z, z, w, w), so they load as packed operands). Per lane the
// FP32 partials are one f32x2 per component, flushed into the two sinks'
// accumulators every kSinkFlushIters sources; at row end the J phases of a
// pair are summed with shuffles. A pair whose FP32 u falls in the cutoff band
// is re-decided at once from FP64 positions (band_pair) by its own lane.
constexpr int kSinkFlushIters = 128;

template <int SOFT, bool MASSES, int ACC, int NC>
__global__ void __launch_bounds__(128, 5)
pair_sink2_kernel(const __grid_constant__ PairArgs a, const int stage_cap) {
    extern __shared__ float4 smem_f4[];
    using Acc = typename AccSel<ACC>::T;
    const int lane = threadIdx.x & 31;
    // per warp: staged sources (two float4 each) and their particle indices,
    // with room for up to 32 padding slots past stage_cap
    const int cap = stage_cap + 32;
    float4 *stage = smem_f4 + (threadIdx.x >> 5) * (2 * cap + cap / 4);
    int *sidx = reinterpret_cast<int *>(stage + 2 * cap);
    const float2 eps2v = make_float2(a.eps2, a.eps2), negu0v = make_float2(-a.u0, -a.u0);
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf) break;
        const int li = item_leaf(a, item, lane);
        const int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (rb >= re) continue;
        const LeafMeta mt = a.leaf[li];
        for (int s0 = 0; s0 < mt.npart; s0 += 32) {
            const int ns = min(32, mt.npart - s0);
            const int npairs = (ns + 1) >> 1;
            const int P = npairs, J = 32 / npairs;
            const int p = lane % P, j = lane / P;
            const bool owner = j < J;  // lanes past P * J take no sources
            // this lane's sink pair (a missing second sink repeats the first)
            const int sa = 2 * p, sb = min(2 * p + 1, ns - 1);
            const float4 qa = a.pos4[mt.ipart + s0 + sa], qb = a.pos4[mt.ipart + s0 + sb];
            SinkPair sp;
            sp.xy = make_float4(-qa.x, -qb.x, -qa.y, -qb.y);
            sp.z = make_float2(-qa.z, -qb.z);
            float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
            Acc acc_a, acc_b;
            int iters = 0;
            auto consume = [&](int fill) {
                // pad to whole iterations with far sources that take the
                // cutoff test (they contribute nothing)
                const int nit = (fill + J - 1) / J;
                for (int q = fill + lane; q < nit * J; q += 32) {
                    stage[2 * q] = make_float4(1.0e4f, 1.0e4f, 1.0e4f, 1.0e4f);
                    stage[2 * q + 1] = make_float4(1.0e4f, 1.0e4f, 0.f, 0.f);
                    sidx[q] = (int)0x80000000;
                }
                __syncwarp();
                // lanes past P * J stay on slot 0; their results are never used
                const float4 *pa = stage + 2 * (owner ? j : 0);
                const int *ps = sidx + (owner ? j : 0);
                const int da = owner ? 2 * J : 0, ds = owner ? J : 0;
                for (int ib = 0; ib < nit; ib += 32) {
                    const int nb = min(32, nit - ib);
                    unsigned ambbits = 0;  // iterations of this block with a pair in the cutoff band
#pragma unroll 2
                    for (int k = 0; k < nb; ++k) {
                        const float4 A = pa[0];
                        const float4 B = pa[1];
                        const int sid = *ps;
                        pa += da;
                        ps += ds;
                        const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w),
                                     sz = make_float2(B.x, B.y);
                        bool amb = false;
                        if (__any_sync(kFull, owner && sid < 0))
                            pair_split_x2<SOFT, MASSES, NC, true>(sx, sy, sz, B.z, sp, a, eps2v, negu0v, ax, ay,
                                                                  az, amb);
                        else
                            pair_split_x2<SOFT, MASSES, NC, false>(sx, sy, sz, B.z, sp, a, eps2v, negu0v, ax, ay,
                                                                   az, amb);
                        ambbits |= amb ? (1u << k) : 0u;
                    }
                    // rare: pairs inside the cutoff band, decided in FP64 by the owning lane
                    if (owner) {
                        while (ambbits) {
                            const int k = __ffs(ambbits) - 1;
                            ambbits &= ambbits - 1;
                            const int slot = (ib + k) * J + j;
                            const float4 A = stage[2 * slot], B = stage[2 * slot + 1];
                            const float4 src = make_float4(A.x, A.z, B.x, B.z);
                            const int isrc = sidx[slot] & 0x7fffffff;
                            float3 cb;
                            if (band_pair<SOFT, MASSES, NC>(src, sp.xy.x, sp.xy.z, sp.z.x, isrc, mt.ipart + s0 + sa,
                                                            a, &cb)) {
                                ax.x += cb.x;
                                ay.x += cb.y;
                                az.x += cb.z;
                            }
                            if (sb != sa && band_pair<SOFT, MASSES, NC>(src, sp.xy.y, sp.xy.w, sp.z.y, isrc,
                                                                        mt.ipart + s0 + sb, a, &cb)) {
                                ax.y += cb.x;
                                ay.y += cb.y;
                                az.y += cb.z;
                            }
                        }
                    }
                    iters += nb;
                    if (iters >= kSinkFlushIters) {
                        acc_a.add(ax.x, ay.x, az.x);
                        acc_b.add(ax.y, ay.y, az.y);
                        ax = ay = az = make_float2(0.f, 0.f);
                        iters = 0;
                    }
                }
                __syncwarp();
            };
            int fill = 0;
            stage_row_flat(a, mt, rb, re, lane, stage_cap, fill,
                           [&](int slot, const float4 v, int idx) {
                               stage[2 * slot] = make_float4(v.x, v.x, v.y, v.y);
                               stage[2 * slot + 1] = make_float4(v.z, v.z, v.w, v.w);
                               sidx[slot] = idx;
                           },
                           [&]() {
                               consume(fill);
                               fill = 0;
                           });
            if (fill) consume(fill);
            acc_a.add(ax.x, ay.x, az.x);
            acc_b.add(ax.y, ay.y, az.y);
            // sum the J phases of each sink pair into phase 0
            double t[6] = {acc_a.vx(), acc_a.vy(), acc_a.vz(), acc_b.vx(), acc_b.vy(), acc_b.vz()};
            for (int ph = 1; ph < J; ++ph) {
                const int from = (lane + ph * P) & 31;
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const double v = __shfl_sync(kFull, t[k], from);
                    if (j == 0) t[k] += v;
                }
            }
            if (j == 0 && p < npairs) {
                const size_t n = (size_t)a.npart;
                const int ia = mt.ipart + s0 + sa;
                a.acc[ia] += t[0] * a.out_scale;
                a.acc[n + ia] += t[1] * a.out_scale;
                a.acc[2 * n + ia] += t[2] * a.out_scale;
                if (2 * p + 1 < ns) {
                    const int ib = mt.ipart + s0 + 2 * p + 1;
                    a.acc[ib] += t[3] * a.out_scale;
                    a.acc[n + ib] += t[4] * a.out_scale;
                    a.acc[2 * n + ib] += t[5] * a.out_scale;
                }
            }
            __syncwarp();  // the stage is rewritten by the next slice
        }
    }
}

// ------------------------------------------------------------ pair: FP64 ---

// P2P_core_lite (src/gpu_kernel.impl.h:160-257) and P2P_core_1 (:260-362),
// non-SPI branches, in FP64 with CUDA's erfc / exp / rsqrt.
template <int SOFT, bool MASSES>
__device__ __forceinline__ void pair_plain(const double4 s, const double px, const double py,
                                           const double pz, const PairArgs &a, double &ax,
                                           double &ay, double &az) {
    const double dx = s.x - px, dy = s.y - py, dz = s.z - pz;
    double dr, drs;
    if (SOFT == SOFT_CLAMP) {
        const double dr2 = dx * dx + dy * dy + dz * dz;
        dr = a.soft;
        if (dr2 > a.soft * a.soft) {
            const double rdr = rsqrt(dr2);
            dr = rdr * dr2;
        }
        drs = dr * a.hrrs;
    } else {
        dr = sqrt(dx * dx + dy * dy + dz * dz + a.soft * a.soft);
        drs = 0.5 * dr * a.rrs;
    }
    if (a.xcut > 0.0 && drs > a.xcut) return;
    double ir3 = 1.0 / (dr * dr * dr);
    ir3 *= (erfc(drs) + a.coeff * drs * exp(-drs * drs));
    if (MASSES) ir3 *= s.w;
    ax += dx * ir3;
    ay += dy * ir3;
    az += dz * ir3;
}

template <int SOFT, bool MASSES>
__global__ void __launch_bounds__(256)
pair_plain_kernel(const __grid_constant__ PairArgs a, const int stage_cap) {
    extern __shared__ double4 smem_d4[];
    const int lane = threadIdx.x & 31;
    double4 *stage = smem_d4 + (threadIdx.x >> 5) * stage_cap;
    const double *X = a.pos, *Y = a.pos + a.npart, *Z = a.pos + 2 * (size_t)a.npart;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.queue, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item >= a.nleaf) break;
        const int li = item_leaf(a, item, lane);
        const int64_t rb = a.row_off[li], re = a.row_off[li + 1];
        if (rb >= re) continue;
        const LeafMeta mt = a.leaf[li];
        for (int s0 = 0; s0 < mt.npart; s0 += 32) {
            const int ns = min(32, mt.npart - s0);
            const int gs = group_size(ns);
            const int kk = 32 / gs;
            const int i = lane & (gs - 1), sub = lane / gs;
            const bool act = i < ns;
            const int pi = mt.ipart + s0 + (act ? i : 0);
            const double px = X[pi], py = Y[pi], pz = Z[pi];
            double ax = 0.0, ay = 0.0, az = 0.0;
            int fill = 0;
            for (int64_t e0 = rb; e0 < re; e0 += 32) {
                const int ne = (int)min((int64_t)32, re - e0);
                int sip = 0, snp = 0;
                if (lane < ne) {
                    const LeafMeta ms = a.leaf[a.row_src[e0 + lane]];
                    sip = ms.ipart;
                    snp = ms.npart;
                }
                for (int j = 0; j < ne; ++j) {
                    const int jnp = __shfl_sync(kFull, snp, j);
                    const int jip = __shfl_sync(kFull, sip, j);
                    int q0 = 0;
                    while (q0 < jnp) {
                        if (fill == stage_cap) {
                            __syncwarp();
                            for (int jj = sub; jj < fill; jj += kk)
                                pair_plain<SOFT, MASSES>(stage[jj], px, py, pz, a, ax, ay, az);
                            __syncwarp();
                            fill = 0;
                        }
                        const int take = min(jnp - q0, stage_cap - fill);
                        for (int q = lane; q < take; q += 32) {
                            const int k = jip + q0 + q;
                            stage[fill + q] = make_double4(X[k], Y[k], Z[k], a.mass ? a.mass[k] : 1.0);
                        }
                        fill += take;
                        q0 += take;
                    }
                }
            }
            __syncwarp();
            for (int jj = sub; jj < fill; jj += kk)
                pair_plain<SOFT, MASSES>(stage[jj], px, py, pz, a, ax, ay, az);
            __syncwarp();
            for (int off = gs; off < 32; off <<= 1) {
                ax += __shfl_xor_sync(kFull, ax, off);
                ay += __shfl_xor_sync(kFull, ay, off);
                az += __shfl_xor_sync(kFull, az, off);
            }
            if (act && sub == 0) {
                const int idx = mt.ipart + s0 + i;
                const double m = MASSES ? 1.0 : a.mass_eq;
                a.acc[idx] += ax * m;
                a.acc[(size_t)a.npart + idx] += ay * m;
                a.acc[2 * (size_t)a.npart + idx] += az * m;
            }
        }
    }
}

}  // namespace p2p
