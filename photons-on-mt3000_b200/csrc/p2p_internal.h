// Internal definitions shared by the host and device code of libphotons_p2p.
#pragma once

#include <cstdint>

#include <vector_types.h>

namespace p2p {

// Per-leaf record the pair kernels read for every source entry: the FP64
// frame centre the leaf's FP32 coordinates are relative to, and its particle
// range. 32 bytes, one 32 B sector per lookup.
struct __align__(16) LeafMeta {
    double cx, cy, cz;
    int ipart, npart;
    float hx, hy, hz;  // half-extents of the particles' bounding box, scaled by c (FP32 forms)
    float pad;
};

// Status bits the device sets instead of faulting on bad input.
enum : int {
    ST_LEAF_RANGE = 1,  // a leaf's particle range lies outside [0, npart)
    ST_TASK_RANGE = 2,  // a task entry names a leaf outside [0, nleaf)
};

constexpr int kMaxCoef = 21;  // polynomial degree <= 20
constexpr int kMaxSeg = 32;   // boxes per packed launch (one warp ballot maps an item)

// Relative half-width of the cutoff band around x_cut^2 inside which FP32
// rounding of u cannot decide a pair (coordinate rounding bounds the FP32
// error of u at about 2.4e-6 relative; the band keeps a 4x margin).
constexpr double kCutBand = 1.0e-5;
// Entries whose bound on u is below x_cut^2 (1 - kInsideMargin) cannot hold a
// band pair; the margin covers the FP32 rounding of the bound itself.
constexpr double kInsideMargin = 5.0e-5;
// Entries whose lower bound on u exceeds x_cut^2 (1 + kCutBand)(1 + kOutsideMargin)
// hold no pair the FP32 forms keep; the margin covers the FP32 rounding of the bound.
constexpr double kOutsideMargin = 5.0e-5;
// Default bound on x |dH| of the fitted polynomial.
constexpr double kDefaultPolyTol = 1.0e-7;

// Template selectors of the pair kernels.
enum { ACC_F64 = 0, ACC_KAHAN = 1, ACC_F32 = 2 };  // accumulation of the FP32 partials
enum { SOFT_CLAMP = 0, SOFT_PLUMMER = 1 };         // softening

// Arguments of the pair kernels, passed by value (constant bank).
struct PairArgs {
    const LeafMeta *leaf;
    const int64_t *row_off;  // nleaf + 1
    const int *row_src;      // source leaf ids, grouped by sink row
    const float4 *pos4;      // FP32 forms: (x', y', z', w) in the leaf frame, scaled by c
    const double *pos;       // FP64 form: SoA positions
    const double *mass;      // FP64 form: per-particle masses or null
    double *acc;             // SoA 3 * npart, +=
    int *queue;              // persistent work counter (reset to 0 before launch)
    unsigned long long *evaluated;  // nullable: += pair interactions the kernel evaluated
    int npart, nleaf;
    // FP32 forms (scaled units: lengths times c = 1 / (2 r_s))
    float eps2;              // (c * eps)^2
    float u0;                // polynomial expansion point
    float ucut;              // x_cut^2 (or the fitted domain end without cutoff)
    float pad0;
    // Cutoff band: FP32 u in (ucut_lo, ucut_hi] is too close to the cutoff for
    // FP32 rounding to decide; such pairs are re-decided from FP64 positions
    // (box units: r^2 (+ eps^2 for Plummer, max(r^2, eps^2) for clamp) <= rcut2).
    float ucut_lo, ucut_hi;
    double rcut2, eps2_box;
    double cscale;           // c
    double out_scale;        // c^2 * mass (equal masses) or c^2 (per-particle masses)
    float coef[kMaxCoef];    // -H(u) ~ sum coef[k] (u - u0)^k (negated, so f = rinv^2 * rinv + poly)
    float2 coef2[kMaxCoef];  // the same as (coef[k], coef[k]): packed FMA operands read from the
                             // constant bank as they are, with no register pair to build
    float uin;               // entries whose bound on u stays below uin hold no cutoff-band pair
    float uout;              // entries whose lower bound on u exceeds uout hold no kept pair
    // FP64 form (reference units)
    double soft, r_soft, hrrs, rrs, coeff, xcut, mass_eq;
    // Packed launches over several resident boxes (nseg > 0): work items
    // [seg_item[k], seg_item[k + 1]) are the sink leaves seg_leaf[k] + 0, 1, ...
    // of box k; nleaf then counts the items. nseg = 0: item i is leaf i.
    int nseg;
    int leaf_warps;          // sink-register kernels: warps sharing one sink leaf's row (<= 1: one)
    int seg_item[kMaxSeg + 1];
    int seg_leaf[kMaxSeg];
};

}  // namespace p2p
