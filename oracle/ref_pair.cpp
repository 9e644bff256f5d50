/*
 * TEST INFRASTRUCTURE ONLY: the reference's own P2P pair arithmetic, compiled
 * for the host from the reference sources (src/gpu_kernel.impl.h, included
 * from the reference tree at build time, never copied), driven in the order
 * of P2P_kernel3 (src/gpu_kernel.impl.h:439-524) over a stable sink-sorted
 * CSR (src/gpu_entry.cu:132-138). Built by oracle/build_ref.sh into
 * oracle/_ref with one of:
 *   -DGPU_DP [-DGPUCUTOFF]        FP64, erfc/exp direct      (REF_SUFFIX dp / dp_cut)
 *   -DSPI -DGPUCUTOFF             FP32, 512-entry SPI tables  (REF_SUFFIX sp_spi)
 * The FP32 SPI build is the reference's production arithmetic (Makefile:70-75)
 * and is the timed CPU reference arm; the FP64 builds pin oracle/p2p_oracle.c.
 */
#include "cuda_host_shim.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#ifndef REF_SUFFIX
#error "REF_SUFFIX must name the build variant"
#endif

/* Each variant gets its own namespace so the three builds link together. */
namespace REF_SUFFIX {
#include "gpu_kernel.impl.h"
}
using namespace REF_SUFFIX;
#define REF_CAT2(a, b) a##_##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF_FN(name) REF_CAT(name, REF_SUFFIX)

namespace {

/* SPI tables, filled as every CTA of P2P_kernel3 fills them
 * (src/gpu_kernel.impl.h:453-459), here once per call. */
struct SpiTables {
    gpuT tab0[NTABINT];
    gpuT tab1[NTABINT];
    explicit SpiTables(gpuT coeff) {
        gpuT x, neg_two = -2.0;
        for (int i = 0; i < NTABINT; ++i) {
            x = (gpuT)i * WIDTH;
            tab0[i] = erfc(x) + x * exp(-x * x) * coeff;
            tab1[i] = neg_two * coeff * exp(-x * x);
        }
    }
};

void stable_csr(int64_t n, const int *task_t, const int *task_s, int nleaf,
                std::vector<int64_t> &row_begin, std::vector<int> &row_src) {
    row_begin.assign((size_t)nleaf + 1, 0);
    row_src.resize((size_t)n);
    for (int64_t e = 0; e < n; ++e) row_begin[task_t[e] + 1]++;
    for (int l = 0; l < nleaf; ++l) row_begin[l + 1] += row_begin[l];
    std::vector<int64_t> cur(row_begin.begin(), row_begin.end() - 1);
    for (int64_t e = 0; e < n; ++e) row_src[cur[task_t[e]]++] = task_s[e];
}

}  // namespace

extern "C" {

/*
 * soft_mode 0: P2P_core_lite (clamp), 1: P2P_core_1 (Plummer, MASSPART
 * argument 1, mass applied after the row as P2P_kernel3 does).
 * pos: SoA doubles, cast to gpuT like the SoA pack of src/gpu_entry.cu:85-105.
 * acc: SoA doubles, += gpuT partials per chunk (devMemcpyDH_updateAcc,
 * src/gpu_func.impl.h:644-681). Returns the pair-interaction count.
 */
int64_t REF_FN(ref_p2p_lists)(int soft_mode, double soften, double split_radius, double mass,
                              int npart, const double *pos, int nleaf, const int *leaf_ipart,
                              const int *leaf_npart, int64_t ntask, const int *task_t,
                              const int *task_s, int64_t len_chunk, double *acc) {
    gpuT SoftenScale = (gpuT)soften;
    gpuT rrs = 1.0 / split_radius;       /* src/gpu_entry.cu:79 */
    gpuT coeff = 2.0 * (1.0 / sqrt(M_PI)); /* src/gpu_entry.cu:80 with PIisq */
    gpuT hrrs = HALF * rrs, r_SoftenScale = 1.0 / SoftenScale; /* :465 */
    gpuT MASSPART = (gpuT)mass;
#ifdef SPI
    SpiTables tabs(coeff);
#endif
    std::vector<gpuT> P((size_t)npart * 3);
    for (size_t i = 0; i < P.size(); ++i) P[i] = (gpuT)pos[i];
    const gpuT *dev_part_pos = P.data();
    int64_t pairs = 0;
    if (len_chunk <= 0) len_chunk = ntask > 0 ? ntask : 1;
    std::vector<int64_t> row_begin;
    std::vector<int> row_src;
    std::vector<gpuT> buf((size_t)npart * 3, (gpuT)0);
    for (int64_t c0 = 0; c0 < ntask; c0 += len_chunk) {
        int64_t n = ntask - c0 < len_chunk ? ntask - c0 : len_chunk;
        stable_csr(n, task_t + c0, task_s + c0, nleaf, row_begin, row_src);
        int64_t cpairs = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : cpairs)
        for (int t = 0; t < nleaf; ++t) {
            int64_t b = row_begin[t], e = row_begin[t + 1];
            if (b == e) continue;
            int iip = leaf_ipart[t], inp = leaf_npart[t];
            for (int64_t k = b; k < e; ++k) cpairs += (int64_t)inp * leaf_npart[row_src[k]];
            for (int tid = 0; tid < inp; ++tid) {
                gpuT3 ipos, jpos, iacc;
                ipos.x = dev_part_pos[tid + iip];
                ipos.y = dev_part_pos[tid + iip + npart];
                ipos.z = dev_part_pos[tid + iip + 2 * npart];
                iacc.x = iacc.y = iacc.z = 0.0;
                for (int64_t j = b; j < e; ++j) {
                    int jnode = row_src[j];
                    int jip = leaf_ipart[jnode], jnp = leaf_npart[jnode];
                    for (int k = 0; k < jnp; ++k) {
                        jpos.x = dev_part_pos[k + jip];
                        jpos.y = dev_part_pos[k + jip + npart];
                        jpos.z = dev_part_pos[k + jip + 2 * npart];
                        if (soft_mode == 1) {
#ifdef SPI
                            iacc = P2P_core_1(SoftenScale, (gpuT)1.0, rrs, coeff, ipos, jpos, iacc,
                                              tabs.tab0, tabs.tab1);
#else
                            iacc = P2P_core_1(SoftenScale, (gpuT)1.0, rrs, coeff, ipos, jpos, iacc);
#endif
                        } else {
#ifdef SPI
                            iacc = P2P_core_lite(SoftenScale, r_SoftenScale, hrrs, coeff, ipos, jpos,
                                                 iacc, tabs.tab0, tabs.tab1);
#else
                            iacc = P2P_core_lite(SoftenScale, r_SoftenScale, hrrs, coeff, ipos, jpos,
                                                 iacc);
#endif
                        }
                    }
                }
                buf[tid + iip] += iacc.x * MASSPART;
                buf[tid + iip + npart] += iacc.y * MASSPART;
                buf[tid + iip + 2 * npart] += iacc.z * MASSPART;
            }
        }
        pairs += cpairs;
    }
    for (size_t i = 0; i < buf.size(); ++i) acc[i] += (double)buf[i];
    return pairs;
}

/* One pair through the reference function, for known-answer tests. */
void REF_FN(ref_pair)(int soft_mode, double soften, double split_radius, const double *ii,
                      const double *jj, double *out) {
    gpuT SoftenScale = (gpuT)soften;
    gpuT rrs = 1.0 / split_radius;
    gpuT coeff = 2.0 * (1.0 / sqrt(M_PI));
    gpuT hrrs = HALF * rrs, r_SoftenScale = 1.0 / SoftenScale;
#ifdef SPI
    SpiTables tabs(coeff);
#endif
    gpuT3 a, i3, j3;
    a.x = a.y = a.z = 0;
    i3.x = (gpuT)ii[0]; i3.y = (gpuT)ii[1]; i3.z = (gpuT)ii[2];
    j3.x = (gpuT)jj[0]; j3.y = (gpuT)jj[1]; j3.z = (gpuT)jj[2];
#ifdef SPI
    if (soft_mode == 1) a = P2P_core_1(SoftenScale, (gpuT)1.0, rrs, coeff, i3, j3, a, tabs.tab0, tabs.tab1);
    else a = P2P_core_lite(SoftenScale, r_SoftenScale, hrrs, coeff, i3, j3, a, tabs.tab0, tabs.tab1);
#else
    if (soft_mode == 1) a = P2P_core_1(SoftenScale, (gpuT)1.0, rrs, coeff, i3, j3, a);
    else a = P2P_core_lite(SoftenScale, r_SoftenScale, hrrs, coeff, i3, j3, a);
#endif
    out[0] = a.x; out[1] = a.y; out[2] = a.z;
}

}  // extern "C"
