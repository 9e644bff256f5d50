/*
 * CPU oracle for the TreePM short-range particle-particle (P2P) pass.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker the parity tests,
 * smoke() and bench.py's cpu_baseline leg compare the CUDA path against.
 * Nothing in the product library links or calls it.
 *
 * It restates, in plain C and FP64, what the reference computes on the GPU:
 *   - pair functions: P2P_core_lite (clamp softening, the production kernel)
 *     src/gpu_kernel.impl.h:160-257, non-SPI branch :246-248, and P2P_core_1
 *     (Plummer softening) src/gpu_kernel.impl.h:260-362, non-SPI branch
 *     :278-280 and :350-355;
 *   - the driver order of P2P_kernel3 src/gpu_kernel.impl.h:439-524: one sink
 *     leaf at a time, sources summed in CSR row order, source particles in
 *     index order, then acc[i] += iacc * MASSPART (:516-519);
 *   - the CSR row order produced by the stable thrust::sort_by_key on sink
 *     ids in src/gpu_entry.cu:132-138 (entries of one sink keep list order);
 *   - chunked calls: each task_compute_p2p_gpu call (src/fmm.c:500-515,
 *     src/gpu_entry.cu:124-191) launches on its own chunk of the list, so a
 *     sink's partial sums are added to the device accumulator once per chunk.
 * Pinned against the reference's own pair functions compiled for the host
 * (oracle/ref_pair.cpp, built from the reference sources into oracle/_ref)
 * and against tests/golden fixtures made from them.
 *
 * It also holds an FP64 direct evaluator of the same truncated kernel
 * (cell list, minimum image, per-pair cutoff) that is independent of any
 * tree or interaction list.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORACLE_SOFT_CLAMP = 0, ORACLE_SOFT_PLUMMER = 1 };

typedef struct {
    int soft_mode;        /* ORACLE_SOFT_CLAMP or ORACLE_SOFT_PLUMMER */
    double soften;        /* SoftenScale */
    double split_radius;  /* splitRadius (r_s) */
    double x_cut;         /* per-pair cutoff on x = r / (2 r_s); <= 0: none */
    double mass;          /* MASSPART, used when masses == NULL */
} oracle_params;

/* 2/sqrt(pi): coeff = 2.0 * PIisq, src/gpu_entry.cu:80, src/setparam.c:59 */
static double two_over_sqrt_pi(void) { return 2.0 * (1.0 / sqrt(M_PI)); }

/* P2P_core_lite, FP64, non-SPI (src/gpu_kernel.impl.h:160-257).
 * hrrs = 0.5 / splitRadius (P2P_kernel3 passes HALF*rrs, :465). */
static inline void pair_clamp(double soft, double r_soft, double hrrs, double coeff,
                              double x_cut, const double ii[3], const double jj[3],
                              double acc[3]) {
    double dx = jj[0] - ii[0], dy = jj[1] - ii[1], dz = jj[2] - ii[2];
    double dr2 = dx * dx + dy * dy + dz * dz;
    double dr = soft, rdr = r_soft;
    if (dr2 > soft * soft) {
        rdr = 1.0 / sqrt(dr2);
        dr = rdr * dr2;
    }
    double drs = dr * hrrs;
    if (x_cut > 0.0 && drs > x_cut) return; /* GPUCUTOFF, :192-196 */
    double ir3 = 1.0 / (dr * dr * dr);
    ir3 *= (erfc(drs) + coeff * drs * exp(-drs * drs));
    acc[0] += dx * ir3;
    acc[1] += dy * ir3;
    acc[2] += dz * ir3;
}

/* P2P_core_1, FP64, non-SPI (src/gpu_kernel.impl.h:260-362) with its
 * MASSPART argument set to 1 so the mass is applied by the driver, as
 * P2P_kernel3 does for P2P_core_lite. The reference also zeroes the pair
 * beyond x > 2.8125 unconditionally (:353-355); x_cut carries that value. */
static inline void pair_plummer(double soft, double rrs, double coeff, double x_cut,
                                const double ii[3], const double jj[3], double acc[3]) {
    double dx = jj[0] - ii[0], dy = jj[1] - ii[1], dz = jj[2] - ii[2];
    double dr = sqrt(dx * dx + dy * dy + dz * dz + soft * soft);
    double drs = 0.5 * dr * rrs;
    if (x_cut > 0.0 && drs > x_cut) return;
    double ir3 = 1.0 / (dr * dr * dr);
    ir3 *= (erfc(drs) + coeff * drs * exp(-drs * drs));
    acc[0] += dx * ir3;
    acc[1] += dy * ir3;
    acc[2] += dz * ir3;
}

/* Evaluate one pair on explicit coordinates; exposed for known-answer tests. */
void oracle_pair(const oracle_params *p, const double ii[3], const double jj[3],
                 double out[3]) {
    double coeff = two_over_sqrt_pi();
    out[0] = out[1] = out[2] = 0.0;
    if (p->soft_mode == ORACLE_SOFT_PLUMMER)
        pair_plummer(p->soften, 1.0 / p->split_radius, coeff, p->x_cut, ii, jj, out);
    else
        pair_clamp(p->soften, 1.0 / p->soften, 0.5 * (1.0 / p->split_radius), coeff,
                   p->x_cut, ii, jj, out);
}

/* Stable counting sort of one chunk's entries by sink leaf: the row order the
 * reference's stable sort_by_key produces (src/gpu_entry.cu:132-138). */
static void chunk_csr(int64_t n, const int *task_t, const int *task_s, int nleaf,
                      int64_t *row_begin /* nleaf+1 */, int *row_src /* n */) {
    memset(row_begin, 0, sizeof(int64_t) * (size_t)(nleaf + 1));
    for (int64_t e = 0; e < n; ++e) row_begin[task_t[e] + 1]++;
    for (int l = 0; l < nleaf; ++l) row_begin[l + 1] += row_begin[l];
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)nleaf);
    memcpy(cur, row_begin, sizeof(int64_t) * (size_t)nleaf);
    for (int64_t e = 0; e < n; ++e) row_src[cur[task_t[e]]++] = task_s[e];
    free(cur);
}

/*
 * The reference-list oracle. Positions are SoA (x[0..n), then y, then z),
 * exactly the d_part_pos layout of src/gpu_entry.cu:85-105. Leaf ids in
 * task_t/task_s are 0-based (already rebased by first_leaf, as
 * devMemcpyHD_task does, src/gpu_func.impl.h:704-713). The list is processed
 * in chunks of len_chunk entries (len_chunk <= 0: one chunk), each chunk
 * adding its partial sums into acc (SoA, +=), as successive
 * task_compute_p2p_gpu calls do. masses (nullable) replaces MASSPART by a
 * per-source mass inside the pair sum.
 * Returns the pair-interaction count sum(n_t * n_s) of src/gpu_entry.cu:53-58.
 */
int64_t oracle_p2p_lists(const oracle_params *p, int npart, const double *pos,
                         const double *masses, int nleaf, const int *leaf_ipart,
                         const int *leaf_npart, int64_t ntask, const int *task_t,
                         const int *task_s, int64_t len_chunk, double *acc) {
    const double coeff = two_over_sqrt_pi();
    const double rrs = 1.0 / p->split_radius;
    const double hrrs = 0.5 * rrs;
    const double r_soft = 1.0 / p->soften;
    const double *X = pos, *Y = pos + npart, *Z = pos + 2 * (size_t)npart;
    double *AX = acc, *AY = acc + npart, *AZ = acc + 2 * (size_t)npart;
    int64_t pairs = 0;
    if (len_chunk <= 0) len_chunk = ntask > 0 ? ntask : 1;
    int64_t *row_begin = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nleaf + 1));
    int *row_src = (int *)malloc(sizeof(int) * (size_t)(len_chunk > 0 ? len_chunk : 1));
    for (int64_t c0 = 0; c0 < ntask; c0 += len_chunk) {
        int64_t n = ntask - c0 < len_chunk ? ntask - c0 : len_chunk;
        chunk_csr(n, task_t + c0, task_s + c0, nleaf, row_begin, row_src);
        int64_t cpairs = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : cpairs)
        for (int t = 0; t < nleaf; ++t) {
            int64_t b = row_begin[t], e = row_begin[t + 1];
            if (b == e) continue;
            int iip = leaf_ipart[t], inp = leaf_npart[t];
            for (int64_t k = b; k < e; ++k) cpairs += (int64_t)inp * leaf_npart[row_src[k]];
            for (int i = 0; i < inp; ++i) {
                int pi = iip + i;
                double ii[3] = {X[pi], Y[pi], Z[pi]};
                double iacc[3] = {0.0, 0.0, 0.0};
                for (int64_t k = b; k < e; ++k) {
                    int s = row_src[k];
                    int jip = leaf_ipart[s], jnp = leaf_npart[s];
                    for (int j = 0; j < jnp; ++j) {
                        int pj = jip + j;
                        double jj[3] = {X[pj], Y[pj], Z[pj]};
                        if (masses) {
                            double one[3] = {0.0, 0.0, 0.0};
                            if (p->soft_mode == ORACLE_SOFT_PLUMMER)
                                pair_plummer(p->soften, rrs, coeff, p->x_cut, ii, jj, one);
                            else
                                pair_clamp(p->soften, r_soft, hrrs, coeff, p->x_cut, ii, jj, one);
                            iacc[0] += masses[pj] * one[0];
                            iacc[1] += masses[pj] * one[1];
                            iacc[2] += masses[pj] * one[2];
                        } else if (p->soft_mode == ORACLE_SOFT_PLUMMER) {
                            pair_plummer(p->soften, rrs, coeff, p->x_cut, ii, jj, iacc);
                        } else {
                            pair_clamp(p->soften, r_soft, hrrs, coeff, p->x_cut, ii, jj, iacc);
                        }
                    }
                }
                double m = masses ? 1.0 : p->mass;
                AX[pi] += iacc[0] * m;
                AY[pi] += iacc[1] * m;
                AZ[pi] += iacc[2] * m;
            }
        }
        pairs += cpairs;
    }
    free(row_begin);
    free(row_src);
    return pairs;
}

/* Pair-interaction count of a list: sum over entries of n_t * n_s
 * (src/gpu_entry.cu:53-58). */
int64_t oracle_pair_count(const int *leaf_npart, int64_t ntask, const int *task_t,
                          const int *task_s) {
    int64_t c = 0;
#pragma omp parallel for reduction(+ : c)
    for (int64_t e = 0; e < ntask; ++e) c += (int64_t)leaf_npart[task_t[e]] * leaf_npart[task_s[e]];
    return c;
}

/*
 * FP64 direct oracle: for each requested sink particle, the sum over ALL
 * particles j != i of the same truncated pair kernel, with minimum-image
 * separations in a periodic cube of side box (box <= 0: open boundaries).
 * Independent of the tree and lists; comparable to the list-based pass when
 * the lists hold every leaf pair within r_cut = 2 r_s x_cut and there are no
 * ghost particles. pos is SoA over the n particles of the box; out is SoA
 * over the nsink requested sinks.
 *
 * Candidates come from a cell list of cell side >= r_cut / 2 (5^3 cells
 * around the sink's), with the positions copied into cell order so the scan
 * is sequential; candidates farther than r_cut are rejected on r^2 before
 * the pair function (which makes the exact cutoff decision) is called.
 */
void oracle_direct(const oracle_params *p, int n, const double *pos,
                   const double *masses, double box, int nsink, const int *sinks,
                   double *out) {
    const double coeff = two_over_sqrt_pi();
    const double rrs = 1.0 / p->split_radius;
    const double hrrs = 0.5 * rrs;
    const double r_soft = 1.0 / p->soften;
    const double r_cut = 2.0 * p->split_radius * p->x_cut;
    const double *X = pos, *Y = pos + n, *Z = pos + 2 * (size_t)n;
    const int wrap = box > 0;
    double lo[3] = {0, 0, 0}, span = box;
    if (!wrap) {
        double hi[3] = {X[0], Y[0], Z[0]};
        lo[0] = X[0]; lo[1] = Y[0]; lo[2] = Z[0];
        for (int i = 0; i < n; ++i) {
            const double q[3] = {X[i], Y[i], Z[i]};
            for (int d = 0; d < 3; ++d) {
                if (q[d] < lo[d]) lo[d] = q[d];
                if (q[d] > hi[d]) hi[d] = q[d];
            }
        }
        span = 0;
        for (int d = 0; d < 3; ++d)
            if (hi[d] - lo[d] > span) span = hi[d] - lo[d];
        span *= 1.000001;
        if (span <= 0) span = 1;
    } else {
        /* cells tile [lo, lo + box) per axis, lo the box-multiple at or below
         * the smallest coordinate; positions outside are wrapped into it. */
        double mn = X[0];
        for (int i = 0; i < n; ++i) {
            if (X[i] < mn) mn = X[i];
            if (Y[i] < mn) mn = Y[i];
            if (Z[i] < mn) mn = Z[i];
        }
        lo[0] = lo[1] = lo[2] = floor(mn / box) * box;
    }
    /* r_cut <= 0 (no per-pair cutoff) makes every particle a candidate */
    int nc = r_cut > 0.0 ? (int)floor(span / (0.5 * r_cut)) : 1;
    if (nc < 1) nc = 1;
    if (nc > 256) nc = 256;
    const double cw = span / nc;
    const int64_t ncell = (int64_t)nc * nc * nc;
    int64_t *cstart = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
    int *cell_of = (int *)malloc(sizeof(int) * (size_t)n);
    int *order = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        int c[3];
        const double q[3] = {X[i], Y[i], Z[i]};
        for (int d = 0; d < 3; ++d) {
            double v = q[d] - lo[d];
            if (wrap) v = fmod(fmod(v, box) + box, box);
            int k = (int)floor(v / cw);
            c[d] = k < 0 ? 0 : (k >= nc ? nc - 1 : k);
        }
        cell_of[i] = (c[0] * nc + c[1]) * nc + c[2];
        cstart[cell_of[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)ncell);
        memcpy(cur, cstart, sizeof(int64_t) * (size_t)ncell);
        for (int i = 0; i < n; ++i) order[cur[cell_of[i]]++] = i;
        free(cur);
    }
    /* positions (and masses) in cell order */
    double *cx = (double *)malloc(sizeof(double) * (size_t)n * 4);
    double *cy = cx + n, *cz = cx + 2 * (size_t)n, *cm = cx + 3 * (size_t)n;
    for (int q = 0; q < n; ++q) {
        const int j = order[q];
        cx[q] = X[j]; cy[q] = Y[j]; cz[q] = Z[j];
        cm[q] = masses ? masses[j] : 1.0;
    }
    const int reach = r_cut > 0.0 ? (int)ceil(r_cut / cw) : nc;
    /* candidates beyond this cannot pass the pair's own cutoff test */
    const double reject2 = r_cut > 0.0 ? r_cut * r_cut * (1.0 + 1e-9) : INFINITY;
    const double hb = 0.5 * box;
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < nsink; ++s) {
        const int i = sinks[s];
        const int ci = cell_of[i];
        const int c0 = ci / (nc * nc), c1 = (ci / nc) % nc, c2 = ci % nc;
        const double ii[3] = {X[i], Y[i], Z[i]};
        double a[3] = {0, 0, 0};
        int lim = reach;
        int span_cells = 2 * lim + 1;
        if (span_cells > nc) { lim = nc / 2; span_cells = nc; }
        for (int a0 = -lim; a0 < -lim + span_cells; ++a0)
            for (int a1 = -lim; a1 < -lim + span_cells; ++a1)
                for (int a2 = -lim; a2 < -lim + span_cells; ++a2) {
                    int k0 = c0 + a0, k1 = c1 + a1, k2 = c2 + a2;
                    if (wrap) {
                        k0 = (k0 % nc + nc) % nc; k1 = (k1 % nc + nc) % nc; k2 = (k2 % nc + nc) % nc;
                    } else if (k0 < 0 || k1 < 0 || k2 < 0 || k0 >= nc || k1 >= nc || k2 >= nc) {
                        continue;
                    }
                    const int64_t cc = ((int64_t)k0 * nc + k1) * nc + k2;
                    for (int64_t q = cstart[cc]; q < cstart[cc + 1]; ++q) {
                        double dd[3] = {cx[q] - ii[0], cy[q] - ii[1], cz[q] - ii[2]};
                        if (wrap) {
                            for (int d = 0; d < 3; ++d) {
                                /* minimum image: dd - box * nearbyint(dd / box) */
                                if (dd[d] > hb || dd[d] < -hb) {
                                    if (dd[d] < 3.0 * hb && dd[d] > -3.0 * hb)
                                        dd[d] += dd[d] > 0 ? -box : box;
                                    else
                                        dd[d] -= box * nearbyint(dd[d] / box);
                                }
                            }
                        }
                        if (dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2] > reject2) continue;
                        if (order[q] == i) continue;
                        const double jj[3] = {ii[0] + dd[0], ii[1] + dd[1], ii[2] + dd[2]};
                        double one[3] = {0, 0, 0};
                        if (p->soft_mode == ORACLE_SOFT_PLUMMER)
                            pair_plummer(p->soften, rrs, coeff, p->x_cut, ii, jj, one);
                        else
                            pair_clamp(p->soften, r_soft, hrrs, coeff, p->x_cut, ii, jj, one);
                        a[0] += cm[q] * one[0];
                        a[1] += cm[q] * one[1];
                        a[2] += cm[q] * one[2];
                    }
                }
        const double m = masses ? 1.0 : p->mass;
        out[s] = a[0] * m;
        out[nsink + s] = a[1] * m;
        out[2 * (size_t)nsink + s] = a[2] * m;
    }
    free(cx);
    free(cstart);
    free(cell_of);
    free(order);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
