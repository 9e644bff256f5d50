/*
 * photons_p2p.h - C ABI of libphotons_p2p.so, the B200 (sm_100a) TreePM
 * short-range particle-particle (P2P) force pass.
 *
 * Plain pointers and sizes, no CUDA or C++ types in the signatures. Every
 * function returns a status (P2P_OK = 0) and records a message readable with
 * p2p_last_error(). Nothing here exits the process; the legacy PhotoNs entry
 * points built on top of it (photons_gpu_entry.h) keep the reference's
 * print-and-exit behaviour.
 *
 * The pass protocol mirrors the reference's task_compute_p2p_gpu call
 * sequence (src/gpu_entry.cu:32-209, src/fmm.c:500-515 and :1275,
 * src/gravity.c:440-449):
 *   p2p_pass_begin        first call of a pass: particles + leaves uploaded,
 *                         device accumulator zeroed    (src/gpu_entry.cu:82-122)
 *   p2p_pass_submit       one list chunk: uploaded, CSR built on the device,
 *                         kernel launched, returns before the GPU finishes
 *                                                       (src/gpu_entry.cu:124-191)
 *   p2p_pass_end          completion barrier, GPU seconds of the pass
 *                                                       (get_last_kntime, src/gpu_func.impl.h:715-730)
 *   p2p_pass_accumulate   acc[d][i] += result           (devMemcpyDH_updateAcc,
 *                                                        src/gpu_func.impl.h:644-681)
 * Leaf ids in task lists are 0-based (first_leaf already subtracted, as
 * devMemcpyHD_task does, src/gpu_func.impl.h:704-713). Positions and
 * accelerations are SoA: x[0..npart), y[0..npart), z[0..npart) - the
 * d_part_pos / d_part_buf layout of the reference.
 */
#ifndef PHOTONS_P2P_H
#define PHOTONS_P2P_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define P2P_OK 0
#define P2P_ERR_ARG 1      /* invalid argument (null pointer, negative size, bad enum) */
#define P2P_ERR_CUDA 2     /* a CUDA runtime call failed; see p2p_last_error() */
#define P2P_ERR_STATE 3    /* call out of protocol order */
#define P2P_ERR_NOMEM 4    /* device allocation failed */
#define P2P_ERR_RANGE 5    /* a leaf id / particle range in the input was out of range;
                              the offending entries were skipped, never dereferenced */
#define P2P_ERR_CAPACITY 6 /* a fixed-capacity buffer is too small for the input */

/* Softening (runtime choice; the reference fixes it per kernel). */
#define P2P_SOFT_CLAMP 0   /* r < eps => r := eps (P2P_core_lite, src/gpu_kernel.impl.h:174-188) */
#define P2P_SOFT_PLUMMER 1 /* r := sqrt(r^2 + eps^2) (P2P_core_1, src/gpu_kernel.impl.h:275-279) */

/* Arithmetic forms of the pass. */
#define P2P_FORM_PLAIN_FP64 0 /* FP64 throughout, CUDA erfc/exp: the drop-in form */
#define P2P_FORM_SPLIT 1      /* FP32 leaf-local pair math, FP64 leaf offsets and
                                 FP64 accumulation, fitted erfc polynomial: the chosen form */
#define P2P_FORM_NAIVE_FP32 2 /* FP32 global coordinates, FP32 accumulation (precision study) */
#define P2P_FORM_KAHAN_FP32 3 /* FP32 leaf-local math, Kahan-compensated FP32 accumulation */

typedef struct {
    int form;            /* P2P_FORM_* */
    int soft_mode;       /* P2P_SOFT_* */
    double soften;       /* SoftenScale (box units) */
    double split_radius; /* splitRadius r_s (box units); x = r / (2 r_s) */
    double x_cut;        /* pairs with x > x_cut contribute nothing (GPUCUTOFF uses
                            2.8125, src/gpu_kernel.impl.h:192-196); <= 0: no cutoff */
    double mass;         /* MASSPART: equal particle mass, used when no masses are given */
    int warps_per_block; /* launch shape of the pair kernel; 0 = default */
    int stage_sources;   /* sources staged per warp in shared memory, multiple of 32,
                            at most 1024; 0 = default */
    int blocks_per_sm;   /* persistent grid = blocks_per_sm * SMs; 0 = as many as fit */
    int kernel_variant;  /* FP32 forms: P2P_VARIANT_*; ignored by the FP64 form */
    double poly_tol;     /* FP32 forms: bound on x * |dH| of the fitted polynomial
                            (H: g(x) = 1 - x^3 H(x^2)); the smallest degree meeting it
                            is used; 0 = default 1e-7 (degree 10 at x_cut 2.25) */
    int warps_per_leaf;  /* sink-register mappings: 1, 2 or 4 warps share one sink leaf's
                            row, each taking a contiguous share of its list entries and
                            adding its partial forces with FP64 atomics (the summation
                            order then varies between runs); 0 = 1. Ignored by the
                            other mappings */
} p2p_params;

/* Lane mappings of the FP32 pair kernel. */
#define P2P_VARIANT_AUTO 0            /* the fastest mapping, P2P_VARIANT_SINK_REGS (session and
                                         ensemble server) */
#define P2P_VARIANT_SINK_LANES 1      /* one lane per sink particle, sources broadcast */
#define P2P_VARIANT_SOURCE_LANES 2    /* one lane per staged source, sinks broadcast */
#define P2P_VARIANT_SOURCE_LANES_X2 3 /* source lanes, two sinks per packed f32x2 instruction,
                                         32-sink tile */
#define P2P_VARIANT_SOURCE_LANES_X2_S16 4 /* the same with a 16-sink tile (fewer registers,
                                             more resident warps; for small leaves) */
#define P2P_VARIANT_SINK_LANES_X2 5       /* packed sink lanes: each lane keeps a sink pair,
                                             the leaf's pairs share the lanes' sources */
#define P2P_VARIANT_SINK_REGS 6           /* each lane keeps four sinks in registers (two packed
                                             pairs) and takes every J-th staged source; sources
                                             are classified per particle against the sink slice's
                                             box (dropped / no cutoff test / cutoff test) */
#define P2P_VARIANT_SINK_REGS8 7          /* the same with eight sinks per lane (four packed pairs)
                                             and 64-sink slices: a leaf of up to 64 particles
                                             stages each source once */

typedef struct p2p_session p2p_session;

/* Fills params with the reference's defaults for the plain drop-in form:
 * clamp softening, x_cut 2.8125, given soften / split radius / mass. */
void p2p_params_default(p2p_params *params);

const char *p2p_status_string(int status);
/* Message of the last failing call on this thread ("" when none). */
const char *p2p_last_error(void);
/* Library version as major*10000 + minor*100 + patch. */
int p2p_version(void);

/* Number of CUDA devices visible to the process (0 when none). */
int p2p_device_count(int *count);

/* Sessions own the device buffers (grow-only) and one CUDA stream. */
int p2p_session_create(int device, p2p_session **out);
int p2p_session_destroy(p2p_session *s);
int p2p_session_set_params(p2p_session *s, const p2p_params *params);
int p2p_session_get_params(const p2p_session *s, p2p_params *params);
/* The cudaStream_t (as void*) every launch of this session goes to. */
void *p2p_session_stream(p2p_session *s);
/* Degree of the fitted polynomial used by the FP32 forms (0 for FP64). */
int p2p_session_poly_degree(const p2p_session *s);
/* Max over the fitted range of x * |P(x^2) - H(x^2)| (H defined by
 * g(x) = 1 - x^3 H(x^2)): the per-pair force error bound of the polynomial
 * in units of the force at x = 1. */
double p2p_session_poly_error(const p2p_session *s);

/* First call of a pass. pos: 3*npart doubles (SoA, host). masses: npart
 * doubles or NULL (equal mass params.mass). leaf_ipart/leaf_npart: nleaf
 * ints, each leaf a range of particle slots [ipart, ipart+npart). */
int p2p_pass_begin(p2p_session *s, int npart, const double *pos, const double *masses,
                   int nleaf, const int *leaf_ipart, const int *leaf_npart);
/* p2p_pass_begin with equal masses for positions that mostly equal the
 * previous pass's: the session keeps the positions of its last host-input
 * begin on the device, and only the chunks flagged in dirty (chunk c holds
 * particles [c*chunk, (c+1)*chunk), all three coordinate rows) are uploaded.
 * The caller guarantees that unflagged chunks equal what it passed before.
 * Every chunk is uploaded when dirty is NULL, when npart differs from the
 * previous host-input pass, or when the session's buffers had to grow.
 * uploaded_bytes (nullable) receives the bytes queued. The device half of
 * PhotoNs' per-pass particle upload (src/gpu_entry.cu:82-122) made
 * incremental; no counterpart in the reference. */
int p2p_pass_begin_update(p2p_session *s, int npart, const double *pos, int nleaf, const int *leaf_ipart,
                          const int *leaf_npart, const unsigned char *dirty, int64_t chunk,
                          int64_t *uploaded_bytes);
/* Same with device pointers (already resident in HBM; not copied). */
int p2p_pass_begin_device(p2p_session *s, int npart, const double *d_pos, const double *d_masses,
                          int nleaf, const int *d_leaf_ipart, const int *d_leaf_npart);
/* One chunk of the interaction list: ntask (sink, source) leaf-id pairs.
 * Host arrays (here and in p2p_pass_begin) are copied asynchronously: arrays
 * in page-locked memory must stay unchanged until p2p_pass_end; pageable
 * arrays may be reused once the call returns (the CUDA runtime stages a
 * pageable source before cudaMemcpyAsync returns). */
int p2p_pass_submit(p2p_session *s, int64_t ntask, const int *task_t, const int *task_s);
int p2p_pass_submit_device(p2p_session *s, int64_t ntask, const int *d_task_t, const int *d_task_s);
/* Completion barrier; *gpu_seconds (nullable) = device time from begin to
 * the last submitted chunk. Reports P2P_ERR_RANGE if any input was out of range. */
int p2p_pass_end(p2p_session *s, double *gpu_seconds);
/* acc[d*npart + i] += result (host SoA doubles). Call after p2p_pass_end. */
int p2p_pass_accumulate(p2p_session *s, double *acc);
/* out[d*npart + i] = result (host SoA doubles, copied). Call after p2p_pass_end. */
int p2p_pass_result(p2p_session *s, double *out);
/* Device pointer to the result (SoA doubles, 3*npart), valid until the next begin. */
int p2p_pass_result_device(p2p_session *s, const double **d_acc);
/* Pair-interaction count sum(n_sink * n_source) of the chunks submitted in
 * the current pass, counted on the device (src/gpu_entry.cu:53-58). */
int p2p_pass_pair_count(p2p_session *s, int64_t *pairs);
/* No counterpart in the reference: of those, the pair interactions the
 * kernels evaluated. The packed FP32 kernels skip list entries whose
 * particles' bounding boxes lie wholly beyond the cutoff (all their pairs
 * would be dropped, so the result is the same); the count excludes them.
 * The sink-register kernel also drops single source particles that lie
 * beyond the cutoff from every sink of a slice, and counts on the device the
 * pairs it evaluates (staged sources times the slice's sinks). */
int p2p_pass_evaluated_pairs(p2p_session *s, int64_t *pairs);

/* Whole pass on device-resident inputs in one call, enqueued on the session
 * stream without waiting: zero, prepare, CSR build, pair kernel. The launch
 * sequence is captured once as a CUDA graph and replayed while the inputs
 * (pointers and sizes) stay the same. Finish with p2p_pass_end. */
int p2p_pass_run_device(p2p_session *s, int npart, const double *d_pos, const double *d_masses,
                        int nleaf, const int *d_leaf_ipart, const int *d_leaf_npart,
                        int64_t ntask, const int *d_task_t, const int *d_task_s);

/* ---- Device list walk (no counterpart in the reference's GPU code) ------
 * The caller's kd-tree, as PhotoNs builds it (build_kdtree / center_kdtree,
 * src/fmm.c:231-327), in device memory; child codes are leaf l -> 2l and
 * node k -> 2k+1, the root is node 0, leaves are numbered in pre-order (the
 * leaves of son[0]'s subtree precede those of son[1]'s). */
typedef struct p2p_walk_tree {
    int nnode, nleaf;
    const int *son;             /* 2*nnode child codes */
    const int *node_first;      /* nnode: smallest leaf id in the node's subtree */
    const double *node_center;  /* 3*nnode (AoS) box centres, src/fmm.c:273-327 */
    const double *node_width;   /* 3*nnode box widths */
    const double *leaf_center;  /* 3*nleaf */
    const double *leaf_width;   /* 3*nleaf */
    const int *leaf_active;     /* nleaf: >= 0 for leaves with a local particle (sinks) */
} p2p_walk_tree;
/* Replaces the caller's walk_task_p2p (src/fmm.c:656-792, acceptance
 * src/fmm.c:409-479, called from fmm_task src/fmm.c:1221-1300) plus the
 * list submit: the P2P lists are walked on the GPU, one warp per sink leaf,
 * straight into CSR rows equal entry for entry to those p2p_pass_submit
 * builds from the serial walk's list, then the pair kernel runs on them.
 * Within an open pass (its leaves are the tree's leaves). Waits for the row
 * count (one device-to-host read); *ntask (nullable) = list entries. The
 * leaves are walked once: rows of up to 2048 entries are kept in a slab the
 * session holds between passes (2048 ids per leaf, halved while it would
 * exceed 8 GB) and gathered, longer rows walked a second time.
 * P2P_ERR_ARG for a child code outside the tree, P2P_ERR_CAPACITY when a
 * sink's pending pairs exceed the walk's fixed stack. */
int p2p_pass_submit_walk(p2p_session *s, const p2p_walk_tree *tree, double cutoff, double open_angle,
                         int64_t *ntask);
/* ---- Device kd-tree (no counterpart in the reference's GPU code) --------
 * Builds on the GPU the tree PhotoNs builds on the host before its walk
 * (build_kdtree / center_kdtree, src/fmm.c:69-122,231-327; leaf.active,
 * src/fmm.c:1226-1236): the same mean splits (axis depth % 3, sampled mean
 * summed in slot order, the same in-place partition), the same particle
 * order, pre-order node and leaf numbering and boxes; the root box is
 * particle_combine's float-rounded bounds widened by 1e-6 boxsize
 * (src/gravity.c:69-121). d_pos: 3*npart doubles (SoA, device), d_tag
 * (nullable: all local): npart ints, 1 for local particles. Runs on the
 * session's stream and returns when the tree is complete. The tree owns its
 * device arrays until p2p_dtree_free. P2P_ERR_CAPACITY when the tree needs
 * more than min(npart + 1, 8 npart / maxleaf + 1024) nodes or leaves. */
typedef struct p2p_dtree p2p_dtree;
int p2p_dtree_build(p2p_session *s, int npart, const double *d_pos, const int *d_tag, int maxleaf,
                    double boxsize, p2p_dtree **out);
int p2p_dtree_free(p2p_dtree *t);
/* Rebuilds t in place (PhotoNs rebuilds its tree every step): the same tree
 * p2p_dtree_build makes from these inputs, in t's device arrays where they
 * are large enough (a rebuild of the same or a smaller size allocates
 * nothing; the build's temporaries stay in the session's scratch). Device
 * pointers of t may change: read them again (p2p_dtree_device_arrays,
 * p2p_dtree_walk_tree). On an error t holds no tree (counts 0) until the
 * next successful rebuild, and must still be freed. */
int p2p_dtree_rebuild(p2p_session *s, p2p_dtree *t, int npart, const double *d_pos, const int *d_tag,
                      int maxleaf, double boxsize);
/* Sizes and the build's device time (ms, CUDA events; nullable outputs). */
int p2p_dtree_counts(const p2p_dtree *t, int *npart, int *nleaf, int *nnode, float *build_ms);
/* Device arrays owned by the tree (nullable outputs): positions in tree
 * order (3*npart SoA), perm[slot] = input index, leaf particle ranges: the
 * inputs of p2p_pass_begin_device. */
int p2p_dtree_device_arrays(const p2p_dtree *t, const double **d_pos, const int **d_perm,
                            const int **d_leaf_ipart, const int **d_leaf_npart);
/* The node and leaf tables as the walk reads them (p2p_pass_submit_walk). */
int p2p_dtree_walk_tree(const p2p_dtree *t, p2p_walk_tree *tree);
/* Reorders a per-particle SoA result (3*npart doubles, device) from tree
 * order to the order of the build's input positions: d_out[d*npart +
 * perm[i]] = d_in[d*npart + i]. Queued on the session's stream. */
int p2p_dtree_unpermute(const p2p_dtree *t, p2p_session *s, const double *d_in, double *d_out);
/* Host copies of the tree (every output nullable; sizes from p2p_dtree_counts;
 * centres and widths AoS, 3 per entry; son 2 per node). */
int p2p_dtree_download(const p2p_dtree *t, double *pos, int *perm, int *leaf_ipart, int *leaf_npart,
                       int *leaf_active, double *leaf_center, double *leaf_width, int *son, int *node_first,
                       double *node_center, double *node_width);

/* ---- Particle-mesh long-range force (the TreePM complement) ------------
 * Replaces partmesh_kick's force part (src/partmesh.c:12-1470 with
 * src/conv.f90:239-330) for one periodic domain: cloud-in-cell deposit of
 * the particles with tag 1, scaled to density by (N/L)^3, FFT, times the
 * Green's function pref exp(-k2 (2 pi r_s / L)^2) / k2 / (sinc_x sinc_y
 * sinc_z)^4 (integer wave numbers, pref = L^2 / (pi N^3), zero mode 0),
 * inverse FFT without normalisation, the 4-point difference (4/3, 1/6,
 * step N / (2 L)) per axis, cloud-in-cell interpolation. The reference's MPI
 * sub-domains and halos become periodic wraps; the FFTs are cuFFT (the
 * reference calls FFTW through 2DECOMP&FFT). Device memory: N^3 doubles
 * (mass), N^3 (potential), 4 N^3 (interleaved gradient), N^2 (N/2 + 1)
 * complex, allocated at create.
 * nmesh even in [4, 1024]; positions in [0, boxsize). */
typedef struct p2p_pm p2p_pm;
int p2p_pm_create(p2p_session *s, int nmesh, double boxsize, double split_radius, p2p_pm **out);
int p2p_pm_destroy(p2p_pm *pm);
/* Queues the PM force on the session's stream: d_pos 3*npart doubles (SoA,
 * device), d_tag nullable (all tag 1), equal masses; d_acc (3*npart doubles,
 * SoA, device) receives the long-range acceleration, 0 for tag != 1. */
int p2p_pm_forces(p2p_pm *pm, int npart, const double *d_pos, const int *d_tag, double mass, double *d_acc);
/* Device times in ms of the last p2p_pm_forces (waits for it): deposit,
 * FFT-Green-FFT, gradient, interpolation, total. */
int p2p_pm_timings(p2p_pm *pm, float ms[5]);
/* Host copies of the last deposit (mass per cell, index (x N + y) N + z) and
 * potential (nullable outputs, N^3 doubles each). */
int p2p_pm_download(p2p_pm *pm, double *mass_mesh, double *potential);

/* ---- Far field within the cutoff: P2M, M2M, M2L, L2L, L2P --------------
 * The multipole part of PhotoNs' short-range FMM on the kd-tree of the P2P
 * pass: p2m / walk_m2m (src/operator.c:14-199, src/fmm.c:975-979), the M2L
 * dual-tree walk and m2l with the erfc-truncated kernel (walk_task_m2l +
 * task_compute_m2l, src/fmm.c:812-957 and :1188-1217; m2l LONGSHORT,
 * src/operator.c:331-475), walk_l2l (:477-606) and l2p on the leaves that
 * hold a local particle (:203-262, src/gravity.c:427-428); octupole order,
 * the reference's 20-coefficient layout. The tree is the walk's
 * (p2p_walk_tree: device arrays, e.g. from p2p_dtree_walk_tree); d_pos
 * (3*npart doubles, SoA, tree order) and the leaf ranges are the pass's.
 * d_acc (3*npart doubles, SoA, device) receives the far-field acceleration
 * of the particles of active leaves, 0 for the others. Equal masses.
 * min_r2: M2L tasks whose centres lie closer than sqrt(min_r2) contribute
 * nothing. The reference's m2l tests abs(r2) <= 1e-15 with the integer abs()
 * (src/operator.c:340-344), which skips every task with r2 < 1 in its length
 * unit: min_r2 = 1 reproduces it, 1e-15 what the test evidently means.
 * Queued on the session's stream; the M2L walk reads one count per tree
 * level back to the host, so the call returns when the pass is done. */
typedef struct p2p_fmm p2p_fmm;
int p2p_fmm_create(p2p_session *s, p2p_fmm **out);
int p2p_fmm_destroy(p2p_fmm *f);
int p2p_fmm_far(p2p_fmm *f, const p2p_walk_tree *t, int npart, const double *d_pos, const int *d_leaf_ipart,
                const int *d_leaf_npart, double mass, double split_radius, double cutoff, double open_angle,
                double min_r2, double *d_acc);
/* Counts and device times (ms: upward, walk, M2L, downward, total; nullable
 * outputs) of the last p2p_fmm_far: M2L tasks, tasks applied (r2 >= min_r2),
 * walk levels. */
int p2p_fmm_stats(p2p_fmm *f, int64_t *n_m2l, int64_t *n_applied, int *levels, float ms[5]);
/* Host copies (nullable) of the leaves' multipoles after P2M and their locals
 * after L2L, 20 doubles per leaf in the reference's coefficient order. */
int p2p_fmm_download(p2p_fmm *f, double *leaf_M, double *leaf_L);

/* Host copy of the CSR rows of the last submitted chunk or walk (row_off:
 * nleaf+1 entries; row_src (nullable: rows not copied): row_off[nleaf]
 * entries). Call after p2p_pass_end. */
int p2p_pass_rows(p2p_session *s, int64_t *row_off, int *row_src);

/* Waits for all work queued on the session stream. */
int p2p_session_synchronize(p2p_session *s);

/* Number of kernels this library has launched in the process (graph replays
 * count each kernel node), for launch accounting. */
int64_t p2p_kernel_launch_count(void);

/* Duration in ms of the last pair-kernel launch of the session, measured with
 * CUDA events on the session stream (0 if none). Call after p2p_pass_end. */
int p2p_session_last_kernel_ms(p2p_session *s, float *ms);

/* ---- Allocation-free pass (no counterpart in the reference) ------------
 * For callers that cannot have a library call cudaMalloc / cudaFree while
 * they run: codes that reserve nearly all device memory for their own pool
 * at start-up, processes held to a fixed device-memory quota on a shared GPU,
 * and codes that keep other work running on their own streams (cudaFree
 * synchronises the whole device; this call waits for its own stream only).
 * The pass's scratch is one file-scope __device__ array of
 * P2P_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * the process exits; nothing else is allocated (no cudaMalloc / cudaFree, no
 * allocating library call, no session).
 *
 * Inputs and the output are caller device pointers: d_pos (3*npart doubles,
 * SoA), the leaf ranges, the (sink, source) list, and d_acc (3*npart doubles,
 * SoA), which is overwritten with the result. Equal masses (params->mass).
 * Forms: P2P_FORM_SPLIT (packed source-lane kernel) or P2P_FORM_PLAIN_FP64.
 * The pass is queued on `stream` (a cudaStream_t, 0 for the default stream)
 * and the call blocks the calling host thread until the pass has finished
 * on that stream (it reads the pass's status word there); other streams and
 * the rest of the device are not synchronised. The numeric fields of params
 * are checked as p2p_session_set_params checks them; warps_per_block,
 * blocks_per_sm, kernel_variant and warps_per_leaf are ignored (the split
 * form always runs the packed source-lane kernel, 4 warps per block, as many
 * blocks as fit, one warp per sink leaf).
 *
 * Limit: the scratch needed, about 16*npart (split form only) + 48*nleaf +
 * 4*ntask bytes plus 256-byte alignment of each piece, must fit in
 * P2P_NOALLOC_SCRATCH_BYTES; larger passes return P2P_ERR_CAPACITY before
 * anything is queued. Set-up: the first call on a device resolves the
 * array's device address with cudaGetSymbolAddress (that device current), so
 * make the first call on each device before any stream capture. All calls
 * share the one array: calls whose work overlaps on the GPU (other threads or
 * streams) race and must be serialised by the caller. Errors are reported by
 * the status only; p2p_last_error() is not updated by this call. */
#define P2P_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int p2p_pass_noalloc(const p2p_params *params, int npart, const double *d_pos, int nleaf,
                     const int *d_leaf_ipart, const int *d_leaf_npart, int64_t ntask,
                     const int *d_task_t, const int *d_task_s, double *d_acc, void *stream);

/* Measured FP32 FFMA throughput of this GPU (TFLOP/s, FMA = 2 flops) from a
 * dependent-chain microbenchmark run on the session stream. */
int p2p_measure_fp32_peak(p2p_session *s, double *tflops);

/* Measured FP64 DFMA throughput of this GPU (TFLOP/s, FMA = 2 flops), the
 * same microbenchmark in double precision. */
int p2p_measure_fp64_peak(p2p_session *s, double *tflops);

/* ---- Serving an ensemble of boxes (no counterpart in the reference) -----
 * A server takes force-pass requests for many independent periodic boxes.
 * Each box's particles, leaf frames and CSR list are built once on the
 * device and stay resident in an arena of fixed size (hbm_bytes); a box is
 * admitted when its footprint fits, evicting least recently used idle boxes
 * when it does not, and otherwise waits until memory frees up. Requests of
 * different boxes that are pending together are packed into one persistent
 * pair-kernel launch (up to max_pack boxes); up to `slots` launches are in
 * flight at once on their own streams, so requests arriving while others run
 * are admitted as slots and memory free up and run alongside them. A box's
 * result does not depend on which other boxes share its launch.
 *
 * Units. All boxes share the kernel shape `shape` (form, softening mode,
 * x_cut, poly_tol, kernel variant, and soften / split_radius in shape length
 * units; shape->mass is ignored). A box is given in its own length unit with
 * length_scale = (shape length unit) / (box length unit), i.e. box positions
 * times length_scale are shape positions: a box with split radius r_s and
 * softening eps uses length_scale = shape->split_radius / r_s and then has
 * eps = shape->soften / length_scale. Its result is in box units with the
 * box's equal particle mass `mass`. */
typedef struct p2p_server p2p_server;

typedef struct {
    int slots;                 /* packed launches in flight at once; 0: 1 (measured best
                                  throughput; results still drain on a copy stream while
                                  the next launch computes) */
    int max_pack;              /* boxes per launch, 1..32; 0: 32 */
    int full_grid;             /* 0: each launch takes 1/slots of the GPU's resident
                                  blocks; 1 (default): every launch takes all of them */
    size_t hbm_bytes;          /* device memory for resident boxes; 0: half the free memory */
    double rows_per_particle;  /* arena split hint: list entries per particle; 0: 24 */
    double particles_per_leaf; /* arena split hint; 0: 16 */
    double batch_window_ms;    /* 0 (default): a free slot launches whatever is pending.
                                  > 0: pending requests wait up to this long (from the
                                  oldest one's submit) for others to share their launch,
                                  unless the pack already holds max_pack boxes or
                                  min_pack_pairs pair interactions; at most 1e4 */
    double min_pack_pairs;     /* work at which a pack launches without waiting; 0: none */
} p2p_server_config;

typedef struct {
    int64_t requests_done;
    int64_t launches;          /* packed pair-kernel launches */
    int64_t boxes_launched;    /* sum over launches of boxes packed */
    int64_t builds;            /* residency builds (first admission or re-admission) */
    int64_t evictions;
    int64_t pairs;             /* pair interactions computed */
    double kernel_ms;          /* sum over launches of pair-kernel time (CUDA events) */
    double build_ms;           /* sum over builds of their device time */
    int resident_boxes;
    size_t resident_bytes, capacity_bytes;
} p2p_server_stats;

void p2p_server_config_default(p2p_server_config *cfg);
int p2p_server_create(int device, const p2p_params *shape, const p2p_server_config *cfg,
                      p2p_server **out);
/* Waits for every submitted request, then frees everything. */
int p2p_server_destroy(p2p_server *srv);
/* Registers a box (nothing is copied yet). pos: 3*npart doubles, SoA, in the
 * box's tree order; leaf ranges and the (sink, source) list as for
 * p2p_pass_begin / p2p_pass_submit. result_slots (nresult particle slots,
 * may be NULL) selects and orders the particles whose accelerations a
 * request returns, e.g. the local particles in their original order without
 * the ghosts; NULL returns every particle in slot order (nresult ignored).
 * The host arrays are read whenever the box is (re)admitted and must stay
 * valid and unchanged until the server is destroyed. Checks every range
 * (P2P_ERR_RANGE) and that the box fits in the arena at all
 * (P2P_ERR_CAPACITY). Preloaded boxes (p2p_server_preload) are exempt from
 * the lifetime rule once that call has returned. */
int p2p_server_add_box(p2p_server *srv, double length_scale, double mass, int npart,
                       const double *pos, int nleaf, const int *leaf_ipart, const int *leaf_npart,
                       int64_t ntask, const int *task_t, const int *task_s, int nresult,
                       const int *result_slots, int *box_id);
/* Makes the box resident now and pins it (never evicted); after it returns
 * the box's host arrays are no longer read and may be freed. Returns
 * P2P_ERR_CAPACITY if it cannot fit beside the pinned and queued boxes. */
int p2p_server_preload(p2p_server *srv, int box_id);
/* Device bytes the box holds while resident. */
int p2p_server_box_bytes(p2p_server *srv, int box_id, size_t *bytes);
/* Queues one force pass of the box. out: 3*nresult doubles (3*npart without
 * a result map) of page-locked host memory (p2p_host_alloc, cudaHostAlloc or
 * cudaHostRegister), SoA, overwritten with the selected particles'
 * accelerations in box units. */
int p2p_server_submit(p2p_server *srv, int box_id, double *out, int64_t *ticket);
/* Blocks until the request's result is in `out`; latency_s (may be null) is
 * the time from its submit to that moment. */
int p2p_server_wait(p2p_server *srv, int64_t ticket, double *latency_s);
/* Non-blocking: *done = 1 and the latency once the result is in `out`. */
int p2p_server_query(p2p_server *srv, int64_t ticket, int *done, double *latency_s);
/* Blocks until every submitted request has finished. */
int p2p_server_drain(p2p_server *srv);
/* Changes the batching window of a running server (the config fields
 * batch_window_ms and min_pack_pairs); applies from the next scheduling
 * round. */
int p2p_server_set_batching(p2p_server *srv, double batch_window_ms, double min_pack_pairs);
int p2p_server_get_stats(p2p_server *srv, p2p_server_stats *stats);
/* Page-locked, device-mapped host memory for server results. */
int p2p_host_alloc(size_t bytes, void **ptr);
int p2p_host_free(void *ptr);

#ifdef __cplusplus
}
#endif

#endif /* PHOTONS_P2P_H */
