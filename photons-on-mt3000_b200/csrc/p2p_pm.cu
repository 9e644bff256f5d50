// Particle-mesh (PM) long-range force on the GPU (C ABI p2p_pm_*): the
// complement of the short-range P2P pass in PhotoNs' TreePM split, for one
// periodic domain.
//
//   deposit   cloud-in-cell mass assignment of the particles with tag 1
//             (src/partmesh.c:96-204): FP64 atomics into an N^3 mesh of mass
//             per cell; the reference's scaling to density, times (N / L)^3
//             (src/partmesh.c:319-327), is folded into the Green's function
//   convolve  real-to-complex FFT (cuFFT), times the reference's Green's
//             function pref exp(-k2 s2) / k2 / (sinc_x sinc_y sinc_z)^4 with
//             integer k2, s2 = (2 pi r_s / L)^2, pref = L^2 / (pi N^3), zero
//             mode 0 (src/conv.f90:239-316), complex-to-real FFT without
//             normalisation (pm_green_kernel is this file's own)
//   gradient  the reference's 4-point difference f1 h (M[+1] - M[-1]) -
//             f2 h (M[+2] - M[-2]), f1 = 4/3, f2 = 1/6, h = N / (2 L), per axis
//             (src/partmesh.c:1116-1262), for every cell into one interleaved
//             mesh (gx, gy, gz, 0): 32 bytes, one sector, per cell
//   interp    per particle, the 8 cloud-in-cell cells' gradients weighted as
//             in the deposit and summed in the reference's cell order
//             (src/partmesh.c:1415-1450)
// The reference splits the mesh over MPI sub-domains with halos; on one
// periodic domain every halo read is a periodic wrap. The FFTs are cuFFT
// (the reference calls FFTW through 2DECOMP&FFT); the other steps are the
// kernels below.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "photons_p2p.h"
#include "p2p_host_shared.h"

#define P2P_API extern "C" __attribute__((visibility("default")))

using namespace p2p;

struct p2p_pm {
    int device = 0;
    int n = 0;
    double box = 1.0, split_radius = 1.0;
    double *density = nullptr;      // N^3, mass per cell
    cufftDoubleComplex *spec = nullptr;  // N * N * (N/2 + 1)
    double *potential = nullptr;    // N^3
    double4 *grad = nullptr;        // N^3 cells of (gx, gy, gz, 0)
    double *sinc = nullptr;         // N: sin(pi l / N) / (pi l / N), l the wrapped index
    cufftHandle fwd = 0, inv = 0;
    bool fwd_ok = false, inv_ok = false;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaStream_t stream = nullptr;
};

namespace {

__device__ __forceinline__ int wrap(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// Cell, neighbour cell and the neighbour's weight on one axis
// (src/partmesh.c:99-143): i = (int)(x norm), w = (x - (i + 1/2) delta) norm,
// the neighbour on the side of w, weight |w|.
__device__ __forceinline__ void cic_axis(double x, double norm, double delta, int n, int &c, int &nb, double &w) {
    const int i = (int)__dmul_rn(x, norm);
    double d = __dmul_rn(__dsub_rn(x, __dmul_rn(__dadd_rn((double)i, 0.5), delta)), norm);
    int ii;
    if (d > 0) {
        ii = i + 1;
    } else {
        d = -d;
        ii = i - 1;
    }
    c = wrap(i, n);
    nb = wrap(ii, n);
    w = d;
}

constexpr unsigned kFull = 0xffffffffu;

// Cloud-in-cell deposit, one particle per lane. Whole warps stay converged
// (the loop bound is per warp) so that each of the 8 corners can first be
// summed over lanes that hold the same cell in a run (particles in the same
// cell, next to each other in the input, as in tree or cell order): a
// segmented scan over the lanes, as many steps as the longest run needs,
// then one FP64 atomic per run. A warp whose lanes all differ skips the scan.
__global__ void __launch_bounds__(256) pm_deposit_kernel(const double *__restrict__ pos, const int *__restrict__ tag,
                                                         int npart, double mass, int n, double norm, double delta,
                                                         double *__restrict__ mesh) {
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + threadIdx.x - lane; base < npart; base += stride) {
        const int p = base + lane;
        const bool on = p < npart && (!tag || tag[p] == 1);
        int c[3] = {0, 0, 0}, nb[3] = {0, 0, 0};
        double w[3] = {0.0, 0.0, 0.0};
        if (on)
            for (int a = 0; a < 3; ++a) cic_axis(pos[(size_t)a * npart + p], norm, delta, n, c[a], nb[a], w[a]);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int ix = (q & 1) ? nb[0] : c[0], iy = (q & 2) ? nb[1] : c[1], iz = (q & 4) ? nb[2] : c[2];
            const double wx = (q & 1) ? w[0] : 1.0 - w[0], wy = (q & 2) ? w[1] : 1.0 - w[1],
                         wz = (q & 4) ? w[2] : 1.0 - w[2];
            const int key = on ? (ix * n + iy) * n + iz : -1;
            double v = on ? __dmul_rn(__dmul_rn(__dmul_rn(mass, wx), wy), wz) : 0.0;
            const int prev = __shfl_up_sync(kFull, key, 1), next = __shfl_down_sync(kFull, key, 1);
            const bool head = lane == 0 || prev != key, tail = lane == 31 || next != key;
            const unsigned heads = __ballot_sync(kFull, head);
            if (heads != kFull) {
                // sum each run of equal keys into its last lane: a scan over
                // the lanes that adds lane - d only while it is in the run
                const unsigned upto = heads & (0xffffffffu >> (31 - lane));
                const int first = 31 - __clz(upto);
                const int depth = __reduce_max_sync(kFull, (unsigned)(lane - first));
                for (int d = 1; d <= depth; d <<= 1) {
                    const double vu = __shfl_up_sync(kFull, v, d);
                    if (lane - d >= first) v = __dadd_rn(vu, v);
                }
            }
            if (tail && key >= 0) atomicAdd(&mesh[key], v);
        }
    }
}

// The Green's function on the half spectrum (z halved): block row y is the
// x index i, the flattened (j, kz) runs over threads; l, m are i, j wrapped
// above N/2, n = kz.
__global__ void pm_green_kernel(cufftDoubleComplex *__restrict__ spec, const double *__restrict__ sinc, int n,
                                double s2, double pref, double renormal) {
    const int nz = n / 2 + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * nz) return;
    const int i = blockIdx.y, j = t / nz, kz = t - j * nz;
    const int l = i > n / 2 ? i - n : i, m = j > n / 2 ? j - n : j;
    const size_t q = (size_t)i * n * nz + t;
    double g = 0.0;
    if (l != 0 || m != 0 || kz != 0) {
        const double k2 = (double)(l * l + m * m + kz * kz);
        const double ff = 1.0 / (sinc[i] * sinc[j] * sinc[kz]);
        g = pref * (exp(-k2 * s2) / k2 * (ff * ff * ff * ff)) * renormal;
    }
    spec[q].x *= g;
    spec[q].y *= g;
}

__device__ __forceinline__ int wrap_near(int i, int n) {
    return i < 0 ? i + n : (i >= n ? i - n : i);
}

// The 4-point difference along one axis: row = the cell's offset without
// this axis, v = its coordinate on the axis, s = the axis's stride.
__device__ __forceinline__ double diff4(const double *__restrict__ phi, size_t row, int v, int n, size_t s,
                                       double f1h, double f2h) {
    const double m1 = __ldg(phi + row + (size_t)wrap_near(v - 1, n) * s);
    const double p1 = __ldg(phi + row + (size_t)wrap_near(v + 1, n) * s);
    const double m2 = __ldg(phi + row + (size_t)wrap_near(v - 2, n) * s);
    const double p2 = __ldg(phi + row + (size_t)wrap_near(v + 2, n) * s);
    return __dsub_rn(__dmul_rn(f1h, __dsub_rn(p1, m1)), __dmul_rn(f2h, __dsub_rn(p2, m2)));
}

// One cell per thread: block row y is the x index i, the flattened (j, k)
// runs over threads, so a warp reads and writes consecutive z.
__global__ void __launch_bounds__(256) pm_gradient_kernel(const double *__restrict__ phi, int n, double f1h,
                                                          double f2h, double4 *__restrict__ grad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * n) return;
    const int i = blockIdx.y, j = t / n, k = t - j * n;
    const size_t sx = (size_t)n * n, sy = n;
    double2 *out = reinterpret_cast<double2 *>(grad + (size_t)i * sx + t);
    const double gx = diff4(phi, (size_t)j * sy + k, i, n, sx, f1h, f2h);
    const double gy = diff4(phi, (size_t)i * sx + k, j, n, sy, f1h, f2h);
    const double gz = diff4(phi, (size_t)i * sx + (size_t)j * sy, k, n, 1, f1h, f2h);
    out[0] = make_double2(gx, gy);
    out[1] = make_double2(gz, 0.0);
}

__global__ void __launch_bounds__(256) pm_interp_kernel(const double *__restrict__ pos, const int *__restrict__ tag,
                                                        int npart, int n, double norm, double delta,
                                                        const double4 *__restrict__ grad,
                                                        double *__restrict__ acc) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npart; p += gridDim.x * blockDim.x) {
        double out[3] = {0.0, 0.0, 0.0};
        if (!tag || tag[p] == 1) {
            int c[3], nb[3];
            double w[3];
            for (int a = 0; a < 3; ++a) cic_axis(pos[(size_t)a * npart + p], norm, delta, n, c[a], nb[a], w[a]);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int ix = (q & 1) ? nb[0] : c[0], iy = (q & 2) ? nb[1] : c[1], iz = (q & 4) ? nb[2] : c[2];
                const double wx = (q & 1) ? w[0] : 1.0 - w[0], wy = (q & 2) ? w[1] : 1.0 - w[1],
                             wz = (q & 4) ? w[2] : 1.0 - w[2];
                const double wt = __dmul_rn(__dmul_rn(wx, wy), wz);
                const double2 *g = reinterpret_cast<const double2 *>(grad + ((size_t)ix * n + iy) * n + iz);
                const double2 gxy = __ldg(g), gz = __ldg(g + 1);
                out[0] = __dadd_rn(out[0], __dmul_rn(wt, gxy.x));
                out[1] = __dadd_rn(out[1], __dmul_rn(wt, gxy.y));
                out[2] = __dadd_rn(out[2], __dmul_rn(wt, gz.x));
            }
        }
        acc[p] = out[0];
        acc[(size_t)npart + p] = out[1];
        acc[2 * (size_t)npart + p] = out[2];
    }
}

void destroy(p2p_pm *pm) {
    if (pm->fwd_ok) cufftDestroy(pm->fwd);
    if (pm->inv_ok) cufftDestroy(pm->inv);
    void *ptrs[] = {pm->density, pm->spec, pm->potential, pm->grad, pm->sinc};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : pm->ev)
        if (e) cudaEventDestroy(e);
    delete pm;
}

int grid(size_t n, int threads) {
    size_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (int)b;
}

int fail_cuda(cudaError_t e, const char *what) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return report_error(P2P_ERR_CUDA, msg);
}

}  // namespace

P2P_API int p2p_pm_create(p2p_session *s, int nmesh, double boxsize, double split_radius, p2p_pm **out) {
    if (!s || !out) return report_error(P2P_ERR_ARG, "null argument");
    *out = nullptr;
    if (nmesh < 4 || nmesh > 1024 || (nmesh & 1)) return report_error(P2P_ERR_ARG, "nmesh must be even, in [4, 1024]");
    if (!(boxsize > 0.0) || !(split_radius > 0.0)) return report_error(P2P_ERR_ARG, "box and split radius must be positive");
    cudaError_t e = cudaSetDevice(session_device(s));
    if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
    p2p_pm *pm = new p2p_pm();
    pm->device = session_device(s);
    pm->n = nmesh;
    pm->box = boxsize;
    pm->split_radius = split_radius;
    pm->stream = (cudaStream_t)p2p_session_stream(s);
    const size_t n3 = (size_t)nmesh * nmesh * nmesh, nc = (size_t)nmesh * nmesh * (nmesh / 2 + 1);
    bool ok = cudaMalloc(&pm->density, sizeof(double) * n3) == cudaSuccess &&
              cudaMalloc(&pm->spec, sizeof(cufftDoubleComplex) * nc) == cudaSuccess &&
              cudaMalloc(&pm->potential, sizeof(double) * n3) == cudaSuccess &&
              cudaMalloc(&pm->grad, sizeof(double4) * n3) == cudaSuccess &&
              cudaMalloc(&pm->sinc, sizeof(double) * nmesh) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        destroy(pm);
        return report_error(P2P_ERR_NOMEM, "PM mesh allocation failed");
    }
    {
        std::vector<double> sinc(nmesh);
        for (int i = 0; i < nmesh; ++i) {
            const int l = i > nmesh / 2 ? i - nmesh : i;
            const double a = M_PI * (double)l / (double)nmesh;
            sinc[i] = l == 0 ? 1.0 : std::sin(a) / a;
        }
        ok = cudaMemcpy(pm->sinc, sinc.data(), sizeof(double) * nmesh, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    for (cudaEvent_t &ev : pm->ev)
        if (cudaEventCreate(&ev) != cudaSuccess) ok = false;
    pm->fwd_ok = cufftPlan3d(&pm->fwd, nmesh, nmesh, nmesh, CUFFT_D2Z) == CUFFT_SUCCESS;
    pm->inv_ok = cufftPlan3d(&pm->inv, nmesh, nmesh, nmesh, CUFFT_Z2D) == CUFFT_SUCCESS;
    ok = ok && pm->fwd_ok && pm->inv_ok && cufftSetStream(pm->fwd, pm->stream) == CUFFT_SUCCESS &&
         cufftSetStream(pm->inv, pm->stream) == CUFFT_SUCCESS;
    if (!ok) {
        cudaGetLastError();
        destroy(pm);
        return report_error(P2P_ERR_CUDA, "PM FFT plan or event creation failed");
    }
    *out = pm;
    return P2P_OK;
}

P2P_API int p2p_pm_destroy(p2p_pm *pm) {
    if (!pm) return P2P_OK;
    cudaSetDevice(pm->device);
    cudaStreamSynchronize(pm->stream);
    destroy(pm);
    return P2P_OK;
}

P2P_API int p2p_pm_forces(p2p_pm *pm, int npart, const double *d_pos, const int *d_tag, double mass, double *d_acc) {
    if (!pm) return report_error(P2P_ERR_ARG, "null PM");
    if (npart < 0 || (npart > 0 && (!d_pos || !d_acc))) return report_error(P2P_ERR_ARG, "bad particle arrays");
    cudaError_t e = cudaSetDevice(pm->device);
    if (e != cudaSuccess) return fail_cuda(e, "cudaSetDevice");
    const int n = pm->n;
    const size_t n3 = (size_t)n * n * n;
    const double norm = (double)n / pm->box, delta = 1.0 / norm;
    cudaStream_t st = pm->stream;
    const int threads = 256;
    e = cudaEventRecord(pm->ev[0], st);
    if (e == cudaSuccess) e = cudaMemsetAsync(pm->density, 0, sizeof(double) * n3, st);
    if (e != cudaSuccess) return fail_cuda(e, "PM deposit");
    if (npart) pm_deposit_kernel<<<grid(npart, threads), threads, 0, st>>>(d_pos, d_tag, npart, mass, n, norm, delta, pm->density);
    e = cudaEventRecord(pm->ev[1], st);
    if (e != cudaSuccess) return fail_cuda(e, "PM deposit");
    if (cufftExecD2Z(pm->fwd, pm->density, pm->spec) != CUFFT_SUCCESS) return report_error(P2P_ERR_CUDA, "PM forward FFT failed");
    const double s2 = (2.0 * M_PI * pm->split_radius / pm->box) * (2.0 * M_PI * pm->split_radius / pm->box);
    const double pref = pm->box * pm->box / (M_PI * (double)n * (double)n * (double)n);
    const double renormal = norm * norm * norm;
    const int nz = n / 2 + 1;
    pm_green_kernel<<<dim3((n * nz + threads - 1) / threads, n), threads, 0, st>>>(pm->spec, pm->sinc, n, s2, pref,
                                                                                   renormal);
    if (cufftExecZ2D(pm->inv, pm->spec, pm->potential) != CUFFT_SUCCESS) return report_error(P2P_ERR_CUDA, "PM inverse FFT failed");
    e = cudaEventRecord(pm->ev[2], st);
    if (e != cudaSuccess) return fail_cuda(e, "PM convolution");
    const double h = 0.5 * n / pm->box;
    pm_gradient_kernel<<<dim3((n * n + threads - 1) / threads, n), threads, 0, st>>>(
        pm->potential, n, (4.0 / 3.0) * h, (1.0 / 6.0) * h, pm->grad);
    e = cudaEventRecord(pm->ev[3], st);
    if (e != cudaSuccess) return fail_cuda(e, "PM gradient");
    if (npart)
        pm_interp_kernel<<<grid(npart, threads), threads, 0, st>>>(d_pos, d_tag, npart, n, norm, delta, pm->grad,
                                                                   d_acc);
    e = cudaEventRecord(pm->ev[4], st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e, "PM interpolation");
    count_launches(npart ? 4 : 2);
    return P2P_OK;
}

P2P_API int p2p_pm_timings(p2p_pm *pm, float *ms) {
    if (!pm || !ms) return report_error(P2P_ERR_ARG, "null argument");
    cudaError_t e = cudaEventSynchronize(pm->ev[4]);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = cudaEventElapsedTime(&ms[k], pm->ev[k], pm->ev[k + 1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[4], pm->ev[0], pm->ev[4]);
    if (e != cudaSuccess) return fail_cuda(e, "PM timings");
    return P2P_OK;
}

P2P_API int p2p_pm_download(p2p_pm *pm, double *density, double *potential) {
    if (!pm) return report_error(P2P_ERR_ARG, "null PM");
    cudaError_t e = cudaSetDevice(pm->device);
    const size_t n3 = (size_t)pm->n * pm->n * pm->n;
    if (e == cudaSuccess) e = cudaStreamSynchronize(pm->stream);
    if (e == cudaSuccess && density) e = cudaMemcpy(density, pm->density, sizeof(double) * n3, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && potential) e = cudaMemcpy(potential, pm->potential, sizeof(double) * n3, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail_cuda(e, "PM download");
    return P2P_OK;
}
