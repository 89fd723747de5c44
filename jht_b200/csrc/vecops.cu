// FP64 vector kernels for the analysis (Jacobi) and CG drivers.
//
//   jhtb_weighted_residual  out = W (m - S a), W the per-pixel quadrature weight
//                           (jht _analysis.py:49-60, weights.py:86-106)
//   jhtb_axpy               y += alpha x           (_analysis.py:60, masked.py:313)
//   jhtb_dot                FP64 inner product, fixed reduction order (masked.py:313)
// All are HBM-bound streaming kernels: grid-stride loops, 8-byte coalesced accesses.
#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kVecThreads = 256;
constexpr int kDotBlocks = 1184;  // 8 x 148 SMs

__global__ void weighted_residual_kernel(const double *__restrict__ maps, const double *__restrict__ synth,
                                         const double *__restrict__ ring_w, double *__restrict__ out,
                                         long long npix, int nside, long long total) {
    const double base = 4.0 * M_PI / (double)npix;
    const long long ncap = 2LL * nside * (nside - 1);  // pixels in one polar cap
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long pix = i % npix;
        double w = base;
        if (ring_w) {
            // ring index of the pixel (RING scheme), then its north partner r' <= 2 nside - 1
            long long r;
            if (pix < ncap) {
                // north cap: ring i (1-based) starts at 2 i (i - 1)
                long long ii = (long long)floor(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)pix)));
                while (2 * ii * (ii - 1) > pix) --ii;
                while (2 * (ii + 1) * ii <= pix) ++ii;
                r = ii - 1;
            } else if (pix < npix - ncap) {
                r = (nside - 1) + (pix - ncap) / (4LL * nside);
            } else {
                const long long q = npix - 1 - pix;  // mirrored index into the south cap
                long long ii = (long long)floor(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)q)));
                while (2 * ii * (ii - 1) > q) --ii;
                while (2 * (ii + 1) * ii <= q) ++ii;
                r = 4LL * nside - 2 - (ii - 1);
            }
            const long long half = r < 2LL * nside ? r : 4LL * nside - 2 - r;
            w = JHTB_IN(half, 2LL * nside, 501) ? base * (1.0 + ring_w[half]) : 0.0;  // the ring weights of the half grid
        }
        const double v = synth ? maps[i] - synth[i] : maps[i];
        out[i] = w * v;
    }
}

__global__ void axpy_kernel(long long n, double alpha, const double *__restrict__ x, double *__restrict__ y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = fma(alpha, x[i], y[i]);
}

// Two-pass deterministic dot: fixed per-block partials, then one block sums them in order.
__global__ void dot_partial_kernel(long long n, const double *__restrict__ x, const double *__restrict__ y,
                                   double *__restrict__ part) {
    __shared__ double sh[kVecThreads];
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc = fma(x[i], y[i], acc);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kVecThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void dot_final_kernel(int nparts, const double *__restrict__ part, double *__restrict__ result) {
    __shared__ double sh[kVecThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += part[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kVecThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *result = sh[0];
}

int grid_for(long long n) {
    long long g = (n + kVecThreads - 1) / kVecThreads;
    if (g > 148LL * 16) g = 148LL * 16;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

JHTB_DEBUG_ACCESSOR(vecops)
}  // namespace jhtb

using namespace jhtb;

extern "C" {

int jhtb_weighted_residual(const jhtb_plan *plan, const double *maps, const double *synth, const double *ring_w,
                           double *out, int batch, void *stream) {
    if (!plan || !maps || !out) return fail(JHTB_ERR_INVALID, "jhtb_weighted_residual: NULL argument");
    if (batch < 0) return fail(JHTB_ERR_INVALID, "jhtb_weighted_residual: negative batch");
    const Plan &p = *reinterpret_cast<const Plan *>(plan);
    if (p.rings_only) return fail(JHTB_ERR_INVALID, "jhtb_weighted_residual: HEALPix plans only");
    const long long total = (long long)batch * p.ncomp * p.npix;
    if (total == 0) return JHTB_OK;
    weighted_residual_kernel<<<grid_for(total), kVecThreads, 0, (cudaStream_t)stream>>>(maps, synth, ring_w, out,
                                                                                        p.npix, p.nside, total);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int jhtb_axpy(int64_t n, double alpha, const double *x, double *y, void *stream) {
    if (n < 0 || (n > 0 && (!x || !y))) return fail(JHTB_ERR_INVALID, "jhtb_axpy: bad argument");
    if (n == 0) return JHTB_OK;
    axpy_kernel<<<grid_for(n), kVecThreads, 0, (cudaStream_t)stream>>>(n, alpha, x, y);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int jhtb_dot(const jhtb_plan *plan, int64_t n, const double *x, const double *y, double *result, void *stream) {
    if (!plan || n < 0 || !result || (n > 0 && (!x || !y))) return fail(JHTB_ERR_INVALID, "jhtb_dot: bad argument");
    const Plan &p = *reinterpret_cast<const Plan *>(plan);
    cudaStream_t s = (cudaStream_t)stream;
    int nb = (int)((n + kVecThreads - 1) / kVecThreads);
    if (nb > kDotBlocks) nb = kDotBlocks;
    if (nb < 1) nb = 1;
    dot_partial_kernel<<<nb, kVecThreads, 0, s>>>(n, x, y, p.d_scratch);
    dot_final_kernel<<<1, kVecThreads, 0, s>>>(nb, p.d_scratch, result);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// FP64 FMA throughput probe (the denominator of the FP64 roofline fraction)
// ---------------------------------------------------------------------------------------
namespace jhtb {
namespace {
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(int iters, double *sink) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-10, a2 = a0 + 2e-10, a3 = a0 + 3e-10;
    double a4 = a0 + 4e-10, a5 = a0 + 5e-10, a6 = a0 + 6e-10, a7 = a0 + 7e-10;
    const double b = 0.999999999, c = 1e-12;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.6789) sink[0] = s;  // never true; keeps the chains live
}
}  // namespace
}  // namespace jhtb

extern "C" int jhtb_probe_fp64_fma(int blocks_per_sm, int iters, double *sink, double *ms, double *flops,
                                   void *stream) {
    using namespace jhtb;
    if (blocks_per_sm < 1 || iters < 1 || !sink || !ms || !flops) return fail(JHTB_ERR_INVALID, "jhtb_probe_fp64_fma: bad argument");
    int dev = 0, nsm = 148;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    JHTB_CUDA_TRY(cudaEventCreate(&e0));
    JHTB_CUDA_TRY(cudaEventCreate(&e1));
    const int grid = nsm * blocks_per_sm;
    JHTB_CUDA_TRY(cudaEventRecord(e0, s));
    fp64_fma_probe_kernel<<<grid, 256, 0, s>>>(iters, sink);
    JHTB_CUDA_TRY(cudaGetLastError());
    JHTB_CUDA_TRY(cudaEventRecord(e1, s));
    JHTB_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    JHTB_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t;
    *flops = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * (double)grid;
    return JHTB_OK;
}
