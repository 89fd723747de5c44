// 2D NUFFT interpolation and spreading on the oversampled torus grid (sm_100a), the
// point-dependent stages of the off-grid transforms (jht _nufft.py:150-191).
//
// The grid is complex128 [nk][nm] (theta axis k, phi axis m), row-major.  A point
// (theta, phi) touches the W x W window whose first cell is ceil(u - W/2), u = coord *
// n / 2 pi, on each axis (indices taken mod n), with the "exponential of semicircle"
// weights psi(u - idx) = exp(beta (sqrt(1 - (2 t / W)^2) - 1)) on |t| < W / 2
// (Barnett, Magland & af Klinteberg 2019; _nufft.py:69-84).
//
//   interp (type 2):  f_j = sum_ab wk_a wm_b grid[ik_a][im_b], optionally with
//                     d f_j / d theta and d f_j / d phi (the kernel's derivative
//                     weights times n / 2 pi);
//   spread (type 1):  grid[ik_a][im_b] += wk_a wm_b v_j for every point (FP64 atomic
//                     adds: the summation order over points is not fixed).
//
// One thread per point; its 2 W weights stay in registers (W is a template parameter).
// The grid of a typical case (lmax <= 2048: <= 8640^2 cells) is read through L2.
#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kNuThreads = 256;
constexpr double kTwoPi = 6.283185307179586476925286766559;

// Window start and weights (and derivative weights d psi / d u) of one coordinate.
template <int W, bool DERIV>
__device__ __forceinline__ void window(double coord, int n, double beta, long long &first, double (&w)[W],
                                       double (&dw)[W]) {
    const double u = coord * (double)n / kTwoPi;
    const double f = ceil(u - 0.5 * W);
    // far outside any sensible range (or NaN) the start saturates; every index is then
    // still reduced into [0, n) by wrap
    first = (f > -4.0e18 && f < 4.0e18) ? (long long)f : 0;
    const double inv_half = 2.0 / W;
#pragma unroll
    for (int a = 0; a < W; ++a) {
        const double t = u - (f + a);
        const double z = t * inv_half;
        const double z2 = z * z;
        if (z2 < 1.0) {
            const double r = sqrt(1.0 - z2);
            const double v = exp(beta * (r - 1.0));
            w[a] = v;
            if (DERIV) dw[a] = -v * beta * z * inv_half / r;
        } else {
            w[a] = 0.0;
            if (DERIV) dw[a] = 0.0;
        }
    }
}

__device__ __forceinline__ int wrap(long long i, int n) {
    const long long r = i % n;
    return (int)(r < 0 ? r + n : r);
}

template <int W, bool DERIV>
__global__ void __launch_bounds__(kNuThreads) interp_kernel(const double2 *__restrict__ grid, int nk, int nm,
                                                            double beta, const double *__restrict__ theta,
                                                            const double *__restrict__ phi, long long npts,
                                                            double2 *__restrict__ out, double2 *__restrict__ dth,
                                                            double2 *__restrict__ dph) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts;
         j += (long long)gridDim.x * blockDim.x) {
        long long k0, m0;
        double wk[W], wm[W], dk[W], dm[W];
        window<W, DERIV>(theta[j], nk, beta, k0, wk, dk);
        window<W, DERIV>(phi[j], nm, beta, m0, wm, dm);
        int mi[W];
#pragma unroll
        for (int b = 0; b < W; ++b) mi[b] = wrap(m0 + b, nm);
        double2 f = make_double2(0.0, 0.0), gk = make_double2(0.0, 0.0), gm = make_double2(0.0, 0.0);
#pragma unroll 2
        for (int a = 0; a < W; ++a) {
            const double2 *row = grid + (size_t)wrap(k0 + a, nk) * nm;
            double2 s = make_double2(0.0, 0.0), sd = make_double2(0.0, 0.0);
#pragma unroll
            for (int b = 0; b < W; ++b) {
                const double2 g = __ldg(&row[mi[b]]);
                s.x = fma(wm[b], g.x, s.x);
                s.y = fma(wm[b], g.y, s.y);
                if (DERIV) {
                    sd.x = fma(dm[b], g.x, sd.x);
                    sd.y = fma(dm[b], g.y, sd.y);
                }
            }
            f.x = fma(wk[a], s.x, f.x);
            f.y = fma(wk[a], s.y, f.y);
            if (DERIV) {
                gk.x = fma(dk[a], s.x, gk.x);
                gk.y = fma(dk[a], s.y, gk.y);
                gm.x = fma(wk[a], sd.x, gm.x);
                gm.y = fma(wk[a], sd.y, gm.y);
            }
        }
        out[j] = f;
        if (DERIV) {
            // d/dcoord = (n / 2 pi) d/du
            const double ck = (double)nk / kTwoPi, cm = (double)nm / kTwoPi;
            dth[j] = make_double2(ck * gk.x, ck * gk.y);
            dph[j] = make_double2(cm * gm.x, cm * gm.y);
        }
    }
}

template <int W>
__global__ void __launch_bounds__(kNuThreads) spread_kernel(const double2 *__restrict__ vals,
                                                            const double *__restrict__ theta,
                                                            const double *__restrict__ phi, long long npts, int nk,
                                                            int nm, double beta, double2 *__restrict__ grid) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < npts;
         j += (long long)gridDim.x * blockDim.x) {
        long long k0, m0;
        double wk[W], wm[W], unused[W];
        window<W, false>(theta[j], nk, beta, k0, wk, unused);
        window<W, false>(phi[j], nm, beta, m0, wm, unused);
        const double2 v = vals[j];
        int mi[W];
#pragma unroll
        for (int b = 0; b < W; ++b) mi[b] = wrap(m0 + b, nm);
#pragma unroll 1
        for (int a = 0; a < W; ++a) {
            double *row = reinterpret_cast<double *>(grid + (size_t)wrap(k0 + a, nk) * nm);
            const double vx = wk[a] * v.x, vy = wk[a] * v.y;
#pragma unroll
            for (int b = 0; b < W; ++b) {
                atomicAdd(row + 2 * mi[b], wm[b] * vx);
                atomicAdd(row + 2 * mi[b] + 1, wm[b] * vy);
            }
        }
    }
}

// Tiled spread: the points arrive grouped by kTile x kTile-cell tiles of the grid (segments
// of one tile, at most kSegPoints points each).  A CTA adds its segment's windows into a
// shared-memory copy of the tile plus its W-cell halo, then adds that block to the grid once
// per cell, so the global atomics fall from 2 W^2 per point to 2 (kTile + W)^2 per segment.
// A point whose window leaves the block (a coordinate outside the tile its key named) is
// added straight to the grid.
constexpr int kTile = 32;
constexpr int kSpreadThreads = 128;

template <int W>
__global__ void __launch_bounds__(kSpreadThreads) spread_tiles_kernel(
    const double2 *__restrict__ vals, const double *__restrict__ theta, const double *__restrict__ phi,
    long long npts, const long long *__restrict__ seg_start, const int *__restrict__ seg_count,
    const long long *__restrict__ seg_tile, int tiles_m, int nk, int nm, double beta, double2 *__restrict__ grid) {
    constexpr int B = kTile + W;  // block edge: the tile and its halo
    __shared__ double acc[B * B * 2];
    for (int i = threadIdx.x; i < B * B * 2; i += blockDim.x) acc[i] = 0.0;
    __syncthreads();
    const long long seg = blockIdx.x;
    const long long tile = seg_tile[seg];
    const long long k_org = (tile / tiles_m) * kTile - W / 2, m_org = (tile % tiles_m) * kTile - W / 2;
    const long long p0 = seg_start[seg];
    const int cnt = seg_count[seg];
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        const long long j = p0 + q;
        if (j < 0 || j >= npts) continue;
        long long k0, m0;
        double wk[W], wm[W], unused[W];
        window<W, false>(theta[j], nk, beta, k0, wk, unused);
        window<W, false>(phi[j], nm, beta, m0, wm, unused);
        const double2 v = vals[j];
        const long long lk = k0 - k_org, lm = m0 - m_org;
        if (lk >= 0 && lk + W <= B && lm >= 0 && lm + W <= B) {
#pragma unroll 1
            for (int a = 0; a < W; ++a) {
                double *row = acc + 2 * ((lk + a) * B + lm);
                const double vx = wk[a] * v.x, vy = wk[a] * v.y;
#pragma unroll
                for (int b = 0; b < W; ++b) {
                    atomicAdd(row + 2 * b, wm[b] * vx);
                    atomicAdd(row + 2 * b + 1, wm[b] * vy);
                }
            }
        } else {
            int mi[W];
#pragma unroll
            for (int b = 0; b < W; ++b) mi[b] = wrap(m0 + b, nm);
#pragma unroll 1
            for (int a = 0; a < W; ++a) {
                double *row = reinterpret_cast<double *>(grid + (size_t)wrap(k0 + a, nk) * nm);
                const double vx = wk[a] * v.x, vy = wk[a] * v.y;
#pragma unroll
                for (int b = 0; b < W; ++b) {
                    atomicAdd(row + 2 * mi[b], wm[b] * vx);
                    atomicAdd(row + 2 * mi[b] + 1, wm[b] * vy);
                }
            }
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < B * B; c += blockDim.x) {
        const double x = acc[2 * c], y = acc[2 * c + 1];
        if (x == 0.0 && y == 0.0) continue;
        const int a = c / B, b = c - a * B;
        double *cell = reinterpret_cast<double *>(grid + (size_t)wrap(k_org + a, nk) * nm + wrap(m_org + b, nm));
        atomicAdd(cell, x);
        atomicAdd(cell + 1, y);
    }
}

int grid_blocks(long long npts) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long long need = (npts + kNuThreads - 1) / kNuThreads;
    return (int)std::max<long long>(1, std::min<long long>(need, (long long)nsm * 16));
}

int check_args(int nk, int nm, int W, long long npts, const char *who) {
    if (W != 6 && W != 8 && W != 10 && W != 14 && W != 16)
        return fail(JHTB_ERR_UNSUPPORTED, std::string(who) + ": kernel width must be 6, 8, 10, 14 or 16");
    if (nk < 1 || nm < 1) return fail(JHTB_ERR_INVALID, std::string(who) + ": empty grid");
    if (npts < 0) return fail(JHTB_ERR_INVALID, std::string(who) + ": negative point count");
    return JHTB_OK;
}

template <int W>
void launch_interp(const double2 *g, int nk, int nm, double beta, const double *th, const double *ph, long long n,
                   double2 *out, double2 *dth, double2 *dph, cudaStream_t s) {
    if (dth && dph)
        interp_kernel<W, true><<<grid_blocks(n), kNuThreads, 0, s>>>(g, nk, nm, beta, th, ph, n, out, dth, dph);
    else
        interp_kernel<W, false><<<grid_blocks(n), kNuThreads, 0, s>>>(g, nk, nm, beta, th, ph, n, out, nullptr, nullptr);
}

template <int W>
void launch_spread(const double2 *v, const double *th, const double *ph, long long n, int nk, int nm, double beta,
                   double2 *g, cudaStream_t s) {
    spread_kernel<W><<<grid_blocks(n), kNuThreads, 0, s>>>(v, th, ph, n, nk, nm, beta, g);
}

template <int W>
void launch_spread_tiles(const double2 *v, const double *th, const double *ph, long long npts, long long nseg,
                         const long long *start, const int *count, const long long *tile, int tiles_m, int nk, int nm,
                         double beta, double2 *g, cudaStream_t s) {
    spread_tiles_kernel<W><<<(unsigned)nseg, kSpreadThreads, 0, s>>>(v, th, ph, npts, start, count, tile, tiles_m, nk,
                                                                    nm, beta, g);
}

}  // namespace
}  // namespace jhtb

using namespace jhtb;

extern "C" {

int jhtb_nufft_interp(const void *grid, int nk, int nm, int W, double beta, const double *theta, const double *phi,
                      int64_t npts, void *out, void *dtheta, void *dphi, void *stream) {
    if (!grid || !theta || !phi || !out) return fail(JHTB_ERR_INVALID, "jhtb_nufft_interp: NULL argument");
    if ((dtheta == nullptr) != (dphi == nullptr))
        return fail(JHTB_ERR_INVALID, "jhtb_nufft_interp: pass both derivative outputs or neither");
    int rc = check_args(nk, nm, W, npts, "jhtb_nufft_interp");
    if (rc) return rc;
    if (npts == 0) return JHTB_OK;
    const double2 *g = (const double2 *)grid;
    double2 *o = (double2 *)out, *dt = (double2 *)dtheta, *dp = (double2 *)dphi;
    cudaStream_t s = (cudaStream_t)stream;
    switch (W) {
        case 6: launch_interp<6>(g, nk, nm, beta, theta, phi, npts, o, dt, dp, s); break;
        case 8: launch_interp<8>(g, nk, nm, beta, theta, phi, npts, o, dt, dp, s); break;
        case 10: launch_interp<10>(g, nk, nm, beta, theta, phi, npts, o, dt, dp, s); break;
        case 14: launch_interp<14>(g, nk, nm, beta, theta, phi, npts, o, dt, dp, s); break;
        default: launch_interp<16>(g, nk, nm, beta, theta, phi, npts, o, dt, dp, s); break;
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int jhtb_nufft_spread(const void *vals, const double *theta, const double *phi, int64_t npts, int nk, int nm, int W,
                      double beta, void *grid, void *stream) {
    if (!vals || !theta || !phi || !grid) return fail(JHTB_ERR_INVALID, "jhtb_nufft_spread: NULL argument");
    int rc = check_args(nk, nm, W, npts, "jhtb_nufft_spread");
    if (rc) return rc;
    if (npts == 0) return JHTB_OK;
    const double2 *v = (const double2 *)vals;
    double2 *g = (double2 *)grid;
    cudaStream_t s = (cudaStream_t)stream;
    switch (W) {
        case 6: launch_spread<6>(v, theta, phi, npts, nk, nm, beta, g, s); break;
        case 8: launch_spread<8>(v, theta, phi, npts, nk, nm, beta, g, s); break;
        case 10: launch_spread<10>(v, theta, phi, npts, nk, nm, beta, g, s); break;
        case 14: launch_spread<14>(v, theta, phi, npts, nk, nm, beta, g, s); break;
        default: launch_spread<16>(v, theta, phi, npts, nk, nm, beta, g, s); break;
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int jhtb_nufft_spread_tiles(const void *vals, const double *theta, const double *phi, int64_t npts, int64_t nseg,
                            const int64_t *seg_start, const int *seg_count, const int64_t *seg_tile, int tiles_m,
                            int nk, int nm, int W, double beta, void *grid, void *stream) {
    if (!vals || !theta || !phi || !grid || (nseg > 0 && (!seg_start || !seg_count || !seg_tile)))
        return fail(JHTB_ERR_INVALID, "jhtb_nufft_spread_tiles: NULL argument");
    int rc = check_args(nk, nm, W, npts, "jhtb_nufft_spread_tiles");
    if (rc) return rc;
    rc = nseg < 0 ? fail(JHTB_ERR_INVALID, "jhtb_nufft_spread_tiles: negative segment count") : JHTB_OK;
    if (rc) return rc;
    if (tiles_m < 1) return fail(JHTB_ERR_INVALID, "jhtb_nufft_spread_tiles: tiles_m must be >= 1");
    if (nseg > 0x7fffffffLL) return fail(JHTB_ERR_INVALID, "jhtb_nufft_spread_tiles: too many segments");
    if (nseg == 0) return JHTB_OK;
    const double2 *v = (const double2 *)vals;
    double2 *g = (double2 *)grid;
    const long long *st = (const long long *)seg_start, *tl = (const long long *)seg_tile;
    cudaStream_t s = (cudaStream_t)stream;
    switch (W) {
        case 6: launch_spread_tiles<6>(v, theta, phi, npts, nseg, st, seg_count, tl, tiles_m, nk, nm, beta, g, s); break;
        case 8: launch_spread_tiles<8>(v, theta, phi, npts, nseg, st, seg_count, tl, tiles_m, nk, nm, beta, g, s); break;
        case 10: launch_spread_tiles<10>(v, theta, phi, npts, nseg, st, seg_count, tl, tiles_m, nk, nm, beta, g, s); break;
        case 14: launch_spread_tiles<14>(v, theta, phi, npts, nseg, st, seg_count, tl, tiles_m, nk, nm, beta, g, s); break;
        default: launch_spread_tiles<16>(v, theta, phi, npts, nseg, st, seg_count, tl, tiles_m, nk, nm, beta, g, s); break;
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // extern "C"
