// jhtb_synthesis_noalloc: spin-0 FP64 synthesis that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code running where the CUDA
// allocator is off limits (inside another framework's memory pool, a plugin host
// that owns all device allocations, or a process that has reserved the device's
// memory up front) -- but still want S: alm -> map for small geometries without
// creating a plan, which allocates its tables and workspace.
//
// How: the only scratch the transform needs, the ring spectra F[ring][m] between the
// recursion/contraction kernel and the ring-DFT kernel, lives in one file-scope
// __device__ array of fixed size (kNoallocScratchBytes, 2 MiB).  Every other table
// (recursion coefficients, seeds, geometry, DFT roots of unity) is computed inside
// the kernels.  Sizes whose ring spectra do not fit, or nside > 64, are rejected.
//
// Sharing: all calls on a device use the same array and it keeps the last call's
// contents.  Both kernels overwrite every element they read, so nothing has to be
// cleared between calls, but calls whose kernels overlap on the GPU (different
// streams without ordering, or several host threads) race on it: order them.
//
// Set-up: the first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it together with the id
// of the CUDA context it belongs to; make that first call before any stream capture
// begins.  When the context changes (cudaDeviceReset destroys the primary context and
// a later runtime call creates a new one, in which the array may sit elsewhere), the
// next call sees a different context id and looks the address up again.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <mutex>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr size_t kNoallocScratchBytes = 2u << 20;  // 2 MiB = 131072 complex doubles
constexpr int kNoallocMaxNside = 64;
constexpr int kNoallocMaxLmax = 1023;
constexpr int kNoallocThreads = 128;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double2 g_noalloc_scratch[kNoallocScratchBytes / sizeof(double2)];

// Per device: the array's address and the id of the context it was looked up in.
struct ScratchSlot {
    std::mutex mu;
    double2 *ptr = nullptr;
    unsigned long long ctx = 0;
};
ScratchSlot g_slot[kMaxDevices];

// Id of the calling thread's current CUDA context (0 if none or if the driver lacks the
// query), through the driver entry points the runtime hands out (no link-time libcuda).
unsigned long long current_context_id() {
    typedef int (*GetCurrentFn)(void **);
    typedef int (*GetIdFn)(void *, unsigned long long *);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **)&get_current, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **)&get_id, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    });
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// z = cos(theta) of half-grid ring t (0-based), as RING geometry defines it.
__device__ double ring_z(int t, int nside) {
    const long long i = t + 1;
    if (i < nside) return 1.0 - (double)(i * i) / (3.0 * (double)nside * (double)nside);
    return 4.0 / 3.0 - (2.0 * (double)i) / (3.0 * (double)nside);
}

__device__ long long ring_len(int r, int nside) {
    const long long i = r + 1;
    if (i < nside) return 4 * i;
    if (i > 3LL * nside) return 4 * (4LL * nside - i);
    return 4LL * nside;
}

__device__ long long ring_start(int r, int nside) {
    const long long i = r + 1;
    if (i < nside) return 2 * i * (i - 1);
    const long long ncap = 2LL * nside * (nside - 1);
    if (i <= 3LL * nside) return ncap + (i - nside) * 4LL * nside;
    const long long j = 4LL * nside - i;  // mirrored cap ring
    return 12LL * nside * nside - 2 * j * (j + 1);
}

// phi0 of ring r as pi * p / q with p in {0, 1}: returns q, and p through *p.
__device__ long long ring_phi0_den(int r, int nside, int *p) {
    const long long i = r + 1;
    *p = 1;
    if (i < nside) return 4 * i;
    if (i > 3LL * nside) return 4 * (4LL * nside - i);
    *p = ((i - nside) % 2 == 0) ? 1 : 0;
    return 4LL * nside;
}

// e^{i m phi0} with the angle reduced exactly: m phi0 / pi = (p m mod 2q) / q.
__device__ void ring_phase(long long m, int p, long long q, double *s, double *c) {
    sincospi((double)((p * m) % (2 * q)) / (double)q, s, c);
}

// One CTA per order m: normalised three-term recursion with scaled seeds
// (value = mu 2^(800 sc)), coefficients built in shared memory by the CTA.
__global__ void __launch_bounds__(kNoallocThreads) noalloc_legendre_kernel(int nside, int lmax,
                                                                          const double2 *__restrict__ alm,
                                                                          double2 *__restrict__ F) {
    __shared__ double s_alpha[kNoallocMaxLmax + 1];
    __shared__ double2 s_a[kNoallocMaxLmax + 1];
    __shared__ double s_logc;
    const int m = blockIdx.x;
    const int M = lmax + 1;
    const long long base = (long long)m * (2 * lmax + 1 - m) / 2;  // index of a_{0,m} shifted: a_{l,m} at base + l
    if (threadIdx.x == 0) {
        // g_l = b_l g_{l-2} (g_m = g_{m+1} = 1); alpha_l = a_l g_{l-1} / g_l; a~_l = a_lm g_l
        double g2 = 1.0, g1 = 1.0;
        s_alpha[m] = 0.0;
        s_a[m] = alm[base + m];
        for (int l = m + 1; l <= lmax; ++l) {
            const double dl = l;
            const double a = sqrt((2 * dl - 1) * (2 * dl + 1) / ((dl - m) * (dl + m)));
            const double b = sqrt((2 * dl + 1) * ((dl - 1) * (dl - 1) - (double)m * m) / ((2 * dl - 3) * (dl - m) * (dl + m)));
            const double g = (l == m + 1) ? 1.0 : b * g2;
            s_alpha[l] = a * g1 / g;
            const double2 c = alm[base + l];
            s_a[l] = make_double2(c.x * g, c.y * g);
            g2 = g1;
            g1 = g;
        }
        double lc = -0.5 * log(4.0 * M_PI);
        for (int k = 1; k <= m; ++k) lc += 0.5 * log((2.0 * k + 1.0) / (2.0 * k));
        s_logc = lc;
    }
    __syncthreads();
    const int T = 2 * nside;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const double x = ring_z(t, nside);
        const double s2 = fmin(fmax(1.0 - x * x, 0.0), 1.0);
        double lg = (m == 0) ? s_logc : s_logc + (double)m * log(sqrt(s2));
        int sc = 0;
        double mant = 0.0;
        if (lg > -1.0e300) {
            int k = (int)floor((lg + kLn2x400) / (kLogScaleHi + kLogScaleLo));
            if (k > 0) k = 0;
            const double r = (lg - (double)k * kLogScaleHi) - (double)k * kLogScaleLo;
            mant = ((m & 1) ? -1.0 : 1.0) * exp(r);
            sc = k;
        }
        double u1 = mant, u2 = 0.0;
        double2 E = make_double2(0.0, 0.0), O = make_double2(0.0, 0.0);
        for (int l = m; l <= lmax; ++l) {
            double u;
            if (l == m) {
                u = u1;
            } else {
                u = fma(s_alpha[l] * x, u1, -u2);
                double prev = u1;
                if (sc < 0 && fabs(u) > kBig) {
                    u *= kScaleDown;
                    prev *= kScaleDown;
                    sc += 1;
                }
                u2 = prev;
                u1 = u;
            }
            if (sc == 0) {
                double2 &acc = (l & 1) ? O : E;
                acc.x = fma(s_a[l].x, u, acc.x);
                acc.y = fma(s_a[l].y, u, acc.y);
            }
        }
        F[(size_t)t * M + m] = make_double2(E.x + O.x, E.y + O.y);
        if (t < T - 1) {
            const double sg = (m & 1) ? -1.0 : 1.0;  // south: (-1)^m (E - O)
            F[(size_t)(4 * nside - 2 - t) * M + m] = make_double2(sg * (E.x - O.x), sg * (E.y - O.y));
        }
    }
}

// One CTA per ring: phase, m -> k fold (gather), direct length-N DFT (N <= 256), real part.
__global__ void __launch_bounds__(kNoallocThreads) noalloc_ring_kernel(int nside, int lmax,
                                                                      const double2 *__restrict__ F,
                                                                      double *__restrict__ map) {
    __shared__ double2 s_D[4 * kNoallocMaxNside];
    const int r = blockIdx.x;
    const int N = (int)ring_len(r, nside);
    int pn = 0;
    const long long qd = ring_phi0_den(r, nside, &pn);
    const double2 *row = F + (size_t)r * (lmax + 1);
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        double2 d = make_double2(0.0, 0.0);
        for (int m = k; m <= lmax; m += N) {
            double s, c;
            ring_phase(m, pn, qd, &s, &c);
            const double2 f = row[m];
            d.x += f.x * c - f.y * s;
            d.y += f.x * s + f.y * c;
        }
        int m0 = (N - k) % N;
        if (m0 == 0) m0 = N;
        for (int m = m0; m <= lmax; m += N) {
            double s, c;
            ring_phase(m, pn, qd, &s, &c);
            const double2 f = row[m];
            d.x += f.x * c - f.y * s;
            d.y -= f.x * s + f.y * c;
        }
        s_D[k] = d;
    }
    __syncthreads();
    double *out = map + ring_start(r, nside);
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < N; ++k) {
            double s, c;
            sincospi(2.0 * (double)(((long long)j * k) % N) / (double)N, &s, &c);
            acc += s_D[k].x * c - s_D[k].y * s;  // Re(D[k] e^{+2 pi i jk/N})
        }
        out[j] = acc;
    }
}

}  // namespace
}  // namespace jhtb

using namespace jhtb;

extern "C" int jhtb_synthesis_noalloc(int nside, int lmax, const void *alm, void *map, void *stream) {
    if (!alm || !map) return fail(JHTB_ERR_INVALID, "jhtb_synthesis_noalloc: NULL argument");
    if (nside < 1 || nside > kNoallocMaxNside)
        return fail(JHTB_ERR_INVALID, "jhtb_synthesis_noalloc: nside must be in [1, 64], got " + std::to_string(nside));
    if (lmax < 0 || lmax > kNoallocMaxLmax)
        return fail(JHTB_ERR_INVALID, "jhtb_synthesis_noalloc: lmax must be in [0, 1023], got " + std::to_string(lmax));
    const size_t need = sizeof(double2) * (size_t)(4 * nside - 1) * (size_t)(lmax + 1);
    if (need > kNoallocScratchBytes)
        return fail(JHTB_ERR_INVALID, "jhtb_synthesis_noalloc: (4 nside - 1)(lmax + 1) ring spectra need " +
                                          std::to_string(need) + " bytes, above the fixed 2 MiB scratch");
    int dev = 0;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(JHTB_ERR_UNSUPPORTED, "jhtb_synthesis_noalloc: device index too large");
    double2 *scratch = nullptr;
    {
        ScratchSlot &slot = g_slot[dev];
        std::lock_guard<std::mutex> lock(slot.mu);
        const unsigned long long ctx = current_context_id();
        if (!slot.ptr || ctx == 0 || ctx != slot.ctx) {
            // set-up on this device and context (the device is current): the array's device
            // address; the lookup also creates the primary context if there is none yet
            JHTB_CUDA_TRY(cudaGetSymbolAddress((void **)&slot.ptr, g_noalloc_scratch));
            slot.ctx = current_context_id();
        }
        scratch = slot.ptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    noalloc_legendre_kernel<<<lmax + 1, kNoallocThreads, 0, s>>>(nside, lmax, (const double2 *)alm, scratch);
    JHTB_CUDA_TRY(cudaGetLastError());
    noalloc_ring_kernel<<<4 * nside - 1, kNoallocThreads, 0, s>>>(nside, lmax, scratch, (double *)map);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}
