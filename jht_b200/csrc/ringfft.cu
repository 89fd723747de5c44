// Azimuthal stage: per-ring phase shift, m -> k fold and length-N DFT (sm_100a).
//
// jht (healpix.py:280-355) groups rings by length and emits one FFT per distinct
// length, with scatter-adds for the m -> k fold.  Here one CTA owns one ring:
//   synthesis  D[k] = sum_{m = k mod N} Fp_m e^{i m phi0} + sum_{m>=1, -m = k mod N} conj(Fm_m e^{i m phi0})
//              out[j] = sum_k D[k] e^{+2 pi i jk/N}      (real part: spin 0; Q + iU: spin 2)
//   adjoint    W[k] = sum_j v[j] e^{-2 pi i jk/N};  V[m] = W[m mod N] e^{-i m phi0}
//              (spin 2 also Vm[m] = conj(W[-m mod N]) e^{-i m phi0})
// The fold is a gather (each k collects its own m's), never a scatter.  Power-of-two
// rings up to 8192 use a radix-2 FFT in shared memory; every other length uses
// Bluestein's chirp-z with an exact (n^2 mod 2N) chirp argument (_azimuth.py:150-191)
// at a power-of-two length P >= 2N-1, split into Q = P/8192 shared-memory pieces when
// P > 8192 (decimation in frequency on the input, twiddled recombination on the output).
#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kFftThreads = 512;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conjd(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ int ilog2i(int n) { return 31 - __clz(n); }
__device__ __forceinline__ int brev(int k, int logn) { return logn ? (int)(__brev((unsigned)k) >> (32 - logn)) : 0; }

// e^{i * sgn * pi * (n^2 mod 2N) / N}: the exact chirp-z argument reduction.
__device__ __forceinline__ double2 chirp(long long n, int N, double sgn) {
    const long long r = (n * n) % (2LL * N);
    double s, c;
    sincospi(sgn * (double)r / (double)N, &s, &c);
    return make_double2(c, s);
}

// e^{i * sgn * 2 pi a / b} for integers, via sincospi with an exact rational argument.
__device__ __forceinline__ double2 root(long long a, long long b, double sgn) {
    const long long r = a % b;
    double s, c;
    sincospi(sgn * 2.0 * (double)r / (double)b, &s, &c);
    return make_double2(c, s);
}

// In-place radix-2 DIT FFT of length n (power of two <= kFftMax) on shared memory.
// Input in bit-reversed order, output natural.  dir = -1: e^{-2 pi i jk/n}; +1: e^{+...}.
__device__ void fft_smem(double2 *buf, int n, int dir, const double2 *__restrict__ tw) {
    const int logn = ilog2i(n);
    for (int s = 1; s <= logn; ++s) {
        const int half = 1 << (s - 1);
        const int shift = kFftLogMax - s;
        for (int bf = threadIdx.x; bf < (n >> 1); bf += blockDim.x) {
            const int k = bf & (half - 1);
            const int i0 = ((bf >> (s - 1)) << s) + k;
            const int i1 = i0 + half;
            double2 w = __ldg(&tw[k << shift]);
            if (dir > 0) w.y = -w.y;
            const double2 a = buf[i0];
            const double2 t = cmul(buf[i1], w);
            buf[i0] = cadd(a, t);
            buf[i1] = csub(a, t);
        }
        __syncthreads();
    }
}

// In-place radix-2 DIF FFT: input natural order, output bit-reversed.
__device__ void fft_smem_dif(double2 *buf, int n, int dir, const double2 *__restrict__ tw) {
    const int logn = ilog2i(n);
    for (int s = logn; s >= 1; --s) {
        const int half = 1 << (s - 1);
        const int shift = kFftLogMax - s;
        for (int bf = threadIdx.x; bf < (n >> 1); bf += blockDim.x) {
            const int k = bf & (half - 1);
            const int i0 = ((bf >> (s - 1)) << s) + k;
            const int i1 = i0 + half;
            double2 w = __ldg(&tw[k << shift]);
            if (dir > 0) w.y = -w.y;
            const double2 a = buf[i0], b = buf[i1];
            buf[i0] = cadd(a, b);
            buf[i1] = cmul(csub(a, b), w);
        }
        __syncthreads();
    }
}

// Bluestein spectrum for the synthesis direction: Bh+ = FFT_P(b)/P with
// b[n] = conj(w(n)) on |n| < N, w(n) = e^{+i pi n^2 / N}.  The adjoint direction
// uses Bh-[k] = conj(Bh+[(P - k) mod P]).
__device__ __forceinline__ double2 bh_get(const double2 *bh, int P, int k, int sgn) {
    if (sgn > 0) return __ldg(&bh[k]);
    return conjd(__ldg(&bh[(P - k) & (P - 1)]));
}

// D[k] of the synthesis fold for one ring (spin 0 passes Fm == Fp).
__device__ __forceinline__ double2 fold_synth(const double2 *__restrict__ Fp, const double2 *__restrict__ Fm,
                                              int k, int N, int lmax, double phi0) {
    double2 d = make_double2(0.0, 0.0);
    for (int m = k; m <= lmax; m += N) {
        double s, c;
        sincos((double)m * phi0, &s, &c);
        d = cadd(d, cmul(Fp[m], make_double2(c, s)));
    }
    int m0 = (N - k) % N;
    if (m0 == 0) m0 = N;
    for (int m = m0; m <= lmax; m += N) {
        double s, c;
        sincos((double)m * phi0, &s, &c);
        d = cadd(d, conjd(cmul(Fm[m], make_double2(c, s))));
    }
    return d;
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads) ring_synth_kernel(const RingDesc *__restrict__ rings, int lmax,
                                                                  int M, int nrings, long long npix,
                                                                  const double2 *__restrict__ F_all,
                                                                  double *__restrict__ maps_all,
                                                                  const double2 *__restrict__ tw,
                                                                  const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    const int r = blockIdx.x;
    const RingDesc rd = rings[r];
    const int N = rd.N;
    constexpr int nchan = SPIN ? 2 : 1;
    const double2 *Fp = F_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    const double2 *Fm = SPIN ? Fp + (size_t)nrings * M : Fp;
    double *outQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    double *outU = outQ + npix;
    if (rd.mode == kDirect) {
        const int logn = ilog2i(N);
        for (int k = threadIdx.x; k < N; k += blockDim.x) buf[brev(k, logn)] = fold_synth(Fp, Fm, k, N, lmax, rd.phi0);
        __syncthreads();
        fft_smem(buf, N, +1, tw);
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            outQ[j] = buf[j].x;
            if (SPIN) outU[j] = buf[j].y;
        }
        return;
    }
    const int P = rd.P, Q = rd.Q, Pp = P / Q, logp = ilog2i(Pp);
    const double2 *B = bh + rd.bh_off;
    for (int s = 0; s < Q; ++s) {
        // piece s of FFT_P(a), a[k] = D[k] w(k): fold a[k] e^{-2 pi i s k / P} modulo Pp
        for (int q = threadIdx.x; q < Pp; q += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int k = q; k < N; k += Pp) {
                double2 a = cmul(fold_synth(Fp, Fm, k, N, lmax, rd.phi0), chirp(k, N, 1.0));
                if (s) a = cmul(a, root((long long)s * k, P, -1.0));
                v = cadd(v, a);
            }
            buf[brev(q, logp)] = v;
        }
        __syncthreads();
        fft_smem(buf, Pp, -1, tw);
        for (int q = threadIdx.x; q < Pp; q += blockDim.x) buf[q] = cmul(buf[q], bh_get(B, P, Q * q + s, 1));
        __syncthreads();
        fft_smem_dif(buf, Pp, +1, tw);  // output in bit-reversed order
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            double2 v = buf[brev(j & (Pp - 1), logp)];
            if (s) v = cmul(v, root((long long)s * j, P, 1.0));
            v = cmul(v, chirp(j, N, 1.0));
            if (s == 0) {
                outQ[j] = v.x;
                if (SPIN) outU[j] = v.y;
            } else {
                outQ[j] += v.x;
                if (SPIN) outU[j] += v.y;
            }
        }
        __syncthreads();
    }
}

// V rows for ring r from its spectrum W (smem or global).
template <int SPIN>
__device__ __forceinline__ void gather_adjoint(const double2 *W, int N, int lmax, double phi0, double2 *Vp,
                                               double2 *Vm) {
    for (int m = threadIdx.x; m <= lmax; m += blockDim.x) {
        double s, c;
        sincos((double)m * phi0, &s, &c);
        const double2 cph = make_double2(c, -s);
        Vp[m] = cmul(W[m % N], cph);
        if (SPIN) Vm[m] = cmul(conjd(W[(N - m % N) % N]), cph);
    }
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads) ring_adjoint_kernel(const RingDesc *__restrict__ rings, int lmax,
                                                                    int M, int nrings, long long npix,
                                                                    const double *__restrict__ maps_all,
                                                                    double2 *__restrict__ V_all,
                                                                    double2 *__restrict__ W_all,
                                                                    const double2 *__restrict__ tw,
                                                                    const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    const int r = blockIdx.x;
    const RingDesc rd = rings[r];
    const int N = rd.N;
    constexpr int nchan = SPIN ? 2 : 1;
    const double *inQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    const double *inU = inQ + npix;
    double2 *Vp = V_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    double2 *Vm = SPIN ? Vp + (size_t)nrings * M : Vp;
    if (rd.mode == kDirect) {
        const int logn = ilog2i(N);
        for (int j = threadIdx.x; j < N; j += blockDim.x)
            buf[brev(j, logn)] = make_double2(inQ[j], SPIN ? inU[j] : 0.0);
        __syncthreads();
        fft_smem(buf, N, -1, tw);
        gather_adjoint<SPIN>(buf, N, lmax, rd.phi0, Vp, Vm);
        return;
    }
    const int P = rd.P, Q = rd.Q, Pp = P / Q, logp = ilog2i(Pp);
    const double2 *B = bh + rd.bh_off;
    double2 *Wg = W_all + (size_t)blockIdx.y * npix + rd.start;
    for (int s = 0; s < Q; ++s) {
        for (int q = threadIdx.x; q < Pp; q += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int j = q; j < N; j += Pp) {
                double2 a = cmul(make_double2(inQ[j], SPIN ? inU[j] : 0.0), chirp(j, N, -1.0));
                if (s) a = cmul(a, root((long long)s * j, P, -1.0));
                v = cadd(v, a);
            }
            buf[brev(q, logp)] = v;
        }
        __syncthreads();
        fft_smem(buf, Pp, -1, tw);
        for (int q = threadIdx.x; q < Pp; q += blockDim.x) buf[q] = cmul(buf[q], bh_get(B, P, Q * q + s, -1));
        __syncthreads();
        fft_smem_dif(buf, Pp, +1, tw);  // output in bit-reversed order
        // W[k] = w'(k) conv[k], accumulated over the pieces in the ring's slot of the scratch
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            double2 v = buf[brev(k & (Pp - 1), logp)];
            if (s) v = cmul(v, root((long long)s * k, P, 1.0));
            v = cmul(v, chirp(k, N, -1.0));
            Wg[k] = s ? cadd(Wg[k], v) : v;
        }
        __syncthreads();
    }
    __threadfence_block();
    gather_adjoint<SPIN>(Wg, N, lmax, rd.phi0, Vp, Vm);
}

// One block per (Bluestein length, piece): Bh+[Q q + s] = (1/P) sum_n b[n] e^{-2 pi i (Qq+s) n / P}.
__global__ void __launch_bounds__(kFftThreads) bluestein_setup_kernel(const int *__restrict__ lens,
                                                                       const long long *__restrict__ offs,
                                                                       const double2 *__restrict__ tw,
                                                                       double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    const int N = lens[blockIdx.x];
    int P = 1;
    while (P < 2 * N - 1) P <<= 1;
    const int Q = P > kFftMax ? P / kFftMax : 1;
    const int s = blockIdx.y;
    if (s >= Q) return;
    const int Pp = P / Q, logp = ilog2i(Pp);
    double2 *out = bh + offs[blockIdx.x];
    for (int q = threadIdx.x; q < Pp; q += blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        for (int idx = q; idx < P; idx += Pp) {
            // circular kernel: b[idx] = conj(w(n)) with n = idx (idx < N) or idx - P (idx > P - N)
            long long n;
            if (idx < N) n = idx;
            else if (idx > P - N) n = (long long)P - idx;  // w(-n) = w(n)
            else continue;
            double2 b = conjd(chirp(n, N, 1.0));
            if (s) b = cmul(b, root((long long)s * idx, P, -1.0));
            v = cadd(v, b);
        }
        buf[brev(q, logp)] = v;
    }
    __syncthreads();
    fft_smem(buf, Pp, -1, tw);
    const double inv = 1.0 / (double)P;
    for (int q = threadIdx.x; q < Pp; q += blockDim.x)
        out[(long long)Q * q + s] = make_double2(buf[q].x * inv, buf[q].y * inv);
}

int smem_bytes() { return kFftMax * (int)sizeof(double2); }

template <typename K>
int ensure_smem(K kernel) {
    JHTB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes()));
    return JHTB_OK;
}

}  // namespace

int launch_ring_synth(const Plan &p, const double2 *F, double *maps, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.nrings, nb);
    int rc;
    if (p.spin == 0) {
        if ((rc = ensure_smem(ring_synth_kernel<0>))) return rc;
        ring_synth_kernel<0><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_rings, p.lmax, p.M, p.nrings, p.npix, F,
                                                                     maps, p.d_tw, p.d_bh);
    } else {
        if ((rc = ensure_smem(ring_synth_kernel<2>))) return rc;
        ring_synth_kernel<2><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_rings, p.lmax, p.M, p.nrings, p.npix, F,
                                                                     maps, p.d_tw, p.d_bh);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_ring_adjoint(const Plan &p, const double *maps, double2 *V, double2 *W, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.nrings, nb);
    int rc;
    if (p.spin == 0) {
        if ((rc = ensure_smem(ring_adjoint_kernel<0>))) return rc;
        ring_adjoint_kernel<0><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_rings, p.lmax, p.M, p.nrings, p.npix,
                                                                       maps, V, W, p.d_tw, p.d_bh);
    } else {
        if ((rc = ensure_smem(ring_adjoint_kernel<2>))) return rc;
        ring_adjoint_kernel<2><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_rings, p.lmax, p.M, p.nrings, p.npix,
                                                                       maps, V, W, p.d_tw, p.d_bh);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_bluestein_setup(const Plan &p, const int *lengths, const long long *offs, int nlen, cudaStream_t s) {
    if (nlen <= 0) return JHTB_OK;
    int rc;
    if ((rc = ensure_smem(bluestein_setup_kernel))) return rc;
    dim3 grid(nlen, 4);
    bluestein_setup_kernel<<<grid, kFftThreads, smem_bytes(), s>>>(lengths, offs, p.d_tw, p.d_bh);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // namespace jhtb
