// Azimuthal stage: per-ring phase shift, m -> k fold and length-N DFT (sm_100a).
//
// jht (healpix.py:280-355) groups rings by length and emits one FFT per distinct
// length, with scatter-adds for the m -> k fold.  Here one CTA owns one ring:
//   synthesis  D[k] = sum_{m = k mod N} Fp_m e^{i m phi0} + sum_{m>=1, -m = k mod N} conj(Fm_m e^{i m phi0})
//              out[j] = sum_k D[k] e^{+2 pi i jk/N}      (real part: spin 0; Q + iU: spin 2)
//   adjoint    W[k] = sum_j v[j] e^{-2 pi i jk/N};  V[m] = W[m mod N] e^{-i m phi0}
//              (spin 2 also Vm[m] = conj(W[-m mod N]) e^{-i m phi0})
// The fold is a gather (each k collects its own m's), never a scatter.  Power-of-two
// rings use an in-place Stockham FFT in shared memory (radix-16 passes held in
// registers, natural order in and out, a padded layout against bank conflicts), in
// Q = N / 4096 pieces by output residue when N > 4096 (the 4 nside belt rings at
// nside >= 2048), so a CTA needs 70 KB of shared memory and two fit on an SM; every
// other length uses
// Bluestein's chirp-z with an exact (n^2 mod 2N) chirp argument (_azimuth.py:150-191)
// at a power-of-two length P >= 2N-1, split into Q = P/4096 shared-memory pieces when
// P > 4096 (decimation in frequency on the input, twiddled recombination on the output).
#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

#ifndef JHTB_FFT_THREADS
#define JHTB_FFT_THREADS 256
#endif
#ifndef JHTB_FFT_MINB
#define JHTB_FFT_MINB 2
#endif
constexpr int kFftThreads = JHTB_FFT_THREADS;  // threads per ring CTA
constexpr int kFftMinBlocks = JHTB_FFT_MINB;   // resident ring CTAs per SM (4096-point buffers)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 conjd(double2 a) { return make_double2(a.x, -a.y); }

__device__ __forceinline__ int ilog2i(int n) { return 31 - __clz(n); }

// e^{i pi (a / N + 2 c / P)} for integers a, c and P a power of two: a is reduced
// exactly modulo 2N and c modulo P before the one rounding of the argument.  Every
// phase of the azimuthal stage is of this form: on the HEALPix grid phi0 is 0 or
// pi / N (healpix.py:107-140), so e^{i m phi0} = e^{i pi m / N}; the chirp-z factors are
// e^{+-i pi n^2 / N} (_azimuth.py:150-191) and the split-length twiddles e^{+-2 pi i s k / P}.
__device__ __forceinline__ double2 cis_pi(int a, int N, int c, int P) {
    const int n2 = 2 * N;
    int r = a % n2;
    if (r < 0) r += n2;
    int q = c % P;
    if (q < 0) q += P;
    double s, co;
    sincospi((double)r / (double)N + 2.0 * (double)q / (double)P, &s, &co);
    return make_double2(co, s);
}

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

// e^{-+2 pi i a / L} from the twiddle table (e^{-2 pi i j / kTwLen}), L a power of two
// dividing kTwLen; `plus` selects the + sign.
__device__ __forceinline__ double2 twid(const double2 *__restrict__ tw, int a, int L, bool plus) {
    int r = a & (L - 1);
    double2 w = __ldg(&tw[r * (kTwLen / L)]);
    if (plus) w.y = -w.y;
    return w;
}

// Shared-memory layout of an FFT buffer: one pad slot every 16 and every 256 elements,
// so the strided accesses of the Stockham passes spread over the banks.
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4) + (i >> 8); }
constexpr int kFftBufLen = kFftPiece + kFftPiece / 16 + kFftPiece / 256;

// cos and sin of k pi / 8, k < 8 (the 16th roots of unity)
__host__ __device__ constexpr double cos16(int k) {
    return k == 0 ? 1.0 : k == 1 ? 0.9238795325112867 : k == 2 ? 0.7071067811865476 : k == 3 ? 0.3826834323650898
         : k == 4 ? 0.0 : k == 5 ? -0.3826834323650898 : k == 6 ? -0.7071067811865476 : -0.9238795325112867;
}
__host__ __device__ constexpr double sin16(int k) { return cos16(k <= 4 ? 4 - k : k - 4); }
__host__ __device__ constexpr int brev_ct(int i, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2_ct(int n) { return n <= 1 ? 0 : 1 + ilog2_ct(n / 2); }

// R-point DFT in registers (R <= 16), natural order in and out: radix-2 DIT after a
// bit-reversal permutation, all indices and roots fixed at compile time.
// dir = -1: e^{-2 pi i jk/R}; +1: e^{+...}.
template <int R, int LEN, int I, int K>
__device__ __forceinline__ void rf_bfly(double2 (&v)[R], double dir) {
    constexpr int h = LEN / 2, ROOT = K * (16 / LEN);  // e^{dir 2 pi i ROOT / 16}
    const double2 a = v[I + K];
    double2 b = v[I + K + h];
    if constexpr (ROOT == 4) b = make_double2(-dir * b.y, dir * b.x);
    else if constexpr (ROOT != 0) b = cmul(b, make_double2(cos16(ROOT), dir * sin16(ROOT)));
    v[I + K] = cadd(a, b);
    v[I + K + h] = csub(a, b);
}
template <int R, int LEN, int IDX>
__device__ __forceinline__ void rf_stage(double2 (&v)[R], double dir) {
    if constexpr (IDX < R / 2) {
        constexpr int h = LEN / 2;
        rf_bfly<R, LEN, (IDX / h) * LEN, IDX % h>(v, dir);
        rf_stage<R, LEN, IDX + 1>(v, dir);
    }
}
template <int R, int LEN>
__device__ __forceinline__ void rf_stages(double2 (&v)[R], double dir) {
    if constexpr (LEN <= R) {
        rf_stage<R, LEN, 0>(v, dir);
        rf_stages<R, LEN * 2>(v, dir);
    }
}
template <int R, int I>
__device__ __forceinline__ void rf_bitrev(double2 (&v)[R]) {
    if constexpr (I < R) {
        constexpr int J = brev_ct(I, ilog2_ct(R));
        if constexpr (J > I) {
            const double2 t = v[I];
            v[I] = v[J];
            v[J] = t;
        }
        rf_bitrev<R, I + 1>(v);
    }
}
template <int R>
__device__ __forceinline__ void reg_fft(double2 (&v)[R], double dir) {
    rf_bitrev<R, 0>(v);
    rf_stages<R, 2>(v, dir);
}

// One in-place Stockham pass of radix R over n points (Ns = product of the earlier
// radices): every thread loads its R inputs (stride n/R), twiddles them by
// e^{dir 2 pi i (j mod Ns) r / (Ns R)}, runs an R-point DFT in registers and, after a
// barrier, stores them at (j / Ns) Ns R + (j mod Ns) + r Ns.  n <= kFftPiece = 4096
// and kFftThreads threads: each thread holds at most kFftPiece / kFftThreads points.
template <int R>
__device__ __forceinline__ void stockham_pass(double2 *buf, int n, int Ns, double dir,
                                              const double2 *__restrict__ tw) {
    constexpr int JM = kFftPiece / (R * kFftThreads);
    const int nj = n / R;
    double2 v[JM][R];
#pragma unroll
    for (int jj = 0; jj < JM; ++jj) {
        const int j = threadIdx.x + jj * kFftThreads;
        if (j < nj) {
            const int jm = j & (Ns - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) v[jj][r] = buf[pidx(j + r * nj)];
            if (Ns > 1) {
                const int step = jm * (kTwLen / (Ns * R));
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    double2 w = __ldg(&tw[step * r]);
                    if (dir > 0) w.y = -w.y;
                    v[jj][r] = cmul(v[jj][r], w);
                }
            }
            reg_fft<R>(v[jj], dir);
        }
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < JM; ++jj) {
        const int j = threadIdx.x + jj * kFftThreads;
        if (j < nj) {
            const int jm = j & (Ns - 1);
            const int d = (j - jm) * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[pidx(d + r * Ns)] = v[jj][r];
        }
    }
    __syncthreads();
}

// One pass as a separate function: each radix is compiled once, with its own registers.
template <int R>
__device__ __noinline__ void stockham_pass_call(double2 *buf, int n, int Ns, double dir,
                                                const double2 *__restrict__ tw) {
    stockham_pass<R>(buf, n, Ns, dir, tw);
}

// In-place FFT of length n (power of two <= kFftPiece) on a padded shared-memory buffer,
// natural order in and out.  dir = -1: e^{-2 pi i jk/n}; +1: e^{+2 pi i jk/n}.
// Passes of radix 16 with one smaller radix for the remaining bits.
__device__ __forceinline__ void fft_stockham(double2 *buf, int n, double dir, const double2 *__restrict__ tw) {
    int bits = ilog2i(n), Ns = 1;
    for (; bits >= 4; bits -= 4, Ns <<= 4) stockham_pass_call<16>(buf, n, Ns, dir, tw);
    if (bits == 3) stockham_pass_call<8>(buf, n, Ns, dir, tw);
    else if (bits == 2) stockham_pass_call<4>(buf, n, Ns, dir, tw);
    else if (bits == 1) stockham_pass_call<2>(buf, n, Ns, dir, tw);
}

// Bluestein spectrum for the synthesis direction: Bh+ = FFT_P(b)/P with
// b[n] = conj(w(n)) on |n| < N, w(n) = e^{+i pi n^2 / N}.  The adjoint direction
// uses Bh-[k] = conj(Bh+[(P - k) mod P]).
__device__ __forceinline__ double2 bh_get(const double2 *bh, int P, int k, int sgn) {
    if (sgn > 0) return __ldg(&bh[k]);
    return conjd(__ldg(&bh[(P - k) & (P - 1)]));
}

// D[k] of the synthesis fold for one ring, without its phase (spin 0 passes Fm == Fp):
// with m = k + jN in the first sum and m = jN - k in the second,
// e^{i m phi0} = (-1)^j e^{+-i pi k / N} when phi0 = pi / N, so
// D[k] = e^{i pi k / N} [sum_j (-1)^j Fp_{k+jN} + sum_j (-1)^j conj(Fm_{jN-k})];
// `shifted` selects the (-1)^j signs, the caller applies e^{i pi k / N}.
__device__ __forceinline__ double2 fold_synth(const double2 *__restrict__ Fp, const double2 *__restrict__ Fm,
                                              int k, int N, int lmax, bool shifted) {
    double2 d = make_double2(0.0, 0.0);
    double sg = 1.0;
    for (int m = k; m <= lmax; m += N) {
        const double2 f = Fp[m];
        d.x = fma(sg, f.x, d.x);
        d.y = fma(sg, f.y, d.y);
        if (shifted) sg = -sg;
    }
    int m0 = N - k;  // m = jN - k, j >= 1
    sg = shifted ? -1.0 : 1.0;
    for (int m = m0; m <= lmax; m += N) {
        const double2 f = Fm[m];
        d.x = fma(sg, f.x, d.x);
        d.y = fma(-sg, f.y, d.y);
        if (shifted) sg = -sg;
    }
    return d;
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads, kFftMinBlocks) ring_synth_kernel(const int *__restrict__ ring_list,
                                                                     const RingDesc *__restrict__ rings, int lmax,
                                                                     int M, int nrings, long long npix,
                                                                     const double2 *__restrict__ F_all,
                                                                     double *__restrict__ maps_all,
                                                                     double2 *__restrict__ A_all,
                                                                     double2 *__restrict__ Y_all,
                                                                     const double2 *__restrict__ tw,
                                                                     const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    const int r = ring_list ? ring_list[blockIdx.x] : (int)blockIdx.x;
    const RingDesc rd = rings[r];
    const int N = rd.N, Q = rd.Q;
    const bool shifted = rd.phi0 != 0.0;
    constexpr int nchan = SPIN ? 2 : 1;
    const double2 *Fp = F_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    const double2 *Fm = SPIN ? Fp + (size_t)nrings * M : Fp;
    double *outQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    double *outU = outQ + npix;
    if (rd.mode == kDirect && Q == 1) {
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            const double2 d = fold_synth(Fp, Fm, k, N, lmax, shifted);
            buf[pidx(k)] = shifted ? cmul(d, cis_pi(k, N, 0, 1)) : d;
        }
        __syncthreads();
        fft_stockham(buf, N, +1.0, tw);
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            const double2 v = buf[pidx(j)];
            outQ[j] = v.x;
            if (SPIN) outU[j] = v.y;
        }
        return;
    }
    // Transform of length L (N, or the chirp-z length P) in Q pieces of Lp points.  One
    // pass writes the phased (and chirped) fold a[k] to the ring's scratch row; piece s
    // then folds a[k] e^{-+2 pi i s k / L} modulo Lp with table twiddles.
    const bool blue = rd.mode == kBluestein;
    const int L = blue ? rd.P : N, Lp = L / Q;
    double2 *Ag = A_all + (size_t)blockIdx.y * npix + rd.start;
    double2 *Yg = Y_all + (size_t)blockIdx.y * npix + rd.start;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const double2 d = fold_synth(Fp, Fm, k, N, lmax, shifted);
        // e^{i pi k / N} ring phase; chirp-z: times w(k) = e^{i pi k^2 / N}
        const int ph = (shifted ? k : 0) + (blue ? (k * k) % (2 * N) : 0);
        Ag[k] = ph ? cmul(d, cis_pi(ph, N, 0, 1)) : d;
    }
    __syncthreads();
    const double2 *B = bh + rd.bh_off;
    for (int s = 0; s < Q; ++s) {
        for (int q = threadIdx.x; q < Lp; q += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int k = q; k < N; k += Lp) {
                const double2 a = Ag[k];
                // direct: inverse DFT, e^{+2 pi i s k / N}; chirp-z: FFT_P, e^{-2 pi i s k / P}
                v = cadd(v, s ? cmul(a, twid(tw, s * k, L, !blue)) : a);
            }
            buf[pidx(q)] = v;
        }
        __syncthreads();
        if (!blue) {
            fft_stockham(buf, Lp, +1.0, tw);
            for (int q = threadIdx.x; q < Lp; q += blockDim.x) {
                const double2 v = buf[pidx(q)];
                outQ[Q * q + s] = v.x;
                if (SPIN) outU[Q * q + s] = v.y;
            }
            __syncthreads();
            continue;
        }
        fft_stockham(buf, Lp, -1.0, tw);
        for (int q = threadIdx.x; q < Lp; q += blockDim.x) buf[pidx(q)] = cmul(buf[pidx(q)], bh_get(B, L, Q * q + s, 1));
        __syncthreads();
        fft_stockham(buf, Lp, +1.0, tw);
        // y[j] += conv_s[j mod Lp] e^{2 pi i s j / P}; the chirp is applied once after the last piece
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            double2 v = buf[pidx(j & (Lp - 1))];
            if (s) v = cadd(Yg[j], cmul(v, twid(tw, s * j, L, true)));
            if (s < Q - 1) {
                Yg[j] = v;
            } else {
                v = cmul(v, cis_pi((j * j) % (2 * N), N, 0, 1));
                outQ[j] = v.x;
                if (SPIN) outU[j] = v.y;
            }
        }
        __syncthreads();
    }
}

// V rows for ring r from its spectrum W (padded shared-memory buffer or natural global).
template <int SPIN, bool PADDED>
__device__ __forceinline__ void gather_adjoint(const double2 *W, int N, int lmax, bool shifted, double2 *Vp,
                                               double2 *Vm) {
    for (int m = threadIdx.x; m <= lmax; m += blockDim.x) {
        const int k1 = m % N, k2 = (N - k1) % N;
        double2 vp = W[PADDED ? pidx(k1) : k1];
        double2 vm = SPIN ? conjd(W[PADDED ? pidx(k2) : k2]) : vp;
        if (shifted) {  // e^{-i m phi0} = e^{-i pi m / N}
            const double2 cph = cis_pi(-(m % (2 * N)), N, 0, 1);
            vp = cmul(vp, cph);
            vm = cmul(vm, cph);
        }
        Vp[m] = vp;
        if (SPIN) Vm[m] = vm;
    }
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads, kFftMinBlocks) ring_adjoint_kernel(const int *__restrict__ ring_list,
                                                                       const RingDesc *__restrict__ rings, int lmax,
                                                                       int M, int nrings, long long npix,
                                                                       const double *__restrict__ maps_all,
                                                                       double2 *__restrict__ V_all,
                                                                       double2 *__restrict__ A_all,
                                                                       double2 *__restrict__ W_all,
                                                                       const double2 *__restrict__ tw,
                                                                       const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    const int r = ring_list ? ring_list[blockIdx.x] : (int)blockIdx.x;
    const RingDesc rd = rings[r];
    const int N = rd.N, Q = rd.Q;
    const bool shifted = rd.phi0 != 0.0;
    constexpr int nchan = SPIN ? 2 : 1;
    const double *inQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    const double *inU = inQ + npix;
    double2 *Vp = V_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    double2 *Vm = SPIN ? Vp + (size_t)nrings * M : Vp;
    if (rd.mode == kDirect && Q == 1) {
        for (int j = threadIdx.x; j < N; j += blockDim.x) buf[pidx(j)] = make_double2(inQ[j], SPIN ? inU[j] : 0.0);
        __syncthreads();
        fft_stockham(buf, N, -1.0, tw);
        gather_adjoint<SPIN, true>(buf, N, lmax, shifted, Vp, Vm);
        return;
    }
    // Forward transform of length L (N, or P) in Q pieces of Lp points; the spectrum
    // W[k], k < N, is assembled in the ring's scratch row and then gathered.
    const bool blue = rd.mode == kBluestein;
    const int L = blue ? rd.P : N, Lp = L / Q;
    double2 *Ag = A_all + (size_t)blockIdx.y * npix + rd.start;
    double2 *Wg = W_all + (size_t)blockIdx.y * npix + rd.start;
    if (blue) {  // chirped input a[j] = v[j] conj(w(j)), once
        for (int j = threadIdx.x; j < N; j += blockDim.x)
            Ag[j] = cmul(make_double2(inQ[j], SPIN ? inU[j] : 0.0), cis_pi(-((j * j) % (2 * N)), N, 0, 1));
        __syncthreads();
    }
    const double2 *B = bh + rd.bh_off;
    for (int s = 0; s < Q; ++s) {
        for (int q = threadIdx.x; q < Lp; q += blockDim.x) {
            double2 v = make_double2(0.0, 0.0);
            for (int j = q; j < N; j += Lp) {
                const double2 a = blue ? Ag[j] : make_double2(inQ[j], SPIN ? inU[j] : 0.0);
                v = cadd(v, s ? cmul(a, twid(tw, s * j, L, false)) : a);  // e^{-2 pi i s j / L}
            }
            buf[pidx(q)] = v;
        }
        __syncthreads();
        fft_stockham(buf, Lp, -1.0, tw);
        if (!blue) {  // W[Q q + s]
            for (int q = threadIdx.x; q < Lp; q += blockDim.x) Wg[Q * q + s] = buf[pidx(q)];
            __syncthreads();
            continue;
        }
        for (int q = threadIdx.x; q < Lp; q += blockDim.x) buf[pidx(q)] = cmul(buf[pidx(q)], bh_get(B, L, Q * q + s, -1));
        __syncthreads();
        fft_stockham(buf, Lp, +1.0, tw);
        // W[k] = conj(w(k)) sum_s conv_s[k mod Lp] e^{2 pi i s k / P}, the chirp after the last piece
        for (int k = threadIdx.x; k < N; k += blockDim.x) {
            double2 v = buf[pidx(k & (Lp - 1))];
            if (s) v = cadd(Wg[k], cmul(v, twid(tw, s * k, L, true)));
            if (s == Q - 1) v = cmul(v, cis_pi(-((k * k) % (2 * N)), N, 0, 1));
            Wg[k] = v;
        }
        __syncthreads();
    }
    __threadfence_block();
    gather_adjoint<SPIN, false>(Wg, N, lmax, shifted, Vp, Vm);
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
    const int Q = P > kFftPiece ? P / kFftPiece : 1;
    const int s = blockIdx.y;
    if (s >= Q) return;
    const int Pp = P / Q;
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
        buf[pidx(q)] = v;
    }
    __syncthreads();
    fft_stockham(buf, Pp, -1.0, tw);
    const double inv = 1.0 / (double)P;
    for (int q = threadIdx.x; q < Pp; q += blockDim.x) {
        const double2 v = buf[pidx(q)];
        out[(long long)Q * q + s] = make_double2(v.x * inv, v.y * inv);
    }
}

int smem_bytes() { return kFftBufLen * (int)sizeof(double2); }

template <typename K>
int ensure_smem(K kernel) {
    JHTB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes()));
    return JHTB_OK;
}

}  // namespace

int launch_ring_synth(const Plan &p, const double2 *F, double *maps, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.d_ring_list ? p.nring_list : p.nrings, nb);
    int rc;
    if (p.spin == 0) {
        if ((rc = ensure_smem(ring_synth_kernel<0>))) return rc;
        ring_synth_kernel<0><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_ring_list, p.d_rings, p.lmax, p.M, p.nrings, p.npix, F,
                                                                     maps, p.d_W, p.d_W2, p.d_tw, p.d_bh);
    } else {
        if ((rc = ensure_smem(ring_synth_kernel<2>))) return rc;
        ring_synth_kernel<2><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_ring_list, p.d_rings, p.lmax, p.M, p.nrings, p.npix, F,
                                                                     maps, p.d_W, p.d_W2, p.d_tw, p.d_bh);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_ring_adjoint(const Plan &p, const double *maps, double2 *V, double2 *W, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.d_ring_list ? p.nring_list : p.nrings, nb);
    int rc;
    if (p.spin == 0) {
        if ((rc = ensure_smem(ring_adjoint_kernel<0>))) return rc;
        ring_adjoint_kernel<0><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_ring_list, p.d_rings, p.lmax, p.M, p.nrings, p.npix,
                                                                       maps, V, p.d_W2, W, p.d_tw, p.d_bh);
    } else {
        if ((rc = ensure_smem(ring_adjoint_kernel<2>))) return rc;
        ring_adjoint_kernel<2><<<grid, kFftThreads, smem_bytes(), s>>>(p.d_ring_list, p.d_rings, p.lmax, p.M, p.nrings, p.npix,
                                                                       maps, V, p.d_W2, W, p.d_tw, p.d_bh);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_bluestein_setup(const Plan &p, const int *lengths, const long long *offs, int nlen, cudaStream_t s) {
    if (nlen <= 0) return JHTB_OK;
    int rc;
    if ((rc = ensure_smem(bluestein_setup_kernel))) return rc;
    dim3 grid(nlen, 8);
    bluestein_setup_kernel<<<grid, kFftThreads, smem_bytes(), s>>>(lengths, offs, p.d_tw, p.d_bh);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // namespace jhtb
