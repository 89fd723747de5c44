// Azimuthal stage: per-ring phase shift, m -> k fold and length-N DFT (sm_100a).
//
// jht (healpix.py:280-355) groups rings by length and emits one FFT per distinct
// length, with scatter-adds for the m -> k fold.  Here a CTA owns a ring (or a piece of one):
//   synthesis  D[k] = sum_{m = k mod N} Fp_m e^{i m phi0} + sum_{m>=1, -m = k mod N} conj(Fm_m e^{i m phi0})
//              out[j] = sum_k D[k] e^{+2 pi i jk/N}      (real part: spin 0; Q + iU: spin 2)
//   adjoint    W[k] = sum_j v[j] e^{-2 pi i jk/N};  V[m] = W[m mod N] e^{-i m phi0}
//              (spin 2 also Vm[m] = conj(W[-m mod N]) e^{-i m phi0})
// The fold is a gather (each k collects its own m's), never a scatter.  Power-of-two
// rings use an in-place Stockham FFT in shared memory (radix-16 passes held in
// registers, natural order in and out, a padded layout against bank conflicts; 70 KB of
// shared memory per CTA, two CTAs per SM); every other length uses Bluestein's chirp-z
// with an exact (n^2 mod 2N) chirp argument (_azimuth.py:150-191) at a power-of-two length
// P >= 2N-1.  Rings whose transform exceeds 4096 points run as independent pieces, one CTA
// per output residue class (decimation in frequency on the input, no data exchange): the
// power-of-two belt rings in N / 4096 pieces and the long polar-cap rings (N = 4 qn) as four
// chirp-z pieces of length qn; only chirp-z lengths above 16384 (cap rings at nside > 2048)
// are split inside one CTA through the ring's scratch rows.
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
#ifndef JHTB_PIECE_MINB
#define JHTB_PIECE_MINB 2
#endif
constexpr int kPieceMinBlocks = JHTB_PIECE_MINB;  // resident CTAs per SM of the piece kernels
#ifndef JHTB_PIECE_U
#define JHTB_PIECE_U 4
#endif
constexpr int kUP = JHTB_PIECE_U;  // elements per thread whose gathers the piece kernels issue together

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
    double2 w = JHTB_IN(r * (kTwLen / L), kTwLen, 107) ? __ldg(&tw[r * (kTwLen / L)]) : make_double2(0.0, 0.0);
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
                    double2 w = JHTB_IN(step * r, kTwLen, 107) ? __ldg(&tw[step * r]) : make_double2(0.0, 0.0);
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

// Twiddles from shared memory: e^{-2 pi i x / kFftPiece} = T[x >> 6] T[64 + (x & 63)] with
// T[a] = e^{-2 pi i a / 64} and T[64 + b] = e^{-2 pi i b / kFftPiece} (each entry rounded once,
// the product adds about one rounding), so the passes make no global loads.
// Eight more entries T[128 + g] = e^{-2 pi i g / kTwLen} refine it to kTwLen points (the ring
// phases and piece twiddles of power-of-two rings up to kTwLen / 2 points).
constexpr int kSmTwLen = 136;
constexpr int kSmTwFine = kTwLen / kFftPiece;  // 8
static_assert(kFftPiece == 64 * 64, "two-level twiddle table of kFftPiece points");
__device__ __forceinline__ void sm_tw_init(double2 *T) {
    for (int a = threadIdx.x; a < kSmTwLen; a += blockDim.x) {
        double s, c;
        if (a < 64) sincospi(-2.0 * (double)a / 64.0, &s, &c);
        else if (a < 128) sincospi(-2.0 * (double)(a - 64) / (double)kFftPiece, &s, &c);
        else sincospi(-2.0 * (double)(a - 128) / (double)kTwLen, &s, &c);
        T[a] = make_double2(c, s);
    }
}
__device__ __forceinline__ double2 sm_tw(const double2 *T, int x, bool plus) {  // e^{-+2 pi i x / kFftPiece}
    x &= kFftPiece - 1;
    double2 w = cmul(T[x >> 6], T[64 + (x & 63)]);
    if (plus) w.y = -w.y;
    return w;
}

// e^{+i pi a / N} for a power-of-two N, kFftPiece / 2 <= N <= kTwLen / 2, from the shared
// table: with x = a mod 2N = q y + f (q = 2N / kFftPiece), the conjugate of
// e^{-2 pi i y / kFftPiece} e^{-2 pi i f / 2N}.
__device__ __forceinline__ double2 sm_tw_pi(const double2 *T, long long a, int N) {
    const int x = (int)(a & (2LL * N - 1)), q = 2 * N / kFftPiece;
    double2 w = cmul(sm_tw(T, x / q, false), T[128 + (x % q) * (kSmTwFine / q)]);
    w.y = -w.y;
    return w;
}

// stockham_pass with the shared-memory twiddle table.
template <int R>
__device__ __forceinline__ void stockham_pass_sm(double2 *buf, int n, int Ns, double dir, const double2 *T) {
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
                const int step = jm * (kFftPiece / (Ns * R));
#pragma unroll
                for (int r = 1; r < R; ++r) v[jj][r] = cmul(v[jj][r], sm_tw(T, step * r, dir > 0));
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

// The FFT with every pass inlined (no call boundary, so no register saves to the stack
// around the passes) and shared-memory twiddles; for kernels that run one or two transforms.
// Largest radix of the piece kernels' passes (16: fewer passes; 8: fewer registers).
#ifndef JHTB_PIECE_RADIX
#define JHTB_PIECE_RADIX 16
#endif
__device__ __forceinline__ void fft_stockham_sm(double2 *buf, int n, double dir, const double2 *T) {
    int bits = ilog2i(n), Ns = 1;
    if (JHTB_PIECE_RADIX >= 16) {
        for (; bits >= 4; bits -= 4, Ns <<= 4) stockham_pass_sm<16>(buf, n, Ns, dir, T);
        if (bits == 3) stockham_pass_sm<8>(buf, n, Ns, dir, T);
    } else {
        for (; bits >= 3; bits -= 3, Ns <<= 3) stockham_pass_sm<8>(buf, n, Ns, dir, T);
    }
    if (bits == 2) stockham_pass_sm<4>(buf, n, Ns, dir, T);
    else if (bits == 1) stockham_pass_sm<2>(buf, n, Ns, dir, T);
}

// Bluestein spectrum for the synthesis direction: Bh+ = FFT_P(b)/P with
// b[n] = conj(w(n)) on |n| < N, w(n) = e^{+i pi n^2 / N}.  The adjoint direction
// uses Bh-[k] = conj(Bh+[(P - k) mod P]).
__device__ __forceinline__ double2 bh_get(const double2 *bh, int P, int k, int sgn) {
    if (!JHTB_IN(k, P, 108)) return make_double2(0.0, 0.0);
    if (sgn > 0) return __ldg(&bh[k]);
    return conjd(__ldg(&bh[(P - k) & (P - 1)]));
}

// D[k] of the synthesis fold for one ring, without its phase (spin 0 passes Fm == Fp):
// with m = k + jN in the first sum and m = jN - k in the second,
// e^{i m phi0} = (-1)^j e^{+-i pi k / N} when phi0 = pi / N, so
// D[k] = e^{i pi k / N} [sum_j (-1)^j Fp_{k+jN} + sum_j (-1)^j conj(Fm_{jN-k})];
// `shifted` selects the (-1)^j signs, the caller applies e^{i pi k / N}.  Aliases
// j = part, part + parts, ... only (the caller sums the parts in a fixed order).
__device__ __forceinline__ double2 fold_synth(const double2 *__restrict__ Fp, const double2 *__restrict__ Fm,
                                              int k, int N, int lmax, bool shifted, int part = 0, int parts = 1) {
    double2 d = make_double2(0.0, 0.0);
    const double flip = (shifted && (parts & 1)) ? -1.0 : 1.0;  // sign change per step of `parts` aliases
    double sg = (shifted && (part & 1)) ? -1.0 : 1.0;
    const int step = parts * N;
#pragma unroll 4
    for (int m = k + part * N; m <= lmax; m += step) {
        const double2 f = JHTB_IN(m, lmax + 1, 101) ? Fp[m] : make_double2(0.0, 0.0);
        d.x = fma(sg, f.x, d.x);
        d.y = fma(sg, f.y, d.y);
        sg *= flip;
    }
    // m = jN - k, j >= 1: alias j = 1 + part, 1 + part + parts, ...
    sg = (shifted && ((1 + part) & 1)) ? -1.0 : 1.0;
#pragma unroll 4
    for (int m = (1 + part) * N - k; m <= lmax; m += step) {
        const double2 f = JHTB_IN(m, lmax + 1, 102) ? Fm[m] : make_double2(0.0, 0.0);
        d.x = fma(sg, f.x, d.x);
        d.y = fma(-sg, f.y, d.y);
        sg *= flip;
    }
    return d;
}

// Elements per thread whose global loads are issued together in the azimuthal loops (the
// loops are bound by L2 / HBM latency, not by arithmetic).
constexpr int kU = 4;

// The phased (and, for chirp-z, chirped) fold a[k] for k < N into dst[k] (padded shared
// buffer or a global row).  Rings longer than lmax have at most one term per sum, loaded
// kU elements at a time; shorter rings split each k's aliases over blockDim / N threads
// when N < blockDim (partial sums combined in a fixed order through `part_buf`).
template <bool PADDED>
__device__ __forceinline__ void synth_fold(const double2 *__restrict__ Fp, const double2 *__restrict__ Fm, int N,
                                           int lmax, bool shifted, bool blue, double2 *dst, double2 *part_buf) {
    auto phase = [&](int k, double2 d) {
        // e^{i pi k / N} ring phase; chirp-z: times w(k) = e^{i pi k^2 / N}
        const int ph = (shifted ? k : 0) + (blue ? (int)(((long long)k * k) % (2 * N)) : 0);
        return ph ? cmul(d, cis_pi(ph, N, 0, 1)) : d;
    };
    if (N > lmax) {
        const double sg = shifted ? -1.0 : 1.0;
        for (int k0 = threadIdx.x; k0 < N; k0 += kU * blockDim.x) {
            double2 fp[kU], fm[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int k = k0 + u * blockDim.x;
                fp[u] = (k < N && k <= lmax && JHTB_IN(k, lmax + 1, 101)) ? Fp[k] : make_double2(0.0, 0.0);
                fm[u] = (k < N && k >= 1 && N - k <= lmax && JHTB_IN(N - k, lmax + 1, 102)) ? Fm[N - k] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int k = k0 + u * blockDim.x;
                if (k < N) {
                    const double2 d = make_double2(fma(sg, fm[u].x, fp[u].x), fma(-sg, fm[u].y, fp[u].y));
                    dst[PADDED ? pidx(k) : k] = phase(k, d);
                }
            }
        }
        return;
    }
    const int parts = N < (int)blockDim.x ? (int)blockDim.x / N : 1;
    if (parts == 1) {
        for (int k = threadIdx.x; k < N; k += blockDim.x) dst[PADDED ? pidx(k) : k] = phase(k, fold_synth(Fp, Fm, k, N, lmax, shifted));
        return;
    }
    if ((int)threadIdx.x < N * parts) {
        const int k = threadIdx.x % N, part = threadIdx.x / N;
        part_buf[threadIdx.x] = fold_synth(Fp, Fm, k, N, lmax, shifted, part, parts);
    }
    __syncthreads();
    if ((int)threadIdx.x < N) {
        double2 d = part_buf[threadIdx.x];
        for (int q = 1; q < parts; ++q) d = cadd(d, part_buf[q * N + threadIdx.x]);
        dst[PADDED ? pidx(threadIdx.x) : threadIdx.x] = phase(threadIdx.x, d);
    }
}

// Scratch for the fold's partial sums of short rings (N < blockDim), past the part of the
// padded FFT buffer such rings use (their transforms have at most 512 points).
constexpr int kPartOff = 2048;

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
    const bool blue = rd.mode == kBluestein;
    constexpr int nchan = SPIN ? 2 : 1;
    const double2 *Fp = F_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    const double2 *Fm = SPIN ? Fp + (size_t)nrings * M : Fp;
    double *outQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    double *outU = outQ + npix;
    const int bd = blockDim.x;
    const double2 *B = bh + rd.bh_off;
    if (Q == 1) {
        // the whole transform in shared memory: fold (chirped for chirp-z, zero-padded to P)
        const int L = blue ? rd.P : N;
        synth_fold<true>(Fp, Fm, N, lmax, shifted, blue, buf, buf + kPartOff);
        for (int k = N + threadIdx.x; k < L; k += bd) buf[pidx(k)] = make_double2(0.0, 0.0);
        __syncthreads();
        if (blue) {
            fft_stockham(buf, L, -1.0, tw);
            for (int q0 = threadIdx.x; q0 < L; q0 += kU * bd) {
                double2 w[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) w[u] = q0 + u * bd < L ? bh_get(B, L, q0 + u * bd, 1) : make_double2(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (q0 + u * bd < L) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
            }
            __syncthreads();
        }
        fft_stockham(buf, L, +1.0, tw);
        for (int j = threadIdx.x; j < N; j += bd) {
            double2 v = buf[pidx(j)];
            if (blue) v = cmul(v, cis_pi((int)(((long long)j * j) % (2 * N)), N, 0, 1));
            if (JHTB_IN(rd.start + j, npix, 104)) {
                outQ[j] = v.x;
                if (SPIN) outU[j] = v.y;
            }
        }
        return;
    }
    // Transform of length L (N, or the chirp-z length P) in Q pieces of Lp points.  One
    // pass writes the phased (and chirped) fold a[k] to the ring's scratch row; piece s
    // then folds a[k] e^{-+2 pi i s k / L} modulo Lp with table twiddles.
    const int L = blue ? rd.P : N, Lp = L / Q;
    double2 *Ag = A_all + (size_t)blockIdx.y * npix + rd.start;
    double2 *Yg = Y_all + (size_t)blockIdx.y * npix + rd.start;
    synth_fold<false>(Fp, Fm, N, lmax, shifted, blue, Ag, buf + kPartOff);
    __syncthreads();
    for (int s = 0; s < Q; ++s) {
        for (int q0 = threadIdx.x; q0 < Lp; q0 += kU * bd) {
            double2 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) v[u] = make_double2(0.0, 0.0);
            for (int t = 0; t * Lp < N; ++t) {
                double2 a[kU], w[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int k = q0 + u * bd + t * Lp;
                    const bool ok = q0 + u * bd < Lp && k < N;
                    a[u] = (ok && JHTB_IN(rd.start + k, npix, 109)) ? Ag[k] : make_double2(0.0, 0.0);
                    // direct: inverse DFT, e^{+2 pi i s k / N}; chirp-z: FFT_P, e^{-2 pi i s k / P}
                    w[u] = (ok && s) ? twid(tw, s * k, L, !blue) : make_double2(1.0, 0.0);
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) v[u] = cadd(v[u], cmul(a[u], w[u]));
            }
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (q0 + u * bd < Lp) buf[pidx(q0 + u * bd)] = v[u];
        }
        __syncthreads();
        if (!blue) {
            fft_stockham(buf, Lp, +1.0, tw);
            for (int q = threadIdx.x; q < Lp; q += bd) {
                const double2 v = buf[pidx(q)];
                if (JHTB_IN(rd.start + (long long)Q * q + s, npix, 104)) {
                    outQ[Q * q + s] = v.x;
                    if (SPIN) outU[Q * q + s] = v.y;
                }
            }
            __syncthreads();
            continue;
        }
        fft_stockham(buf, Lp, -1.0, tw);
        for (int q0 = threadIdx.x; q0 < Lp; q0 += kU * bd) {
            double2 w[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) w[u] = q0 + u * bd < Lp ? bh_get(B, L, Q * (q0 + u * bd) + s, 1) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (q0 + u * bd < Lp) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
        }
        __syncthreads();
        fft_stockham(buf, Lp, +1.0, tw);
        // y[j] += conv_s[j mod Lp] e^{2 pi i s j / P}; the chirp is applied once after the last piece
        for (int j0 = threadIdx.x; j0 < N; j0 += kU * bd) {
            double2 y[kU], w[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int j = j0 + u * bd;
                y[u] = (s && j < N && JHTB_IN(rd.start + j, npix, 109)) ? Yg[j] : make_double2(0.0, 0.0);
                w[u] = (s && j < N) ? twid(tw, s * j, L, true) : make_double2(1.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int j = j0 + u * bd;
                if (j >= N) continue;
                double2 v = cadd(y[u], cmul(buf[pidx(j & (Lp - 1))], w[u]));
                if (s < Q - 1) {
                    if (JHTB_IN(rd.start + j, npix, 109)) Yg[j] = v;
                } else {
                    v = cmul(v, cis_pi((int)(((long long)j * j) % (2 * N)), N, 0, 1));
                    if (JHTB_IN(rd.start + j, npix, 104)) {
                        outQ[j] = v.x;
                        if (SPIN) outU[j] = v.y;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// V rows for ring r from its spectrum W (padded shared-memory buffer or natural global),
// kU orders per thread at a time so the loads of a global W overlap.
template <int SPIN, bool PADDED>
__device__ __forceinline__ void gather_adjoint(const double2 *W, int N, int lmax, bool shifted, double2 *Vp,
                                               double2 *Vm) {
    const int bd = blockDim.x;
    for (int m0 = threadIdx.x; m0 <= lmax; m0 += kU * bd) {
        double2 vp[kU], vm[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int m = m0 + u * bd;
            const int k1 = m % N, k2 = (N - k1) % N;
            vp[u] = m <= lmax ? W[PADDED ? pidx(k1) : k1] : make_double2(0.0, 0.0);
            vm[u] = (SPIN && m <= lmax) ? conjd(W[PADDED ? pidx(k2) : k2]) : vp[u];
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int m = m0 + u * bd;
            if (m > lmax) continue;
            double2 p = vp[u], q = vm[u];
            if (shifted) {  // e^{-i m phi0} = e^{-i pi m / N}
                const double2 cph = cis_pi(-(m % (2 * N)), N, 0, 1);
                p = cmul(p, cph);
                q = cmul(q, cph);
            }
            if (JHTB_IN(m, lmax + 1, 105)) {
                Vp[m] = p;
                if (SPIN) Vm[m] = q;
            }
        }
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
    const bool blue = rd.mode == kBluestein;
    constexpr int nchan = SPIN ? 2 : 1;
    const double *inQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    const double *inU = inQ + npix;
    double2 *Vp = V_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    double2 *Vm = SPIN ? Vp + (size_t)nrings * M : Vp;
    const int bd = blockDim.x;
    const double2 *B = bh + rd.bh_off;
    // the ring's pixels (chirped for chirp-z: a[j] = v[j] conj(w(j))), kU at a time
    auto load_in = [&](int j0, double2 (&a)[kU]) {
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int j = j0 + u * bd;
            a[u] = (j < N && JHTB_IN(rd.start + j, npix, 103)) ? make_double2(inQ[j], SPIN ? inU[j] : 0.0) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int j = j0 + u * bd;
            if (blue && j < N) a[u] = cmul(a[u], cis_pi(-(int)(((long long)j * j) % (2 * N)), N, 0, 1));
        }
    };
    if (Q == 1) {
        // the whole transform in shared memory
        const int L = blue ? rd.P : N;
        for (int j0 = threadIdx.x; j0 < N; j0 += kU * bd) {
            double2 a[kU];
            load_in(j0, a);
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (j0 + u * bd < N) buf[pidx(j0 + u * bd)] = a[u];
        }
        for (int k = N + threadIdx.x; k < L; k += bd) buf[pidx(k)] = make_double2(0.0, 0.0);
        __syncthreads();
        fft_stockham(buf, L, -1.0, tw);
        if (blue) {
            for (int q0 = threadIdx.x; q0 < L; q0 += kU * bd) {
                double2 w[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) w[u] = q0 + u * bd < L ? bh_get(B, L, q0 + u * bd, -1) : make_double2(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < kU; ++u)
                    if (q0 + u * bd < L) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
            }
            __syncthreads();
            fft_stockham(buf, L, +1.0, tw);
            // W[k] = conj(w(k)) conv[k]
            for (int k = threadIdx.x; k < N; k += bd)
                buf[pidx(k)] = cmul(buf[pidx(k)], cis_pi(-(int)(((long long)k * k) % (2 * N)), N, 0, 1));
            __syncthreads();
        }
        gather_adjoint<SPIN, true>(buf, N, lmax, shifted, Vp, Vm);
        return;
    }
    // Forward transform of length L (N, or P) in Q pieces of Lp points; the spectrum
    // W[k], k < N, is assembled in the ring's scratch row and then gathered.
    const int L = blue ? rd.P : N, Lp = L / Q;
    double2 *Ag = A_all + (size_t)blockIdx.y * npix + rd.start;
    double2 *Wg = W_all + (size_t)blockIdx.y * npix + rd.start;
    if (blue) {  // chirped input a[j] = v[j] conj(w(j)), once
        for (int j0 = threadIdx.x; j0 < N; j0 += kU * bd) {
            double2 a[kU];
            load_in(j0, a);
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (j0 + u * bd < N && JHTB_IN(rd.start + j0 + u * bd, npix, 109)) Ag[j0 + u * bd] = a[u];
        }
        __syncthreads();
    }
    for (int s = 0; s < Q; ++s) {
        for (int q0 = threadIdx.x; q0 < Lp; q0 += kU * bd) {
            double2 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) v[u] = make_double2(0.0, 0.0);
            for (int t = 0; t * Lp < N; ++t) {
                double2 a[kU], w[kU];
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const int j = q0 + u * bd + t * Lp;
                    const bool ok = q0 + u * bd < Lp && j < N;
                    a[u] = !ok ? make_double2(0.0, 0.0) : blue ? Ag[j] : make_double2(inQ[j], SPIN ? inU[j] : 0.0);
                    w[u] = (ok && s) ? twid(tw, s * j, L, false) : make_double2(1.0, 0.0);  // e^{-2 pi i s j / L}
                }
#pragma unroll
                for (int u = 0; u < kU; ++u) v[u] = cadd(v[u], cmul(a[u], w[u]));
            }
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (q0 + u * bd < Lp) buf[pidx(q0 + u * bd)] = v[u];
        }
        __syncthreads();
        fft_stockham(buf, Lp, -1.0, tw);
        if (!blue) {  // W[Q q + s]
            for (int q = threadIdx.x; q < Lp; q += bd)
                if (JHTB_IN(rd.start + (long long)Q * q + s, npix, 109)) Wg[Q * q + s] = buf[pidx(q)];
            __syncthreads();
            continue;
        }
        for (int q0 = threadIdx.x; q0 < Lp; q0 += kU * bd) {
            double2 w[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) w[u] = q0 + u * bd < Lp ? bh_get(B, L, Q * (q0 + u * bd) + s, -1) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (q0 + u * bd < Lp) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
        }
        __syncthreads();
        fft_stockham(buf, Lp, +1.0, tw);
        // W[k] = conj(w(k)) sum_s conv_s[k mod Lp] e^{2 pi i s k / P}, the chirp after the last piece
        for (int k0 = threadIdx.x; k0 < N; k0 += kU * bd) {
            double2 y[kU], w[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int k = k0 + u * bd;
                y[u] = (s && k < N && JHTB_IN(rd.start + k, npix, 109)) ? Wg[k] : make_double2(0.0, 0.0);
                w[u] = (s && k < N) ? twid(tw, s * k, L, true) : make_double2(1.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int k = k0 + u * bd;
                if (k >= N) continue;
                double2 v = cadd(y[u], cmul(buf[pidx(k & (Lp - 1))], w[u]));
                if (s == Q - 1) v = cmul(v, cis_pi(-(int)(((long long)k * k) % (2 * N)), N, 0, 1));
                if (JHTB_IN(rd.start + k, npix, 109)) Wg[k] = v;
            }
        }
        __syncthreads();
    }
    __threadfence_block();
    gather_adjoint<SPIN, false>(Wg, N, lmax, shifted, Vp, Vm);
}

// ---------------------------------------------------------------------------------
// Long rings in pieces: a ring of N = Q Lq points (a power of two above kFftPiece, Lq =
// kFftPiece; or a kSplit4 polar-cap ring, N = 4 Lq with Lq not a power of two) runs as Q
// independent CTAs of the 256-thread shared-memory kernel, one per output residue class
// (decimation in frequency).  Piece s:
//   synthesis  out[Q j + s] = sum_{k1 < Lq} e^{+2 pi i j k1 / Lq} a_s[k1],
//              a_s[k1]      = sum_{k2 < Q} D[k1 + Lq k2] e^{+2 pi i s (k1 + Lq k2) / N}
//   adjoint    W[Q k + s]   = sum_{j1 < Lq} e^{-2 pi i k j1 / Lq} b_s[j1],
//              b_s[j1]      = sum_{j2 < Q} v[j1 + Lq j2] e^{-2 pi i s (j1 + Lq j2) / N}
// with D the phased fold of the synthesis and v the ring's pixels.  The length-Lq
// transform is the Stockham FFT (power of two) or a chirp-z transform at P <= kFftPiece
// points (kSplit4).  Every piece gathers the whole ring's input itself (the Q reads of a
// ring's data hit L2), so pieces never exchange data and several fit on an SM at once.
// ---------------------------------------------------------------------------------
// e^{+i pi a / N} for a power-of-two N <= kTwLen / 2, from the twiddle table (entries
// e^{-2 pi i j / kTwLen}, each rounded once).
__device__ __forceinline__ double2 tw_pi(const double2 *__restrict__ tw, long long a, int N) {
    const int r = (int)(a & (2LL * N - 1));
    double2 w = JHTB_IN(r * (kTwLen / (2 * N)), kTwLen, 107) ? __ldg(&tw[r * (kTwLen / (2 * N))]) : make_double2(0.0, 0.0);
    w.y = -w.y;
    return w;
}
// most pieces of a ring (ring_pieces: a power of two N <= kTwLen / 2 in N / kFftPiece, kSplit4 in 4)
constexpr int kMaxPieces = 4;
static_assert(kTwLen / 2 / kFftPiece <= kMaxPieces, "pieces of the longest power-of-two ring");

// e^{i pi k / 4}, k mod 8
__device__ __forceinline__ double2 root8(int k) {
    constexpr double h = 0.70710678118654752440;
    switch (k & 7) {
        case 0: return make_double2(1.0, 0.0);
        case 1: return make_double2(h, h);
        case 2: return make_double2(0.0, 1.0);
        case 3: return make_double2(-h, h);
        case 4: return make_double2(-1.0, 0.0);
        case 5: return make_double2(-h, -h);
        case 6: return make_double2(0.0, -1.0);
        default: return make_double2(h, -h);
    }
}

// D[k] of the synthesis fold without its ring phase (see fold_synth); one term per sum
// when the ring is longer than lmax.
__device__ __forceinline__ double2 fold_one(const double2 *__restrict__ Fp, const double2 *__restrict__ Fm, int k, int N,
                                            int lmax, bool shifted) {
    if (N <= lmax) return fold_synth(Fp, Fm, k, N, lmax, shifted);
    const double2 fp = (k <= lmax && JHTB_IN(k, lmax + 1, 101)) ? Fp[k] : make_double2(0.0, 0.0);
    const double2 fm = (k >= 1 && N - k <= lmax && JHTB_IN(N - k, lmax + 1, 102)) ? Fm[N - k] : make_double2(0.0, 0.0);
    const double sg = shifted ? -1.0 : 1.0;
    return make_double2(fma(sg, fm.x, fp.x), fma(-sg, fm.y, fp.y));
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads, kPieceMinBlocks) ring_synth_piece_kernel(const int *__restrict__ piece_list,
                                                                           const RingDesc *__restrict__ rings, int lmax,
                                                                           int M, int nrings, long long npix,
                                                                           const double2 *__restrict__ F_all,
                                                                           double *__restrict__ maps_all,
                                                                           const double2 *__restrict__ tw,
                                                                           const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    double2 *T = buf + kFftBufLen;  // twiddle table after the FFT buffer
    sm_tw_init(T);
    const int code = piece_list[blockIdx.x];
    const int r = code >> 3, s = code & 7;
    const RingDesc rd = rings[r];
    const int N = rd.N, Q = ring_pieces(rd), Lq = N / Q;
    const bool split = rd.mode == kSplit4;
    const bool shifted = rd.phi0 != 0.0;
    const int c = (shifted ? 1 : 0) + 2 * s;  // term k carries e^{i pi c k / N} (ring phase and piece twiddle)
    constexpr int nchan = SPIN ? 2 : 1;
    const double2 *Fp = F_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    const double2 *Fm = SPIN ? Fp + (size_t)nrings * M : Fp;
    double *outQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    double *outU = outQ + npix;
    const int bd = blockDim.x;
    if (!split && Q == 2) {
        // the belt's two-piece rings: 2 kUP values of k1 per thread and round (two loads each,
        // all issued first), twiddles from the shared table
        constexpr int U = 2 * kUP;
        const double2 r1 = root8(2 * c);  // e^{i pi c / 2}: exactly +-1 or +-i
        for (int k10 = threadIdx.x; k10 < Lq; k10 += U * bd) {
            double2 d0[U], d1[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k1 = k10 + u * bd;
                d0[u] = k1 < Lq ? fold_one(Fp, Fm, k1, N, lmax, shifted) : make_double2(0.0, 0.0);
                d1[u] = k1 < Lq ? fold_one(Fp, Fm, k1 + Lq, N, lmax, shifted) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k1 = k10 + u * bd;
                if (k1 >= Lq) continue;
                const double2 v = cmul(cadd(d0[u], cmul(d1[u], r1)), sm_tw_pi(T, (long long)c * k1, N));
                if (JHTB_IN(pidx(k1), kFftBufLen, 106)) buf[pidx(k1)] = v;
            }
        }
    }
    // a_s[k1]: the Q aliases k1 + Lq k2 of the phased fold, kUP values of k1 per thread at a time
    for (int k10 = threadIdx.x; k10 < Lq && (split || Q != 2); k10 += kUP * bd) {
        double2 acc[kUP];
#pragma unroll
        for (int u = 0; u < kUP; ++u) acc[u] = make_double2(0.0, 0.0);
        // every load of the kUP x Q terms (and, for a power of two, of the kUP twiddles) is
        // issued before the first is used
        double2 d[kMaxPieces][kUP], w1[kUP];
#pragma unroll
        for (int k2 = 0; k2 < kMaxPieces; ++k2)
#pragma unroll
            for (int u = 0; u < kUP; ++u) {
                const int k1 = k10 + u * bd;
                d[k2][u] = (k2 < Q && k1 < Lq) ? fold_one(Fp, Fm, k1 + Lq * k2, N, lmax, shifted) : make_double2(0.0, 0.0);
            }
#pragma unroll
        for (int u = 0; u < kUP; ++u) {
            const int k1 = k10 + u * bd;
            w1[u] = (!split && k1 < Lq) ? tw_pi(tw, (long long)c * k1, N) : make_double2(1.0, 0.0);
        }
        // e^{i pi c (k1 + Lq k2) / N} = e^{i pi c k1 / N} e^{i pi c k2 / Q}: the k2 factor is an
        // eighth root of unity (exactly +-1, +-i for Q = 2), the k1 factor is applied once
#pragma unroll
        for (int k2 = 0; k2 < kMaxPieces; ++k2) {
            if (k2 >= Q) break;
            const double2 w = root8((4 / Q) * c * k2);
#pragma unroll
            for (int u = 0; u < kUP; ++u) acc[u] = cadd(acc[u], k2 ? cmul(d[k2][u], w) : d[k2][u]);
        }
#pragma unroll
        for (int u = 0; u < kUP; ++u) {
            const int k1 = k10 + u * bd;
            if (k1 >= Lq) continue;
            // power of two: e^{i pi c k1 / N} from the table; kSplit4: e^{i pi c k1 / N} times the
            // chirp w(k1) = e^{i pi k1^2 / Lq} = e^{i pi 4 k1^2 / N}, one exactly reduced argument
            const double2 v = split ? cmul(acc[u], cis_pi((int)(((long long)c * k1 + 4LL * k1 * k1) % (2LL * N)), N, 0, 1))
                                    : cmul(acc[u], w1[u]);
            if (JHTB_IN(pidx(k1), kFftBufLen, 106)) buf[pidx(k1)] = v;
        }
    }
    const int L = split ? rd.P : Lq;
    for (int k = Lq + threadIdx.x; k < L; k += bd) buf[pidx(k)] = make_double2(0.0, 0.0);
    __syncthreads();
    if (split) {  // E[j] = w(j) sum_k (a[k] w(k)) conj(w(j - k)): FFT, chirp spectrum, inverse FFT
        fft_stockham_sm(buf, L, -1.0, T);
        for (int q0 = threadIdx.x; q0 < L; q0 += kUP * bd) {
            double2 w[kUP];
#pragma unroll
            for (int u = 0; u < kUP; ++u) w[u] = q0 + u * bd < L ? bh_get(bh + rd.bh_off, L, q0 + u * bd, 1) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < kUP; ++u)
                if (q0 + u * bd < L) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
        }
        __syncthreads();
    }
    fft_stockham_sm(buf, L, +1.0, T);
    for (int j = threadIdx.x; j < Lq; j += bd) {
        double2 v = buf[pidx(j)];
        if (split) v = cmul(v, cis_pi((int)(((long long)j * j) % (2 * Lq)), Lq, 0, 1));
        if (JHTB_IN(rd.start + (long long)Q * j + s, npix, 104)) {
            outQ[(size_t)Q * j + s] = v.x;
            if (SPIN) outU[(size_t)Q * j + s] = v.y;
        }
    }
}

template <int SPIN>
__global__ void __launch_bounds__(kFftThreads, kPieceMinBlocks) ring_adjoint_piece_kernel(const int *__restrict__ piece_list,
                                                                             const RingDesc *__restrict__ rings, int lmax,
                                                                             int M, int nrings, long long npix,
                                                                             const double *__restrict__ maps_all,
                                                                             double2 *__restrict__ V_all,
                                                                             const double2 *__restrict__ tw,
                                                                             const double2 *__restrict__ bh) {
    extern __shared__ double2 buf[];
    double2 *T = buf + kFftBufLen;  // twiddle table after the FFT buffer
    sm_tw_init(T);
    const int code = piece_list[blockIdx.x];
    const int r = code >> 3, s = code & 7;
    const RingDesc rd = rings[r];
    const int N = rd.N, Q = ring_pieces(rd), Lq = N / Q;
    const bool split = rd.mode == kSplit4;
    const bool shifted = rd.phi0 != 0.0;
    constexpr int nchan = SPIN ? 2 : 1;
    const double *inQ = maps_all + (size_t)blockIdx.y * nchan * npix + rd.start;
    const double *inU = inQ + npix;
    double2 *Vp = V_all + ((size_t)blockIdx.y * nchan * nrings + r) * M;
    double2 *Vm = SPIN ? Vp + (size_t)nrings * M : Vp;
    const int bd = blockDim.x;
    if (!split && Q == 2) {
        // the belt's two-piece rings: 2 kUP values of j1 per thread and round (all loads first),
        // twiddles from the shared table
        constexpr int U = 2 * kUP;
        const double sg = (s & 1) ? -1.0 : 1.0;  // e^{-2 pi i s j2 / 2} = (-1)^(s j2)
        for (int j10 = threadIdx.x; j10 < Lq; j10 += U * bd) {
            double2 a0[U], a1[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = j10 + u * bd;
                const bool ok = j < Lq && JHTB_IN(rd.start + j + Lq, npix, 103);
                a0[u] = ok ? make_double2(inQ[j], SPIN ? inU[j] : 0.0) : make_double2(0.0, 0.0);
                a1[u] = ok ? make_double2(inQ[j + Lq], SPIN ? inU[j + Lq] : 0.0) : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j1 = j10 + u * bd;
                if (j1 >= Lq) continue;
                const double2 v = cmul(make_double2(fma(sg, a1[u].x, a0[u].x), fma(sg, a1[u].y, a0[u].y)),
                                       sm_tw_pi(T, -2LL * s * j1, N));
                if (JHTB_IN(pidx(j1), kFftBufLen, 106)) buf[pidx(j1)] = v;
            }
        }
    }
    // b_s[j1]: the Q pixels j1 + Lq j2 with e^{-2 pi i s j / N}
    for (int j10 = threadIdx.x; j10 < Lq && (split || Q != 2); j10 += kUP * bd) {
        double2 acc[kUP];
#pragma unroll
        for (int u = 0; u < kUP; ++u) acc[u] = make_double2(0.0, 0.0);
        double2 a[kMaxPieces][kUP], w1[kUP];  // every load issued before the first is used
#pragma unroll
        for (int j2 = 0; j2 < kMaxPieces; ++j2)
#pragma unroll
            for (int u = 0; u < kUP; ++u) {
                const int j = j10 + u * bd + Lq * j2;
                a[j2][u] = (j2 < Q && j10 + u * bd < Lq && JHTB_IN(rd.start + j, npix, 103)) ? make_double2(inQ[j], SPIN ? inU[j] : 0.0)
                                                                                            : make_double2(0.0, 0.0);
            }
#pragma unroll
        for (int u = 0; u < kUP; ++u) {
            const int j1 = j10 + u * bd;
            w1[u] = (!split && j1 < Lq) ? tw_pi(tw, -2LL * s * j1, N) : make_double2(1.0, 0.0);
        }
        // e^{-2 pi i s (j1 + Lq j2) / N} = e^{-2 pi i s j1 / N} e^{-2 pi i s j2 / Q}: the j2 factor
        // is a fourth root of unity (exact), the j1 factor is applied once
#pragma unroll
        for (int j2 = 0; j2 < kMaxPieces; ++j2) {
            if (j2 >= Q) break;
            const double2 w = root8(-(8 / Q) * s * j2);
#pragma unroll
            for (int u = 0; u < kUP; ++u) acc[u] = cadd(acc[u], j2 ? cmul(a[j2][u], w) : a[j2][u]);
        }
#pragma unroll
        for (int u = 0; u < kUP; ++u) {
            const int j1 = j10 + u * bd;
            if (j1 >= Lq) continue;
            // power of two: e^{-2 pi i s j1 / N} from the table; kSplit4: times the chirp
            // conj(w(j1)) = e^{-i pi 4 j1^2 / N}, one exactly reduced argument
            const double2 v = split ? cmul(acc[u], cis_pi(-(int)(((long long)2 * s * j1 + 4LL * j1 * j1) % (2LL * N)), N, 0, 1))
                                    : cmul(acc[u], w1[u]);
            if (JHTB_IN(pidx(j1), kFftBufLen, 106)) buf[pidx(j1)] = v;
        }
    }
    const int L = split ? rd.P : Lq;
    for (int k = Lq + threadIdx.x; k < L; k += bd) buf[pidx(k)] = make_double2(0.0, 0.0);
    __syncthreads();
    fft_stockham_sm(buf, L, -1.0, T);
    if (split) {  // W[k] = conj(w(k)) sum_j (b[j] conj(w(j))) w(k - j)
        for (int q0 = threadIdx.x; q0 < L; q0 += kUP * bd) {
            double2 w[kUP];
#pragma unroll
            for (int u = 0; u < kUP; ++u) w[u] = q0 + u * bd < L ? bh_get(bh + rd.bh_off, L, q0 + u * bd, -1) : make_double2(0.0, 0.0);
#pragma unroll
            for (int u = 0; u < kUP; ++u)
                if (q0 + u * bd < L) buf[pidx(q0 + u * bd)] = cmul(buf[pidx(q0 + u * bd)], w[u]);
        }
        __syncthreads();
        fft_stockham_sm(buf, L, +1.0, T);
        for (int k = threadIdx.x; k < Lq; k += bd)
            buf[pidx(k)] = cmul(buf[pidx(k)], cis_pi(-(int)(((long long)k * k) % (2 * Lq)), Lq, 0, 1));
        __syncthreads();
    }
    // V rows: Vp[m] = W[m mod N] for m = s (mod Q), Vm[m] = conj(W[-m mod N]) for m = -s (mod Q),
    // both times e^{-i m phi0} (gather_adjoint, restricted to this piece's residue class)
    const int sm = (Q - s) % Q;
    for (int m0 = threadIdx.x * Q; m0 <= lmax; m0 += kUP * bd * Q) {
#pragma unroll
        for (int u = 0; u < kUP; ++u) {
            const int mp = m0 + u * bd * Q + s;  // Vp orders
            if (mp <= lmax) {
                const int kp = (mp % N - s) / Q;
                double2 p = JHTB_IN(kp, Lq, 106) ? buf[pidx(kp)] : make_double2(0.0, 0.0);
                if (shifted) p = cmul(p, split ? cis_pi(-(mp % (2 * N)), N, 0, 1) : tw_pi(tw, -(long long)mp, N));
                if (JHTB_IN(mp, M, 105)) Vp[mp] = p;
            }
            if (SPIN) {
                const int mm = m0 + u * bd * Q + sm;  // Vm orders
                if (mm <= lmax) {
                    const int k = (N - mm % N) % N;
                    const int kq = (k - s) / Q;
                    double2 q = JHTB_IN(kq, Lq, 106) ? conjd(buf[pidx(kq)]) : make_double2(0.0, 0.0);
                    if (shifted) q = cmul(q, split ? cis_pi(-(mm % (2 * N)), N, 0, 1) : tw_pi(tw, -(long long)mm, N));
                    if (JHTB_IN(mm, M, 105)) Vm[mm] = q;
                }
            }
        }
    }
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
int smem_bytes_piece() { return (kFftBufLen + kSmTwLen) * (int)sizeof(double2); }

template <typename K>
int ensure_smem(K kernel, int bytes = smem_bytes()) {
    JHTB_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return JHTB_OK;
}

template <int SPIN>
int launch_ring_synth_t(const Plan &p, const double2 *F, double *maps, int nb, cudaStream_t s) {
    int rc;
    if (p.nring_small > 0) {
        if ((rc = ensure_smem(ring_synth_kernel<SPIN>))) return rc;
        ring_synth_kernel<SPIN><<<dim3(p.nring_small, nb), kFftThreads, smem_bytes(), s>>>(
            p.d_ring_small, p.d_rings, p.lmax, p.M, p.nrings, p.npix, F, maps, p.d_W, p.d_W2, p.d_tw, p.d_bh);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    if (p.nring_piece > 0) {
        if ((rc = ensure_smem(ring_synth_piece_kernel<SPIN>, smem_bytes_piece()))) return rc;
        ring_synth_piece_kernel<SPIN><<<dim3(p.nring_piece, nb), kFftThreads, smem_bytes_piece(), s>>>(
            p.d_ring_piece, p.d_rings, p.lmax, p.M, p.nrings, p.npix, F, maps, p.d_tw, p.d_bh);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    return JHTB_OK;
}

template <int SPIN>
int launch_ring_adjoint_t(const Plan &p, const double *maps, double2 *V, double2 *W, int nb, cudaStream_t s) {
    int rc;
    if (p.nring_small > 0) {
        if ((rc = ensure_smem(ring_adjoint_kernel<SPIN>))) return rc;
        ring_adjoint_kernel<SPIN><<<dim3(p.nring_small, nb), kFftThreads, smem_bytes(), s>>>(
            p.d_ring_small, p.d_rings, p.lmax, p.M, p.nrings, p.npix, maps, V, p.d_W2, W, p.d_tw, p.d_bh);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    if (p.nring_piece > 0) {
        if ((rc = ensure_smem(ring_adjoint_piece_kernel<SPIN>, smem_bytes_piece()))) return rc;
        ring_adjoint_piece_kernel<SPIN><<<dim3(p.nring_piece, nb), kFftThreads, smem_bytes_piece(), s>>>(
            p.d_ring_piece, p.d_rings, p.lmax, p.M, p.nrings, p.npix, maps, V, p.d_tw, p.d_bh);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    return JHTB_OK;
}

}  // namespace

JHTB_DEBUG_ACCESSOR(ringfft)

int launch_ring_synth(const Plan &p, const double2 *F, double *maps, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    return p.spin ? launch_ring_synth_t<2>(p, F, maps, nb, s) : launch_ring_synth_t<0>(p, F, maps, nb, s);
}

int launch_ring_adjoint(const Plan &p, const double *maps, double2 *V, double2 *W, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    return p.spin ? launch_ring_adjoint_t<2>(p, maps, V, W, nb, s) : launch_ring_adjoint_t<0>(p, maps, V, W, nb, s);
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
