// Batched complex FP64 FFTs of 2,3,5-smooth lengths (sm_100a): the off-grid transforms'
// theta FFT and the FFTs of the oversampled torus grid (jht _nufft.py:164-191 runs them as
// jnp.fft inside XLA).
//
// One CTA of kFftSmThreads threads per transform (a grid-stride loop over the batch): the
// transform is gathered into shared memory in mixed-radix digit-reversed order, runs one
// in-place decimation-in-time stage per factor of its length (radices 4, 2, 3, 5; each
// butterfly writes back where it read, so a thread holds one butterfly at a time), and is
// written back in natural order, optionally scaled and multiplied by a four-step twiddle.  Lengths up to kFftSmMax run in
// one CTA; the host composes longer ones from two batched calls (four-step).  Every
// butterfly's root comes from the caller's table of the n-th roots of unity (or, without a
// table, from one sincospi of an exactly reduced rational argument).
//
// Batch index b = outer * inner_count + t: the transform reads in[o * in_dist_outer +
// t * in_dist_inner + i * in_stride] for i < n and writes out[...] likewise with the out
// strides, so row, column and four-step transforms of a row-major array are all one call.
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kFftSmThreads = 1024;
constexpr int kFftSmMax = 10240;  // longest transform held in shared memory (160 KB)

struct FftArgs {
    const double2 *in;
    double2 *out;
    int n;
    int c4, c2, c3, c5;  // passes of each radix, in this order (n = 4^c4 2^c2 3^c3 5^c5)
    long long howmany, inner;
    long long in_stride, in_dist_outer, in_dist_inner;
    long long out_stride, out_dist_outer, out_dist_inner;
    int sign;
    double scale;
    long long tw_n;  // 0: none; else output k of inner index t times e^{sign 2 pi i (t k mod tw_n) / tw_n}
    const double2 *roots;  // e^{-2 pi i k / n} for k < n, or null (each butterfly's root by sincospi)
};

__device__ __forceinline__ double2 f_cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 f_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 f_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// i * sgn * a
__device__ __forceinline__ double2 f_isgn(double2 a, double sgn) { return make_double2(-sgn * a.y, sgn * a.x); }

// e^{sgn 2 pi i a / b} for integers 0 <= a < b.
__device__ __forceinline__ double2 f_root(long long a, long long b, double sgn) {
    double s, c;
    sincospi(sgn * 2.0 * (double)a / (double)b, &s, &c);
    return make_double2(c, s);
}

// R-point DFT in registers, sign sgn: X_k = sum_j x_j e^{sgn 2 pi i j k / R}.
template <int R>
__device__ __forceinline__ void small_dft(double2 (&v)[R], double sgn);
template <>
__device__ __forceinline__ void small_dft<2>(double2 (&v)[2], double) {
    const double2 a = v[0], b = v[1];
    v[0] = f_add(a, b);
    v[1] = f_sub(a, b);
}
template <>
__device__ __forceinline__ void small_dft<4>(double2 (&v)[4], double sgn) {
    const double2 a = f_add(v[0], v[2]), b = f_sub(v[0], v[2]);
    const double2 c = f_add(v[1], v[3]), d = f_isgn(f_sub(v[1], v[3]), sgn);
    v[0] = f_add(a, c);
    v[2] = f_sub(a, c);
    v[1] = f_add(b, d);
    v[3] = f_sub(b, d);
}
template <>
__device__ __forceinline__ void small_dft<3>(double2 (&v)[3], double sgn) {
    constexpr double s3 = 0.86602540378443864676;  // sin(2 pi / 3)
    const double2 t1 = f_add(v[1], v[2]);
    const double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
    const double2 d = f_sub(v[1], v[2]);
    const double2 t3 = f_isgn(make_double2(s3 * d.x, s3 * d.y), sgn);
    v[0] = f_add(v[0], t1);
    v[1] = f_add(t2, t3);
    v[2] = f_sub(t2, t3);
}
template <>
__device__ __forceinline__ void small_dft<5>(double2 (&v)[5], double sgn) {
    constexpr double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;  // cos(2 pi / 5), cos(4 pi / 5)
    constexpr double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;   // sin(2 pi / 5), sin(4 pi / 5)
    const double2 a1 = f_add(v[1], v[4]), b1 = f_sub(v[1], v[4]);
    const double2 a2 = f_add(v[2], v[3]), b2 = f_sub(v[2], v[3]);
    const double2 x0 = v[0];
    const double2 r1 = make_double2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    const double2 r2 = make_double2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    const double2 i1 = f_isgn(make_double2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), sgn);
    const double2 i2 = f_isgn(make_double2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), sgn);
    v[0] = make_double2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = f_add(r1, i1);
    v[4] = f_sub(r1, i1);
    v[2] = f_add(r2, i2);
    v[3] = f_sub(r2, i2);
}

// One in-place decimation-in-time stage of radix R over n points that hold sub-transforms
// of length m (natural order within each): butterfly (g, j), g a multiple of L = m R and
// j < m, combines the R elements g + j + q m (q < R) after twiddling element q by
// w^q, w = e^{sgn 2 pi i j / L} (one table entry per butterfly, its powers by multiplication),
// and stores them back in place, so a thread holds only R values at a time.
template <int R>
__device__ __forceinline__ void dit_stage(double2 *buf, int n, int m, double sgn, const double2 *__restrict__ roots) {
    const int L = m * R, nb = n / R;
    const int rstep = n / L;  // e^{-2 pi i j / L} = roots[j n / L]
    for (int bi = threadIdx.x; bi < nb; bi += kFftSmThreads) {
        const int gq = bi / m, j = bi - gq * m;
        const int base = gq * L + j;
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = buf[base + q * m];
        if (m > 1) {
            double2 w;
            if (roots) {
                w = __ldg(&roots[j * rstep]);
                w.y *= -sgn;  // the table holds e^{-2 pi i k / n}
            } else {
                w = f_root(j, L, sgn);
            }
            double2 wq = w;
#pragma unroll
            for (int q = 1; q < R; ++q) {
                v[q] = f_cmul(v[q], wq);
                if (q + 1 < R) wq = f_cmul(wq, w);
            }
        }
        small_dft<R>(v, sgn);
#pragma unroll
        for (int q = 0; q < R; ++q) buf[base + q * m] = v[q];
    }
    __syncthreads();
}

// Position of input element i after the mixed-radix digit reversal of the stage order
// (radix 4 stages first, then 2, 3 and 5): the last stage's radix is the least significant
// digit of i, and it selects the block of length n / R_last the element lands in.
__device__ __forceinline__ int digit_reversed(int i, int n, int c4, int c2, int c3, int c5) {
    int pos = 0, span = n;
    for (int p = 0; p < c5; ++p) { span /= 5; pos += (i % 5) * span; i /= 5; }
    for (int p = 0; p < c3; ++p) { span /= 3; pos += (i % 3) * span; i /= 3; }
    for (int p = 0; p < c2; ++p) { span /= 2; pos += (i % 2) * span; i /= 2; }
    for (int p = 0; p < c4; ++p) { span /= 4; pos += (i % 4) * span; i /= 4; }
    return pos;
}

__global__ void __launch_bounds__(kFftSmThreads, 1) fft_smooth_kernel(FftArgs a) {
    extern __shared__ double2 fbuf[];
    const int n = a.n;
    const double sgn = a.sign > 0 ? 1.0 : -1.0;
    for (long long b = blockIdx.x; b < a.howmany; b += gridDim.x) {
        const long long o = b / a.inner, t = b - o * a.inner;
        const double2 *src = a.in + o * a.in_dist_outer + t * a.in_dist_inner;
        for (int i = threadIdx.x; i < n; i += kFftSmThreads)
            fbuf[digit_reversed(i, n, a.c4, a.c2, a.c3, a.c5)] = src[(long long)i * a.in_stride];
        __syncthreads();
        int m = 1;
        for (int p = 0; p < a.c4; ++p, m *= 4) dit_stage<4>(fbuf, n, m, sgn, a.roots);
        for (int p = 0; p < a.c2; ++p, m *= 2) dit_stage<2>(fbuf, n, m, sgn, a.roots);
        for (int p = 0; p < a.c3; ++p, m *= 3) dit_stage<3>(fbuf, n, m, sgn, a.roots);
        for (int p = 0; p < a.c5; ++p, m *= 5) dit_stage<5>(fbuf, n, m, sgn, a.roots);
        double2 *dst = a.out + o * a.out_dist_outer + t * a.out_dist_inner;
        for (int k = threadIdx.x; k < n; k += kFftSmThreads) {
            double2 v = fbuf[k];
            v.x *= a.scale;
            v.y *= a.scale;
            if (a.tw_n) v = f_cmul(v, f_root((t * (long long)k) % a.tw_n, a.tw_n, sgn));
            dst[(long long)k * a.out_stride] = v;
        }
        __syncthreads();  // the next transform reuses the buffer
    }
}

}  // namespace
}  // namespace jhtb

using namespace jhtb;

extern "C" int jhtb_fft_c2c(const void *in, void *out, int n, int64_t howmany, int64_t inner, int64_t in_stride,
                            int64_t in_dist_outer, int64_t in_dist_inner, int64_t out_stride, int64_t out_dist_outer,
                            int64_t out_dist_inner, int sign, double scale, int64_t twiddle_n, const void *roots,
                            void *stream) {
    if (!in || !out) return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: NULL argument");
    if (n < 1 || n > kFftSmMax)
        return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: n must be in [1, " + std::to_string(kFftSmMax) + "], got " +
                                          std::to_string(n));
    if (howmany < 0 || inner < 1) return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: howmany must be >= 0 and inner >= 1");
    if (sign != 1 && sign != -1) return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: sign must be +1 or -1");
    if (twiddle_n < 0) return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: twiddle_n must be >= 0");
    if (in == out && (in_stride != out_stride || in_dist_outer != out_dist_outer || in_dist_inner != out_dist_inner))
        return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: an in-place call needs the same input and output layout");
    FftArgs a{};
    a.in = (const double2 *)in;
    a.out = (double2 *)out;
    a.n = n;
    int r = n;
    while (r % 4 == 0) ++a.c4, r /= 4;
    while (r % 2 == 0) ++a.c2, r /= 2;
    while (r % 3 == 0) ++a.c3, r /= 3;
    while (r % 5 == 0) ++a.c5, r /= 5;
    if (r != 1) return fail(JHTB_ERR_INVALID, "jhtb_fft_c2c: n must be 2,3,5-smooth, got " + std::to_string(n));
    a.howmany = howmany;
    a.inner = inner;
    a.in_stride = in_stride;
    a.in_dist_outer = in_dist_outer;
    a.in_dist_inner = in_dist_inner;
    a.out_stride = out_stride;
    a.out_dist_outer = out_dist_outer;
    a.out_dist_inner = out_dist_inner;
    a.sign = sign;
    a.scale = scale;
    a.tw_n = twiddle_n;
    a.roots = (const double2 *)roots;
    if (howmany == 0) return JHTB_OK;
    const int smem = n * (int)sizeof(double2);
    JHTB_CUDA_TRY(cudaFuncSetAttribute(fft_smooth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int dev = 0, nsm = 148;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long grid = std::min<long long>(howmany, 8LL * nsm);
    fft_smooth_kernel<<<(unsigned)grid, kFftSmThreads, smem, (cudaStream_t)stream>>>(a);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}
