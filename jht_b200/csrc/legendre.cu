// Fused Legendre / Wigner-d recursion + l-contraction, FP64 (sm_100a).
//
// Synthesis (jht _recursion.py:441-469 spin 0, :512-543 spin 2) and its exact
// transpose (:472-497, :546-572).  For each order m and half-grid ring t the
// recursion runs over l = lmin..lmax entirely in registers; no lambda table is
// stored.  One CTA owns the m-pair (m, lmax - m) (equal work: lmax + 2 steps) and
// sweeps the 2 nside half-grid rings in tiles of NT*R rings, R rings per thread.
//
// Numerics.  jht carries lambda as (mantissa, log-scale) renormalised every step
// (_recursion.py:352-369: one sqrt, log, exp and two divisions per step).  Here
// the recursion is rewritten with per-(l,m) normalised coefficients (plan.cu):
//     mu_l = (alpha_l x + gamma_l) mu_{l-1} - mu_{l-2},   lambda_l = c_l mu_l,
// two FMAs per step, and underflow is handled with an integer scale
// (value = mu * 2^(800 sc)).  While sc < 0 the value is < 2^-400 and is not
// accumulated; the rescale check runs only in that phase, which a warp leaves as
// soon as all its rings reach sc = 0 (then the loop is branch-free).
//
// Parity.  Step i = l - lmin alternates between accumulator slots A (i even) and
// B (i odd); N/S outputs are A +- B, which realises jht's total / signed sums
// without per-step signs.
#include <cuda_runtime.h>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kChunk = 64;  // recursion steps staged in shared memory per round (even)
constexpr unsigned kFull = 0xffffffffu;

struct LegParams {
    int lmax, T, nrings, M, nside;
    long long K;
    const double *x, *logsin, *logch, *logsh;
    const SeedParam *seed;
    const double *alpha, *gamma, *cnorm;
};

LegParams make_params(const Plan &p) {
    LegParams q;
    q.lmax = p.lmax;
    q.T = p.T;
    q.nrings = p.nrings;
    q.M = p.M;
    q.nside = p.nside;
    q.K = p.K;
    q.x = p.d_x;
    q.logsin = p.d_logsin;
    q.logch = p.d_logch;
    q.logsh = p.d_logsh;
    q.seed = p.d_seed;
    q.alpha = p.d_alpha;
    q.gamma = p.d_gamma;
    q.cnorm = p.d_cnorm;
    return q;
}

// sign * exp(lg) as mant * 2^(800 sc) with |mant| in [2^-400, 2^400), sc <= 0.
// The reduction lg - sc * 800 ln2 uses a two-part constant so it adds no error.
__device__ __forceinline__ void make_seed(double lg, double sign, double &mant, int &sc) {
    if (!(lg > -1.0e300)) {  // log(0): exact zero at a pole
        mant = 0.0;
        sc = 0;
        return;
    }
    int k = (int)floor((lg + kLn2x400) / (kLogScaleHi + kLogScaleLo));
    if (k > 0) k = 0;
    const double dk = (double)k;
    const double r = __dadd_rn(__dadd_rn(lg, -__dmul_rn(dk, kLogScaleHi)), -__dmul_rn(dk, kLogScaleLo));
    mant = sign * exp(r);
    sc = k;
}

// log|seed| for ring t: spin 0 (_recursion.py:315-317), spin +-2 (:181-187).
// Unfused mul/add so the value is rounded exactly as jht's NumPy plan rounds it.
__device__ __forceinline__ double seed_log0(const SeedParam &sp, int m, double logsin) {
    return m == 0 ? sp.lf[0] : __dadd_rn(sp.lf[0], __dmul_rn((double)m, logsin));
}
__device__ __forceinline__ double seed_log2(const SeedParam &sp, int h, double lch, double lsh) {
    double v = sp.lf[h];
    if (sp.pc[h] > 0) v = __dadd_rn(v, __dmul_rn((double)sp.pc[h], lch));
    if (sp.ps[h] > 0) v = __dadd_rn(v, __dmul_rn((double)sp.ps[h], lsh));
    return v;
}

// One scaled-phase bookkeeping step: returns the new value and updates prev/sc.
__device__ __forceinline__ void rescale(double &u, double &prev, int &sc) {
    if (sc < 0 && fabs(u) > kBig) {
        u *= kScaleDown;
        prev *= kScaleDown;
        sc += 1;
    }
}

// =====================================================================================
// synthesis, spin 0
// =====================================================================================
template <int R, bool SLOW>
__device__ __forceinline__ void synth0_step(double al, double2 c, const double (&x)[R], double (&u1)[R],
                                            double (&u2)[R], int (&sc)[R], double (&ar)[R], double (&ai)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        double u = fma(al * x[k], u1[k], -u2[k]);
        double prev = u1[k];
        if (SLOW) rescale(u, prev, sc[k]);
        u2[k] = prev;
        u1[k] = u;
        if (!SLOW || sc[k] == 0) {
            ar[k] = fma(c.x, u, ar[k]);
            ai[k] = fma(c.y, u, ai[k]);
        }
    }
}

template <int R, bool SLOW>
__device__ __forceinline__ void synth0_chunk(int cnt, const double *s_al, const double2 *s_c,
                                             const double (&x)[R], double (&u1)[R], double (&u2)[R],
                                             int (&sc)[R], double (&Ar)[R], double (&Ai)[R], double (&Br)[R],
                                             double (&Bi)[R]) {
    int q = 0;
    for (; q + 1 < cnt; q += 2) {
        synth0_step<R, SLOW>(s_al[q], s_c[q], x, u1, u2, sc, Ar, Ai);
        synth0_step<R, SLOW>(s_al[q + 1], s_c[q + 1], x, u1, u2, sc, Br, Bi);
    }
    if (q < cnt) synth0_step<R, SLOW>(s_al[q], s_c[q], x, u1, u2, sc, Ar, Ai);
}

template <int R, int NT>
__global__ void __launch_bounds__(NT) synth0_kernel(LegParams p, const double2 *__restrict__ alm_all,
                                                     double2 *__restrict__ F_all) {
    __shared__ double s_al[kChunk];
    __shared__ double2 s_c[kChunk];
    const int tid = threadIdx.x;
    const int L = p.lmax;
    const double2 *alm = alm_all + (size_t)blockIdx.y * p.K;
    double2 *F = F_all + (size_t)blockIdx.y * p.nrings * p.M;
    const int j = blockIdx.x;
    for (int pass = 0; pass < 2; ++pass) {
        const int m = pass ? L - j : j;
        if (pass && m <= j) break;
        const SeedParam sp = p.seed[m];
        const long long b0 = alm_index(sp.lmin, m, L);
        const int nst = L - sp.lmin + 1;
        for (int tile = 0; tile < p.T; tile += NT * R) {
            double x[R], u1[R], u2[R], Ar[R], Ai[R], Br[R], Bi[R];
            int sc[R];
            bool fast = true;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                double mant = 0.0, xx = 0.0;
                int s = 0;
                if (t < p.T) {
                    xx = p.x[t];
                    make_seed(seed_log0(sp, m, p.logsin[t]), sp.sign[0], mant, s);
                }
                // (u1, u2) = (0, -seed): the first generic step (alpha = 0) yields the seed.
                x[k] = xx;
                u1[k] = 0.0;
                u2[k] = -mant;
                sc[k] = s;
                fast &= (s == 0);
                Ar[k] = Ai[k] = Br[k] = Bi[k] = 0.0;
            }
            for (int i0 = 0; i0 < nst; i0 += kChunk) {
                const int cnt = min(kChunk, nst - i0);
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    const long long idx = b0 + i0 + q;
                    const double c = p.cnorm[idx];
                    const double2 a = alm[idx];
                    s_al[q] = p.alpha[idx];
                    s_c[q] = make_double2(a.x * c, a.y * c);
                }
                __syncthreads();
                if (__all_sync(kFull, fast)) {
                    synth0_chunk<R, false>(cnt, s_al, s_c, x, u1, u2, sc, Ar, Ai, Br, Bi);
                } else {
                    synth0_chunk<R, true>(cnt, s_al, s_c, x, u1, u2, sc, Ar, Ai, Br, Bi);
                    fast = true;
#pragma unroll
                    for (int k = 0; k < R; ++k) fast &= (sc[k] == 0);
                }
            }
            // F_north = A + B; F_south = (-1)^m (E - O) = A - B   (healpix.py:250-253)
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                if (t < p.T) {
                    F[(size_t)t * p.M + m] = make_double2(Ar[k] + Br[k], Ai[k] + Bi[k]);
                    if (t < p.T - 1)
                        F[(size_t)(4 * p.nside - 2 - t) * p.M + m] = make_double2(Ar[k] - Br[k], Ai[k] - Bi[k]);
                }
            }
        }
    }
}

// =====================================================================================
// synthesis, spin 2: the d^{+2} and d^{-2} recursions advanced together
// =====================================================================================
struct Acc2 {
    double ppr, ppi, pmr, pmi, mmr, mmi, mpr, mpi;
};

template <int R, bool SLOW, int SGN>
__device__ __forceinline__ void synth2_step(double al, double ga, double2 cp, double2 cm, const double (&x)[R],
                                            double (&p1)[R], double (&p2)[R], int (&sp)[R], double (&m1)[R],
                                            double (&m2)[R], int (&sm)[R], Acc2 (&acc)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const double tp = fma(al, x[k], ga);
        const double tm = fma(al, x[k], -ga);
        double up = fma(tp, p1[k], -p2[k]);
        double um = fma(tm, m1[k], -m2[k]);
        double pp = p1[k], pm = m1[k];
        if (SLOW) {
            rescale(up, pp, sp[k]);
            rescale(um, pm, sm[k]);
        }
        p2[k] = pp;
        p1[k] = up;
        m2[k] = pm;
        m1[k] = um;
        if (SLOW) {
            if (sp[k] != 0) up = 0.0;
            if (sm[k] != 0) um = 0.0;
        }
        Acc2 &a = acc[k];
        a.ppr = fma(cp.x, up, a.ppr);
        a.ppi = fma(cp.y, up, a.ppi);
        a.mmr = fma(cm.x, um, a.mmr);
        a.mmi = fma(cm.y, um, a.mmi);
        a.pmr = fma(SGN * cp.x, um, a.pmr);
        a.pmi = fma(SGN * cp.y, um, a.pmi);
        a.mpr = fma(SGN * cm.x, up, a.mpr);
        a.mpi = fma(SGN * cm.y, up, a.mpi);
    }
}

template <int R, bool SLOW>
__device__ __forceinline__ void synth2_chunk(int cnt, const double *s_al, const double *s_ga, const double2 *s_cp,
                                             const double2 *s_cm, const double (&x)[R], double (&p1)[R],
                                             double (&p2)[R], int (&sp)[R], double (&m1)[R], double (&m2)[R],
                                             int (&sm)[R], Acc2 (&acc)[R]) {
    int q = 0;
    for (; q + 1 < cnt; q += 2) {
        synth2_step<R, SLOW, 1>(s_al[q], s_ga[q], s_cp[q], s_cm[q], x, p1, p2, sp, m1, m2, sm, acc);
        synth2_step<R, SLOW, -1>(s_al[q + 1], s_ga[q + 1], s_cp[q + 1], s_cm[q + 1], x, p1, p2, sp, m1, m2, sm, acc);
    }
    if (q < cnt) synth2_step<R, SLOW, 1>(s_al[q], s_ga[q], s_cp[q], s_cm[q], x, p1, p2, sp, m1, m2, sm, acc);
}

template <int R, int NT>
__global__ void __launch_bounds__(NT) synth2_kernel(LegParams p, const double2 *__restrict__ alm_all,
                                                     double2 *__restrict__ F_all) {
    __shared__ double s_al[kChunk], s_ga[kChunk];
    __shared__ double2 s_cp[kChunk], s_cm[kChunk];
    const int tid = threadIdx.x;
    const int L = p.lmax;
    const double2 *aE = alm_all + (size_t)blockIdx.y * 2 * p.K;
    const double2 *aB = aE + p.K;
    double2 *Fp = F_all + (size_t)blockIdx.y * 2 * p.nrings * p.M;
    double2 *Fm = Fp + (size_t)p.nrings * p.M;
    const int j = blockIdx.x;
    for (int pass = 0; pass < 2; ++pass) {
        const int m = pass ? L - j : j;
        if (pass && m <= j) break;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        // south sign (-1)^(m + lmin): the signed sums are relative to l = lmin
        const double ssign = ((m + sd.lmin) & 1) ? -1.0 : 1.0;
        for (int tile = 0; tile < p.T; tile += NT * R) {
            double x[R], p1[R], p2[R], m1[R], m2[R];
            int sp[R], sm[R];
            Acc2 acc[R];
            bool fast = true;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                double mp = 0.0, mm = 0.0, xx = 0.0;
                int s1 = 0, s2 = 0;
                if (t < p.T) {
                    xx = p.x[t];
                    const double lch = p.logch[t], lsh = p.logsh[t];
                    make_seed(seed_log2(sd, 0, lch, lsh), sd.sign[0], mp, s1);
                    make_seed(seed_log2(sd, 1, lch, lsh), sd.sign[1], mm, s2);
                }
                x[k] = xx;
                p1[k] = 0.0;
                p2[k] = -mp;
                sp[k] = s1;
                m1[k] = 0.0;
                m2[k] = -mm;
                sm[k] = s2;
                fast &= (s1 == 0) && (s2 == 0);
                acc[k] = Acc2{0, 0, 0, 0, 0, 0, 0, 0};
            }
            for (int i0 = 0; i0 < nst; i0 += kChunk) {
                const int cnt = min(kChunk, nst - i0);
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    const long long idx = b0 + i0 + q;
                    const double c = p.cnorm[idx];
                    const double2 e = aE[idx], b = aB[idx];
                    s_al[q] = p.alpha[idx];
                    s_ga[q] = p.gamma[idx];
                    // cp = -(aE + i aB) c, cm = -(aE - i aB) c   (healpix.py:316-318)
                    s_cp[q] = make_double2(-(e.x - b.y) * c, -(e.y + b.x) * c);
                    s_cm[q] = make_double2(-(e.x + b.y) * c, -(e.y - b.x) * c);
                }
                __syncthreads();
                if (__all_sync(kFull, fast)) {
                    synth2_chunk<R, false>(cnt, s_al, s_ga, s_cp, s_cm, x, p1, p2, sp, m1, m2, sm, acc);
                } else {
                    synth2_chunk<R, true>(cnt, s_al, s_ga, s_cp, s_cm, x, p1, p2, sp, m1, m2, sm, acc);
                    fast = true;
#pragma unroll
                    for (int k = 0; k < R; ++k) fast &= (sp[k] == 0) && (sm[k] == 0);
                }
            }
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                if (t < p.T) {
                    const Acc2 &a = acc[k];
                    Fp[(size_t)t * p.M + m] = make_double2(a.ppr, a.ppi);
                    Fm[(size_t)t * p.M + m] = make_double2(a.mmr, a.mmi);
                    if (t < p.T - 1) {
                        const size_t rs = (size_t)(4 * p.nside - 2 - t) * p.M + m;
                        Fp[rs] = make_double2(ssign * a.pmr, ssign * a.pmi);
                        Fm[rs] = make_double2(ssign * a.mpr, ssign * a.mpi);
                    }
                }
            }
        }
    }
}

// =====================================================================================
// adjoint: per-step partial sums over the thread's rings, reduced across the warp
// (butterfly reduce-scatter), across warps (shared memory, fixed order) and across
// ring tiles (accumulated in the output by the owning CTA) -- deterministic.
// =====================================================================================
constexpr int kSub = 8;  // steps per warp reduction

// After the call, lane l holds in v[0] the warp total of entry idx(l) where, for
// NV = 8: idx = ((l>>4)&1)*4 + ((l>>3)&1)*2 + ((l>>2)&1); for NV = 16 one more bit.
template <int NV>
__device__ __forceinline__ void warp_reduce_scatter(double2 (&v)[NV], int lane) {
    int mask = 16;
#pragma unroll
    for (int half = NV / 2; half >= 1; half /= 2, mask >>= 1) {
        const bool up = lane & mask;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double2 send = up ? v[i] : v[i + half];
            const double2 keep = up ? v[i + half] : v[i];
            const double rx = __shfl_xor_sync(kFull, send.x, mask);
            const double ry = __shfl_xor_sync(kFull, send.y, mask);
            v[i] = make_double2(keep.x + rx, keep.y + ry);
        }
    }
    for (; mask >= 1; mask >>= 1) {
        v[0].x += __shfl_xor_sync(kFull, v[0].x, mask);
        v[0].y += __shfl_xor_sync(kFull, v[0].y, mask);
    }
}

template <int NV>
__device__ __forceinline__ int scatter_index(int lane) {
    int idx = 0, bit = NV / 2;
    for (int mask = 16; bit >= 1; mask >>= 1, bit >>= 1)
        if (lane & mask) idx += bit;
    return idx;
}

template <int NV>
__device__ __forceinline__ bool scatter_writer(int lane) {
    // lanes whose bits below the scatter bits are zero
    constexpr int used = NV == 8 ? 3 : (NV == 16 ? 4 : 5);
    return (lane & ((1 << (5 - used)) - 1)) == 0;
}

// ---------------- spin 0 ----------------
template <int R, bool SLOW>
__device__ __forceinline__ double2 adj0_step(double al, const double (&x)[R], double (&u1)[R], double (&u2)[R],
                                             int (&sc)[R], const double2 (&U)[R]) {
    double2 part = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        double u = fma(al * x[k], u1[k], -u2[k]);
        double prev = u1[k];
        if (SLOW) rescale(u, prev, sc[k]);
        u2[k] = prev;
        u1[k] = u;
        if (SLOW && sc[k] != 0) u = 0.0;
        part.x = fma(u, U[k].x, part.x);
        part.y = fma(u, U[k].y, part.y);
    }
    return part;
}

template <int R, bool SLOW>
__device__ __forceinline__ void adj0_sub(int cnt, const double *s_al, const double (&x)[R], double (&u1)[R],
                                         double (&u2)[R], int (&sc)[R], const double2 (&UA)[R],
                                         const double2 (&UB)[R], double2 (&part)[kSub]) {
#pragma unroll
    for (int q = 0; q < kSub; q += 2) {
        if (q < cnt) part[q] = adj0_step<R, SLOW>(s_al[q], x, u1, u2, sc, UA);
        else part[q] = make_double2(0.0, 0.0);
        if (q + 1 < cnt) part[q + 1] = adj0_step<R, SLOW>(s_al[q + 1], x, u1, u2, sc, UB);
        else part[q + 1] = make_double2(0.0, 0.0);
    }
}

template <int R, int NT>
__global__ void __launch_bounds__(NT) adj0_kernel(LegParams p, const double2 *__restrict__ V_all,
                                                   double2 *__restrict__ alm_all) {
    constexpr int NW = NT / 32;
    __shared__ double s_al[kChunk], s_c[kChunk];
    __shared__ double2 s_red[NW][kChunk];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int L = p.lmax;
    const double2 *V = V_all + (size_t)blockIdx.y * p.nrings * p.M;
    double2 *alm = alm_all + (size_t)blockIdx.y * p.K;
    const int j = blockIdx.x;
    for (int pass = 0; pass < 2; ++pass) {
        const int m = pass ? L - j : j;
        if (pass && m <= j) break;
        const SeedParam sp = p.seed[m];
        const long long b0 = alm_index(sp.lmin, m, L);
        const int nst = L - sp.lmin + 1;
        for (int tile = 0; tile < p.T; tile += NT * R) {
            double x[R], u1[R], u2[R];
            int sc[R];
            double2 UA[R], UB[R];
            bool fast = true;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                double mant = 0.0, xx = 0.0;
                int s = 0;
                double2 vn = make_double2(0.0, 0.0), vs = make_double2(0.0, 0.0);
                if (t < p.T) {
                    xx = p.x[t];
                    make_seed(seed_log0(sp, m, p.logsin[t]), sp.sign[0], mant, s);
                    vn = V[(size_t)t * p.M + m];
                    if (t < p.T - 1) vs = V[(size_t)(4 * p.nside - 2 - t) * p.M + m];
                }
                // b_l = sum_t lambda (Vn + (-1)^l (-1)^m V_south)  (_recursion.py:472-497, healpix.py:255-258)
                x[k] = xx;
                u1[k] = 0.0;
                u2[k] = -mant;
                sc[k] = s;
                fast &= (s == 0);
                UA[k] = make_double2(vn.x + vs.x, vn.y + vs.y);
                UB[k] = make_double2(vn.x - vs.x, vn.y - vs.y);
            }
            for (int i0 = 0; i0 < nst; i0 += kChunk) {
                const int cnt = min(kChunk, nst - i0);
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    const long long idx = b0 + i0 + q;
                    s_al[q] = p.alpha[idx];
                    s_c[q] = p.cnorm[idx];
                }
                __syncthreads();
                for (int q0 = 0; q0 < cnt; q0 += kSub) {
                    double2 part[kSub];
                    if (__all_sync(kFull, fast)) {
                        adj0_sub<R, false>(cnt - q0, s_al + q0, x, u1, u2, sc, UA, UB, part);
                    } else {
                        adj0_sub<R, true>(cnt - q0, s_al + q0, x, u1, u2, sc, UA, UB, part);
                        fast = true;
#pragma unroll
                        for (int k = 0; k < R; ++k) fast &= (sc[k] == 0);
                    }
                    warp_reduce_scatter<kSub>(part, lane);
                    if (scatter_writer<kSub>(lane)) s_red[warp][q0 + scatter_index<kSub>(lane)] = part[0];
                }
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    double2 s = s_red[0][q];
#pragma unroll
                    for (int w = 1; w < NW; ++w) {
                        s.x += s_red[w][q].x;
                        s.y += s_red[w][q].y;
                    }
                    const double c = s_c[q];
                    const long long idx = b0 + i0 + q;
                    double2 o = make_double2(c * s.x, c * s.y);
                    if (tile > 0) {
                        const double2 prev = alm[idx];
                        o.x += prev.x;
                        o.y += prev.y;
                    }
                    alm[idx] = o;
                }
            }
        }
    }
}

// ---------------- spin 2 ----------------
struct In2 {
    double2 vpn, spA, vmn, smA;  // north data and the (-1)^(m+lmin)-signed south data
};

template <int R, bool SLOW, int SGN>
__device__ __forceinline__ void adj2_step(double al, double ga, const double (&x)[R], double (&p1)[R],
                                          double (&p2)[R], int (&sp)[R], double (&m1)[R], double (&m2)[R],
                                          int (&sm)[R], const In2 (&in)[R], double2 &op, double2 &om) {
    op = make_double2(0.0, 0.0);
    om = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const double tp = fma(al, x[k], ga);
        const double tm = fma(al, x[k], -ga);
        double up = fma(tp, p1[k], -p2[k]);
        double um = fma(tm, m1[k], -m2[k]);
        double pp = p1[k], pm = m1[k];
        if (SLOW) {
            rescale(up, pp, sp[k]);
            rescale(um, pm, sm[k]);
        }
        p2[k] = pp;
        p1[k] = up;
        m2[k] = pm;
        m1[k] = um;
        if (SLOW) {
            if (sp[k] != 0) up = 0.0;
            if (sm[k] != 0) um = 0.0;
        }
        const In2 &d = in[k];
        // p2 += lp Vpn + (-1)^l lm Sp ;  m2 += lm Vmn + (-1)^l lp Sm   (_recursion.py:565-566)
        op.x = fma(up, d.vpn.x, op.x);
        op.y = fma(up, d.vpn.y, op.y);
        op.x = fma(SGN * um, d.spA.x, op.x);
        op.y = fma(SGN * um, d.spA.y, op.y);
        om.x = fma(um, d.vmn.x, om.x);
        om.y = fma(um, d.vmn.y, om.y);
        om.x = fma(SGN * up, d.smA.x, om.x);
        om.y = fma(SGN * up, d.smA.y, om.y);
    }
}

template <int R, bool SLOW>
__device__ __forceinline__ void adj2_sub(int cnt, const double *s_al, const double *s_ga, const double (&x)[R],
                                         double (&p1)[R], double (&p2)[R], int (&sp)[R], double (&m1)[R],
                                         double (&m2)[R], int (&sm)[R], const In2 (&in)[R],
                                         double2 (&part)[2 * kSub]) {
#pragma unroll
    for (int q = 0; q < kSub; q += 2) {
        if (q < cnt) adj2_step<R, SLOW, 1>(s_al[q], s_ga[q], x, p1, p2, sp, m1, m2, sm, in, part[q], part[kSub + q]);
        else part[q] = part[kSub + q] = make_double2(0.0, 0.0);
        if (q + 1 < cnt)
            adj2_step<R, SLOW, -1>(s_al[q + 1], s_ga[q + 1], x, p1, p2, sp, m1, m2, sm, in, part[q + 1],
                                   part[kSub + q + 1]);
        else part[q + 1] = part[kSub + q + 1] = make_double2(0.0, 0.0);
    }
}

template <int R, int NT>
__global__ void __launch_bounds__(NT) adj2_kernel(LegParams p, const double2 *__restrict__ V_all,
                                                   double2 *__restrict__ alm_all) {
    constexpr int NW = NT / 32;
    __shared__ double s_al[kChunk], s_ga[kChunk], s_c[kChunk];
    __shared__ double2 s_red[NW][2 * kChunk];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int L = p.lmax;
    const double2 *Vp = V_all + (size_t)blockIdx.y * 2 * p.nrings * p.M;
    const double2 *Vm = Vp + (size_t)p.nrings * p.M;
    double2 *aE = alm_all + (size_t)blockIdx.y * 2 * p.K;
    double2 *aB = aE + p.K;
    const int j = blockIdx.x;
    for (int pass = 0; pass < 2; ++pass) {
        const int m = pass ? L - j : j;
        if (pass && m <= j) break;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        const double ssign = ((m + sd.lmin) & 1) ? -1.0 : 1.0;
        // modes l in [m, lmin) do not exist for spin 2: zero them
        if (tid < sd.lmin - m) {
            const long long idx = alm_index(m + tid, m, L);
            aE[idx] = make_double2(0.0, 0.0);
            aB[idx] = make_double2(0.0, 0.0);
        }
        for (int tile = 0; tile < p.T; tile += NT * R) {
            double x[R], p1[R], p2[R], m1[R], m2[R];
            int sp[R], sm[R];
            In2 in[R];
            bool fast = true;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int t = tile + k * NT + tid;
                double mp = 0.0, mm = 0.0, xx = 0.0;
                int s1 = 0, s2 = 0;
                In2 d;
                d.vpn = d.spA = d.vmn = d.smA = make_double2(0.0, 0.0);
                if (t < p.T) {
                    xx = p.x[t];
                    const double lch = p.logch[t], lsh = p.logsh[t];
                    make_seed(seed_log2(sd, 0, lch, lsh), sd.sign[0], mp, s1);
                    make_seed(seed_log2(sd, 1, lch, lsh), sd.sign[1], mm, s2);
                    d.vpn = Vp[(size_t)t * p.M + m];
                    d.vmn = Vm[(size_t)t * p.M + m];
                    if (t < p.T - 1) {
                        const size_t rs = (size_t)(4 * p.nside - 2 - t) * p.M + m;
                        const double2 a = Vp[rs], b = Vm[rs];
                        d.spA = make_double2(ssign * a.x, ssign * a.y);
                        d.smA = make_double2(ssign * b.x, ssign * b.y);
                    }
                }
                x[k] = xx;
                p1[k] = 0.0;
                p2[k] = -mp;
                sp[k] = s1;
                m1[k] = 0.0;
                m2[k] = -mm;
                sm[k] = s2;
                fast &= (s1 == 0) && (s2 == 0);
                in[k] = d;
            }
            for (int i0 = 0; i0 < nst; i0 += kChunk) {
                const int cnt = min(kChunk, nst - i0);
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    const long long idx = b0 + i0 + q;
                    s_al[q] = p.alpha[idx];
                    s_ga[q] = p.gamma[idx];
                    s_c[q] = p.cnorm[idx];
                }
                __syncthreads();
                for (int q0 = 0; q0 < cnt; q0 += kSub) {
                    double2 part[2 * kSub];
                    if (__all_sync(kFull, fast)) {
                        adj2_sub<R, false>(cnt - q0, s_al + q0, s_ga + q0, x, p1, p2, sp, m1, m2, sm, in, part);
                    } else {
                        adj2_sub<R, true>(cnt - q0, s_al + q0, s_ga + q0, x, p1, p2, sp, m1, m2, sm, in, part);
                        fast = true;
#pragma unroll
                        for (int k = 0; k < R; ++k) fast &= (sp[k] == 0) && (sm[k] == 0);
                    }
                    warp_reduce_scatter<2 * kSub>(part, lane);
                    if (scatter_writer<2 * kSub>(lane)) {
                        const int e = scatter_index<2 * kSub>(lane);  // 0..7: p2, 8..15: m2
                        s_red[warp][(e >= kSub ? kChunk : 0) + q0 + (e & (kSub - 1))] = part[0];
                    }
                }
                __syncthreads();
                for (int q = tid; q < cnt; q += NT) {
                    double2 sp2 = s_red[0][q], sm2 = s_red[0][kChunk + q];
#pragma unroll
                    for (int w = 1; w < NW; ++w) {
                        sp2.x += s_red[w][q].x;
                        sp2.y += s_red[w][q].y;
                        sm2.x += s_red[w][kChunk + q].x;
                        sm2.y += s_red[w][kChunk + q].y;
                    }
                    const double c = s_c[q];
                    const long long idx = b0 + i0 + q;
                    // aE = (-p2 - m2)/2, aB = i (p2 - m2)/2  (healpix.py:353-354)
                    const double pr = c * sp2.x, pi = c * sp2.y, mr = c * sm2.x, mi = c * sm2.y;
                    double2 e = make_double2(0.5 * (-pr - mr), 0.5 * (-pi - mi));
                    double2 b = make_double2(0.5 * (-(pi - mi)), 0.5 * (pr - mr));
                    if (tile > 0) {
                        const double2 pe = aE[idx], pb = aB[idx];
                        e.x += pe.x;
                        e.y += pe.y;
                        b.x += pb.x;
                        b.y += pb.y;
                    }
                    aE[idx] = e;
                    aB[idx] = b;
                }
            }
        }
    }
}

constexpr int kNT = 256;
constexpr int kR0 = 4;  // rings per thread, spin 0
constexpr int kR2 = 2;  // rings per thread, spin 2

}  // namespace

int launch_legendre_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.npairs, nb);
    LegParams q = make_params(p);
    if (p.spin == 0) synth0_kernel<kR0, kNT><<<grid, kNT, 0, s>>>(q, alm, F);
    else synth2_kernel<kR2, kNT><<<grid, kNT, 0, s>>>(q, alm, F);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_legendre_adjoint(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    dim3 grid(p.npairs, nb);
    LegParams q = make_params(p);
    if (p.spin == 0) adj0_kernel<kR0, kNT><<<grid, kNT, 0, s>>>(q, F, alm);
    else adj2_kernel<kR2, kNT><<<grid, kNT, 0, s>>>(q, F, alm);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // namespace jhtb
