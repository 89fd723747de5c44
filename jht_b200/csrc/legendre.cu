// Fused Legendre / Wigner-d recursion + l-contraction, FP64 (sm_100a).
//
// Synthesis (jht _recursion.py:441-469 spin 0, :512-543 spin 2) and its exact
// transpose (:472-497, :546-572).  For each order m and half-grid ring t the
// recursion runs over l entirely in registers; no lambda table is stored.
//
// Work decomposition.  A warp tile is 32*R consecutive half-grid rings of one m
// (R rings per lane, 32 apart).  Persistent warps pull work items from an atomic
// queue sorted by cost, so the triangle of work over m balances without m-pairing
// and no CTA-wide barrier ever couples warps:
//   synthesis: item = (m, warp tile); each item writes its own F[ring][m] entries.
//   adjoint:   item = (m, quarter of the rings); the warp sweeps its warp tiles in
//              ascending start-l order and accumulates each l's ring sum into its
//              own partial row; a final kernel adds the four quarters in fixed
//              order -- deterministic, no atomics on data.
//
// Numerics.  jht carries lambda as (mantissa, log-scale) renormalised every step
// (_recursion.py:352-369: one sqrt, log, exp and two divisions per step).  Here the
// recursion is rewritten with per-(l,m) normalised coefficients (plan.cu):
//     mu_l = (alpha_l x + gamma_l) mu_{l-1} - mu_{l-2},   lambda_l = c_l mu_l,
// two FMAs per step; underflow is handled with an integer scale (value =
// mu 2^(800 sc)).  While sc < 0 the value is < 2^-400 and is not accumulated.
//
// Dead-work skipping.  For (m, ring) near the poles lambda stays below 2^-400 for
// the first part of the l range (23% of all (l, m, ring) triples at nside 2048,
// lmax 4096).  At plan creation start_state_kernel runs that part once per warp
// tile and stores, at the first l where any ring of the tile is representable
// (rounded down to an even offset from lmin), every ring's (mu_{l-1}, mu_{l-2}, sc).
// The transforms then start there; rings still scaled run the rescale-check
// variant until the whole warp is representable, after which the loop is
// branch-free.
//
// Parity.  Step i = l - lmin alternates between accumulator slots A (i even) and
// B (i odd); N/S outputs are A +- B, realising jht's total / signed sums.
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"
#include "seed.cuh"

namespace jhtb {
namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kStage = 32;  // steps staged per warp per round (one per lane)
#ifndef JHTB_ADJ_SUB
#define JHTB_ADJ_SUB 8
#endif
constexpr int kSub = JHTB_ADJ_SUB;  // adjoint steps per warp reduction
// resident CTAs per SM the adjoint kernels are compiled for (their register budget)
#ifndef JHTB_ADJ0_MINB
#define JHTB_ADJ0_MINB 4
#endif
#ifndef JHTB_ADJ2_MINB
#define JHTB_ADJ2_MINB 3
#endif
constexpr int kAdj0MinBlocks = JHTB_ADJ0_MINB;
constexpr int kAdj2MinBlocks = JHTB_ADJ2_MINB;
constexpr unsigned kFull = 0xffffffffu;

struct LegParams {
    int lmax, T, nrings, M, nside;
    long long K;
    const double *x, *logsin, *logch, *logsh;
    const SeedParam *seed;
    const double *alpha, *gamma, *cnorm;
    // work items
    int ntiles;               // warp tiles per m
    int nsynth;               // entries of synth_order
    int nsuper, tps;          // adjoint: quarters per m, warp tiles per quarter
    const int *lw;            // [M * ntiles] start l per (m, tile)
    const double2 *st;        // [M * ntiles][nrec][R][32] start (u1, u2)
    const int *stsc;          // [M * ntiles][nrec][R][32] start scale
    const int *synth_order;   // [M * ntiles]
    const int *adj_order;     // [M * nsuper]
    const int *adj_tiles;     // [M * nsuper][tps] tile ids, ascending start l, -1 padded
    unsigned *counter;
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
    q.ntiles = p.ntiles;
    q.nsynth = p.nsynth;
    q.nsuper = p.nsuper;
    q.tps = p.tps;
    q.lw = p.d_lw;
    q.st = p.d_st;
    q.stsc = p.d_stsc;
    q.synth_order = p.d_synth_order;
    q.adj_order = p.d_adj_order;
    q.adj_tiles = p.d_adj_tiles;
    q.counter = p.d_counter;
    return q;
}

__device__ __forceinline__ void rescale(double &u, double &prev, int &sc) {
    if (sc < 0 && fabs(u) > kBig) {
        u *= kScaleDown;
        prev *= kScaleDown;
        sc += 1;
    }
}

__device__ __forceinline__ int next_item(unsigned *counter) {
    int it = 0;
    if ((threadIdx.x & 31) == 0) it = (int)atomicAdd(counter, 1u);
    return __shfl_sync(kFull, it, 0);
}

// =====================================================================================
// start states (plan creation): run the scaled recursion of each warp tile up to the
// first step at which any of its rings is representable.
// =====================================================================================
template <int SPIN, int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) start_state_kernel(LegParams p, int nitems) {
    constexpr int NREC = SPIN ? 2 : 1;
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (item >= nitems) return;
    const int m = item / p.ntiles, tile = item % p.ntiles;
    const SeedParam sd = p.seed[m];
    const long long b0 = alm_index(sd.lmin, m, p.lmax);
    const int nst = p.lmax - sd.lmin + 1;
    double x[R], u1[NREC][R], u2[NREC][R];
    int sc[NREC][R];
    bool valid[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int t = tile * 32 * R + r * 32 + lane;
        valid[r] = t < p.T;
        x[r] = valid[r] ? p.x[t] : 0.0;
#pragma unroll
        for (int h = 0; h < NREC; ++h) {
            double mant = 0.0;
            int s = 0;
            if (valid[r]) {
                const double lg = SPIN ? seed_log2(sd, h, p.logch[t], p.logsh[t]) : seed_log0(sd, m, p.logsin[t]);
                make_seed(lg, sd.sign[h], mant, s);
            }
            u1[h][r] = 0.0;
            u2[h][r] = -mant;
            sc[h][r] = s;
        }
    }
    double s1[NREC][R], s2[NREC][R];
    int ssc[NREC][R];
    int iw = nst;  // dead unless a ring becomes representable
    for (int i = 0; i < nst; ++i) {
        if ((i & 1) == 0) {
#pragma unroll
            for (int h = 0; h < NREC; ++h)
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    s1[h][r] = u1[h][r];
                    s2[h][r] = u2[h][r];
                    ssc[h][r] = sc[h][r];
                }
        }
        const double al = p.alpha[b0 + i];
        const double ga = SPIN ? p.gamma[b0 + i] : 0.0;
        bool sig = false;
#pragma unroll
        for (int h = 0; h < NREC; ++h) {
            const double g = h ? -ga : ga;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                double u = fma(fma(al, x[r], g), u1[h][r], -u2[h][r]);
                double prev = u1[h][r];
                rescale(u, prev, sc[h][r]);
                u2[h][r] = prev;
                u1[h][r] = u;
                sig |= valid[r] && sc[h][r] == 0;
            }
        }
        if (__any_sync(kFull, sig)) {
            iw = i & ~1;
            break;
        }
    }
    if (lane == 0) const_cast<int *>(p.lw)[item] = sd.lmin + iw;
    double2 *st = const_cast<double2 *>(p.st) + (size_t)item * NREC * R * 32;
    int *stsc = const_cast<int *>(p.stsc) + (size_t)item * NREC * R * 32;
#pragma unroll
    for (int h = 0; h < NREC; ++h)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int o = (h * R + r) * 32 + lane;
            if (iw < nst) {
                st[o] = make_double2(s1[h][r], s2[h][r]);
                stsc[o] = valid[r] ? ssc[h][r] : 0;
            } else {
                st[o] = make_double2(0.0, 0.0);
                stsc[o] = 0;
            }
        }
}

// Load the start state of ring slot r for recursion h; invalid rings read (0, 0, 0).
template <int R>
__device__ __forceinline__ void load_start(const LegParams &p, int item, int h, int nrec, int lane, double (&u1)[R],
                                           double (&u2)[R], int (&sc)[R]) {
    const double2 *st = p.st + (size_t)item * nrec * R * 32;
    const int *stsc = p.stsc + (size_t)item * nrec * R * 32;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double2 s = st[(h * R + r) * 32 + lane];
        u1[r] = s.x;
        u2[r] = s.y;
        sc[r] = stsc[(h * R + r) * 32 + lane];
    }
}

// =====================================================================================
// synthesis
// =====================================================================================
struct Stage0 {
    double al[kStage];
    double2 c[kStage];
};
struct Stage2 {
    double2 ag[kStage];  // (alpha, gamma)
    double2 cp[kStage], cm[kStage];
};

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
        if (SLOW && sc[k] != 0) u = 0.0;
        ar[k] = fma(c.x, u, ar[k]);
        ai[k] = fma(c.y, u, ai[k]);
    }
}

template <int R, bool SLOW>
__device__ __forceinline__ void synth0_chunk(int cnt, const Stage0 &sb, const double (&x)[R], double (&u1)[R],
                                             double (&u2)[R], int (&sc)[R], double (&Ar)[R], double (&Ai)[R],
                                             double (&Br)[R], double (&Bi)[R]) {
    if (cnt == kStage) {
#pragma unroll
        for (int q = 0; q < kStage; q += 2) {
            synth0_step<R, SLOW>(sb.al[q], sb.c[q], x, u1, u2, sc, Ar, Ai);
            synth0_step<R, SLOW>(sb.al[q + 1], sb.c[q + 1], x, u1, u2, sc, Br, Bi);
        }
        return;
    }
    int q = 0;
    for (; q + 1 < cnt; q += 2) {
        synth0_step<R, SLOW>(sb.al[q], sb.c[q], x, u1, u2, sc, Ar, Ai);
        synth0_step<R, SLOW>(sb.al[q + 1], sb.c[q + 1], x, u1, u2, sc, Br, Bi);
    }
    if (q < cnt) synth0_step<R, SLOW>(sb.al[q], sb.c[q], x, u1, u2, sc, Ar, Ai);
}

template <int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) synth0_kernel(LegParams p, const double2 *__restrict__ alm_all,
                                                                     double2 *__restrict__ F_all, int nb) {
    __shared__ Stage0 stage[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    Stage0 &sb = stage[threadIdx.x >> 5];
    const int nitems = p.nsynth;
    const int L = p.lmax;
    for (;;) {
        const int it = next_item(p.counter);
        if (it >= nitems * nb) break;
        const int b = it / nitems;
        const int item = p.synth_order[it - b * nitems];
        const int m = item / p.ntiles, tile = item % p.ntiles;
        const double2 *alm = alm_all + (size_t)b * p.K;
        double2 *F = F_all + (size_t)b * p.nrings * p.M;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        const int i_start = p.lw[item] - sd.lmin;
        double x[R], u1[R], u2[R], Ar[R], Ai[R], Br[R], Bi[R];
        int sc[R];
        load_start<R>(p, item, 0, 1, lane, u1, u2, sc);
        bool fast = true;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = tile * 32 * R + r * 32 + lane;
            x[r] = t < p.T ? p.x[t] : 0.0;
            fast &= sc[r] == 0;
            Ar[r] = Ai[r] = Br[r] = Bi[r] = 0.0;
        }
        for (int i0 = i_start; i0 < nst; i0 += kStage) {
            const int cnt = min(kStage, nst - i0);
            if (lane < cnt && JHTB_IN(b0 + i0 + lane, p.K, 201)) {
                const long long idx = b0 + i0 + lane;
                const double c = p.cnorm[idx];
                const double2 a = alm[idx];
                sb.al[lane] = p.alpha[idx];
                sb.c[lane] = make_double2(a.x * c, a.y * c);
            }
            __syncwarp();
            if (__all_sync(kFull, fast)) {
                synth0_chunk<R, false>(cnt, sb, x, u1, u2, sc, Ar, Ai, Br, Bi);
            } else {
                synth0_chunk<R, true>(cnt, sb, x, u1, u2, sc, Ar, Ai, Br, Bi);
                fast = true;
#pragma unroll
                for (int r = 0; r < R; ++r) fast &= sc[r] == 0;
            }
            __syncwarp();
        }
        // F_north = A + B; F_south = (-1)^m (E - O) = A - B   (healpix.py:250-253)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = tile * 32 * R + r * 32 + lane;
            if (t < p.T && JHTB_IN((long long)(p.nrings - 1 - t) * p.M + m, (long long)p.nrings * p.M, 202)) {
                F[(size_t)t * p.M + m] = make_double2(Ar[r] + Br[r], Ai[r] + Bi[r]);
                if (t < p.T - 1)
                    F[(size_t)(p.nrings - 1 - t) * p.M + m] = make_double2(Ar[r] - Br[r], Ai[r] - Bi[r]);
            }
        }
    }
}

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
__device__ __forceinline__ void synth2_chunk(int cnt, const Stage2 &sb, const double (&x)[R], double (&p1)[R],
                                             double (&p2)[R], int (&sp)[R], double (&m1)[R], double (&m2)[R],
                                             int (&sm)[R], Acc2 (&acc)[R]) {
    if (cnt == kStage) {  // whole chunk: fully unrolled so the shared-memory loads pipeline
#pragma unroll
        for (int q = 0; q < kStage; q += 2) {
            synth2_step<R, SLOW, 1>(sb.ag[q].x, sb.ag[q].y, sb.cp[q], sb.cm[q], x, p1, p2, sp, m1, m2, sm, acc);
            synth2_step<R, SLOW, -1>(sb.ag[q + 1].x, sb.ag[q + 1].y, sb.cp[q + 1], sb.cm[q + 1], x, p1, p2, sp, m1, m2, sm, acc);
        }
        return;
    }
    int q = 0;
    for (; q + 1 < cnt; q += 2) {
        synth2_step<R, SLOW, 1>(sb.ag[q].x, sb.ag[q].y, sb.cp[q], sb.cm[q], x, p1, p2, sp, m1, m2, sm, acc);
        synth2_step<R, SLOW, -1>(sb.ag[q + 1].x, sb.ag[q + 1].y, sb.cp[q + 1], sb.cm[q + 1], x, p1, p2, sp, m1, m2, sm, acc);
    }
    if (q < cnt) synth2_step<R, SLOW, 1>(sb.ag[q].x, sb.ag[q].y, sb.cp[q], sb.cm[q], x, p1, p2, sp, m1, m2, sm, acc);
}

template <int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) synth2_kernel(LegParams p, const double2 *__restrict__ alm_all,
                                                                     double2 *__restrict__ F_all, int nb) {
    __shared__ Stage2 stage[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    Stage2 &sb = stage[threadIdx.x >> 5];
    const int nitems = p.nsynth;
    const int L = p.lmax;
    for (;;) {
        const int it = next_item(p.counter);
        if (it >= nitems * nb) break;
        const int b = it / nitems;
        const int item = p.synth_order[it - b * nitems];
        const int m = item / p.ntiles, tile = item % p.ntiles;
        const double2 *aE = alm_all + (size_t)b * 2 * p.K;
        const double2 *aB = aE + p.K;
        double2 *Fp = F_all + (size_t)b * 2 * p.nrings * p.M;
        double2 *Fm = Fp + (size_t)p.nrings * p.M;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        const int i_start = p.lw[item] - sd.lmin;
        // south sign (-1)^(m + lmin): the signed sums are relative to l = lmin
        const double ssign = ((m + sd.lmin) & 1) ? -1.0 : 1.0;
        double x[R], p1[R], p2[R], m1[R], m2[R];
        int sp[R], sm[R];
        Acc2 acc[R];
        load_start<R>(p, item, 0, 2, lane, p1, p2, sp);
        load_start<R>(p, item, 1, 2, lane, m1, m2, sm);
        bool fast = true;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = tile * 32 * R + r * 32 + lane;
            x[r] = t < p.T ? p.x[t] : 0.0;
            fast &= (sp[r] == 0) && (sm[r] == 0);
            acc[r] = Acc2{0, 0, 0, 0, 0, 0, 0, 0};
        }
        for (int i0 = i_start; i0 < nst; i0 += kStage) {
            const int cnt = min(kStage, nst - i0);
            if (lane < cnt && JHTB_IN(b0 + i0 + lane, p.K, 201)) {
                const long long idx = b0 + i0 + lane;
                const double c = p.cnorm[idx];
                const double2 e = aE[idx], bb = aB[idx];
                sb.ag[lane] = make_double2(p.alpha[idx], p.gamma[idx]);
                // cp = -(aE + i aB) c, cm = -(aE - i aB) c   (healpix.py:316-318)
                sb.cp[lane] = make_double2(-(e.x - bb.y) * c, -(e.y + bb.x) * c);
                sb.cm[lane] = make_double2(-(e.x + bb.y) * c, -(e.y - bb.x) * c);
            }
            __syncwarp();
            if (__all_sync(kFull, fast)) {
                synth2_chunk<R, false>(cnt, sb, x, p1, p2, sp, m1, m2, sm, acc);
            } else {
                synth2_chunk<R, true>(cnt, sb, x, p1, p2, sp, m1, m2, sm, acc);
                fast = true;
#pragma unroll
                for (int r = 0; r < R; ++r) fast &= (sp[r] == 0) && (sm[r] == 0);
            }
            __syncwarp();
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int t = tile * 32 * R + r * 32 + lane;
            if (t < p.T && JHTB_IN((long long)(p.nrings - 1 - t) * p.M + m, (long long)p.nrings * p.M, 202)) {
                const Acc2 &a = acc[r];
                Fp[(size_t)t * p.M + m] = make_double2(a.ppr, a.ppi);
                Fm[(size_t)t * p.M + m] = make_double2(a.mmr, a.mmi);
                if (t < p.T - 1) {
                    const size_t rs = (size_t)(p.nrings - 1 - t) * p.M + m;
                    Fp[rs] = make_double2(ssign * a.pmr, ssign * a.pmi);
                    Fm[rs] = make_double2(ssign * a.mpr, ssign * a.mpi);
                }
            }
        }
    }
}

// =====================================================================================
// adjoint
// =====================================================================================
// Warp sum of NE per-lane values through shared memory (no shuffles or selects on the
// step path): every lane stores its NE values (one 16-byte row slot per entry), then
// LPE = 32 / NE lanes share each entry, each adding 32 / LPE of the rows in a fixed order
// (two interleaved chains), and a final xor-shuffle combines the LPE partial sums.
// A row holds 32 + LPE slots: with that padding both the stores (8 consecutive slots per
// quarter warp) and the loads (8 distinct 16-byte bank groups per quarter warp) are
// conflict-free.
template <int NE>
struct RedBuf {
    static constexpr int LPE = 32 / NE;
    double2 v[NE][32 + LPE];
};

template <int NE>
__device__ __forceinline__ double2 red_sum(const RedBuf<NE> &rb, int lane) {
    constexpr int LPE = RedBuf<NE>::LPE;
    constexpr int NK = 32 / LPE;
    const int e = lane / LPE, h = lane % LPE;
    double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < NK; k += 2) {
        const double2 a = rb.v[e][LPE * k + h], b = rb.v[e][LPE * (k + 1) + h];
        s0.x += a.x;
        s0.y += a.y;
        s1.x += b.x;
        s1.y += b.y;
    }
    double2 s = make_double2(s0.x + s1.x, s0.y + s1.y);
#pragma unroll
    for (int msk = 1; msk < LPE; msk <<= 1) {
        s.x += __shfl_xor_sync(kFull, s.x, msk);
        s.y += __shfl_xor_sync(kFull, s.y, msk);
    }
    return s;
}

struct AStage {
    double2 ag[kStage];  // (alpha, gamma)
};

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

template <int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kAdj0MinBlocks) adj0_kernel(LegParams p, const double2 *__restrict__ V_all,
                                                                   double2 *__restrict__ part_all, int nb) {
    __shared__ AStage stage[kWarpsPerBlock];
    __shared__ RedBuf<kSub> red[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    AStage &sb = stage[threadIdx.x >> 5];
    RedBuf<kSub> &rb = red[threadIdx.x >> 5];
    constexpr int LPE = RedBuf<kSub>::LPE;
    const int nsup = p.M * p.nsuper;
    const int L = p.lmax;
    for (;;) {
        const int it = next_item(p.counter);
        if (it >= nsup * nb) break;
        const int b = it / nsup;
        const int sitem = p.adj_order[it - b * nsup];
        const int m = sitem / p.nsuper, s = sitem % p.nsuper;
        const double2 *V = V_all + (size_t)b * p.nrings * p.M;
        double2 *part = part_all + ((size_t)b * p.nsuper + s) * p.K;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        bool any = false;  // a live tile has already written the row
        for (int j = 0; j < p.tps; ++j) {
            const int tile = p.adj_tiles[(size_t)sitem * p.tps + j];
            if (tile < 0) break;
            const int item = m * p.ntiles + tile;
            const int i_start = p.lw[item] - sd.lmin;
            if (i_start >= nst) break;  // ascending order: the rest are dead too
            const bool acc = any;       // later tiles add onto the row (their range is inside)
            if (!any)                   // first live tile: zero the prefix no tile reaches
                for (int i = lane; i < i_start; i += 32) part[b0 + i] = make_double2(0.0, 0.0);
            double x[R], u1[R], u2[R];
            int sc[R];
            double2 UA[R], UB[R];
            load_start<R>(p, item, 0, 1, lane, u1, u2, sc);
            bool fast = true;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int t = tile * 32 * R + r * 32 + lane;
                double2 vn = make_double2(0.0, 0.0), vs = make_double2(0.0, 0.0);
                x[r] = 0.0;
                if (t < p.T && JHTB_IN((long long)(p.nrings - 1 - t) * p.M + m, (long long)p.nrings * p.M, 203)) {
                    x[r] = p.x[t];
                    vn = V[(size_t)t * p.M + m];
                    if (t < p.T - 1) vs = V[(size_t)(p.nrings - 1 - t) * p.M + m];
                }
                // b_l = sum_t lambda (Vn + (-1)^l (-1)^m V_south)  (_recursion.py:472-497)
                UA[r] = make_double2(vn.x + vs.x, vn.y + vs.y);
                UB[r] = make_double2(vn.x - vs.x, vn.y - vs.y);
                fast &= sc[r] == 0;
            }
            for (int i0 = i_start; i0 < nst; i0 += kStage) {
                const int cnt = min(kStage, nst - i0);
                if (lane < cnt) sb.ag[lane].x = p.alpha[b0 + i0 + lane];
                __syncwarp();
                for (int q0 = 0; q0 < cnt; q0 += kSub) {
                    // the writer lane's output slot is known up front: issue its load of
                    // the running row sum now so the L2 round trip overlaps the steps
                    const int qw = q0 + lane / LPE;
                    const bool wr = (lane % LPE) == 0 && qw < cnt;
                    double2 prev = make_double2(0.0, 0.0);
                    if (acc && wr && JHTB_IN(b0 + i0 + qw, p.K, 204)) prev = part[b0 + i0 + qw];
                    const bool f = __all_sync(kFull, fast);
                    if (f && q0 + kSub <= cnt) {  // one straight sequence of steps (see adj2_kernel)
#pragma unroll
                        for (int q = 0; q < kSub; q += 2) {
                            rb.v[q][lane] = adj0_step<R, false>(sb.ag[q0 + q].x, x, u1, u2, sc, UA);
                            rb.v[q + 1][lane] = adj0_step<R, false>(sb.ag[q0 + q + 1].x, x, u1, u2, sc, UB);
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < kSub; q += 2) {
                            if (q0 + q < cnt) rb.v[q][lane] = adj0_step<R, true>(sb.ag[q0 + q].x, x, u1, u2, sc, UA);
                            if (q0 + q + 1 < cnt) rb.v[q + 1][lane] = adj0_step<R, true>(sb.ag[q0 + q + 1].x, x, u1, u2, sc, UB);
                        }
                    }
                    if (!f) {
                        fast = true;
#pragma unroll
                        for (int r = 0; r < R; ++r) fast &= sc[r] == 0;
                    }
                    __syncwarp();
                    const double2 tot = red_sum<kSub>(rb, lane);
                    __syncwarp();
                    if (wr && JHTB_IN(b0 + i0 + qw, p.K, 204)) part[b0 + i0 + qw] = make_double2(tot.x + prev.x, tot.y + prev.y);
                }
                __syncwarp();
            }
            any = true;
        }
        if (!any)  // no live tile: the whole row is zero
            for (int i = lane; i < nst; i += 32) part[b0 + i] = make_double2(0.0, 0.0);
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
        double qp = p1[k], qm = m1[k];
        if (SLOW) {
            rescale(up, qp, sp[k]);
            rescale(um, qm, sm[k]);
        }
        p2[k] = qp;
        p1[k] = up;
        m2[k] = qm;
        m1[k] = um;
        if (SLOW) {
            if (sp[k] != 0) up = 0.0;
            if (sm[k] != 0) um = 0.0;
        }
        const In2 &d = in[k];
        // p2 += lp Vpn + (-1)^l lm Sp ;  m2 += lm Vmn + (-1)^l lp Sm   (_recursion.py:565-566)
        op.x = fma(up, d.vpn.x, op.x);
        op.y = fma(up, d.vpn.y, op.y);
        om.x = fma(um, d.vmn.x, om.x);
        om.y = fma(um, d.vmn.y, om.y);
        op.x = fma(SGN * um, d.spA.x, op.x);
        op.y = fma(SGN * um, d.spA.y, op.y);
        om.x = fma(SGN * up, d.smA.x, om.x);
        om.y = fma(SGN * up, d.smA.y, om.y);
    }
}

template <int R>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kAdj2MinBlocks) adj2_kernel(LegParams p, const double2 *__restrict__ V_all,
                                                                   double2 *__restrict__ part_all, int nb) {
    constexpr int NV = 2 * kSub;
    __shared__ AStage stage[kWarpsPerBlock];
    __shared__ RedBuf<NV> red[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    AStage &sb = stage[threadIdx.x >> 5];
    RedBuf<NV> &rb = red[threadIdx.x >> 5];
    constexpr int LPE = RedBuf<NV>::LPE;
    const int nsup = p.M * p.nsuper;
    const int L = p.lmax;
    for (;;) {
        const int it = next_item(p.counter);
        if (it >= nsup * nb) break;
        const int b = it / nsup;
        const int sitem = p.adj_order[it - b * nsup];
        const int m = sitem / p.nsuper, s = sitem % p.nsuper;
        const double2 *Vp = V_all + (size_t)b * 2 * p.nrings * p.M;
        const double2 *Vm = Vp + (size_t)p.nrings * p.M;
        double2 *partP = part_all + ((size_t)b * p.nsuper + s) * 2 * p.K;
        double2 *partM = partP + p.K;
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        const double ssign = ((m + sd.lmin) & 1) ? -1.0 : 1.0;
        bool any = false;
        for (int j = 0; j < p.tps; ++j) {
            const int tile = p.adj_tiles[(size_t)sitem * p.tps + j];
            if (tile < 0) break;
            const int item = m * p.ntiles + tile;
            const int i_start = p.lw[item] - sd.lmin;
            if (i_start >= nst) break;
            const bool acc = any;
            if (!any)
                for (int i = lane; i < i_start; i += 32) {
                    partP[b0 + i] = make_double2(0.0, 0.0);
                    partM[b0 + i] = make_double2(0.0, 0.0);
                }
            double x[R], p1[R], p2[R], m1[R], m2[R];
            int sp[R], sm[R];
            In2 in[R];
            load_start<R>(p, item, 0, 2, lane, p1, p2, sp);
            load_start<R>(p, item, 1, 2, lane, m1, m2, sm);
            bool fast = true;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int t = tile * 32 * R + r * 32 + lane;
                In2 d;
                d.vpn = d.spA = d.vmn = d.smA = make_double2(0.0, 0.0);
                x[r] = 0.0;
                if (t < p.T && JHTB_IN((long long)(p.nrings - 1 - t) * p.M + m, (long long)p.nrings * p.M, 203)) {
                    x[r] = p.x[t];
                    d.vpn = Vp[(size_t)t * p.M + m];
                    d.vmn = Vm[(size_t)t * p.M + m];
                    if (t < p.T - 1) {
                        const size_t rs = (size_t)(p.nrings - 1 - t) * p.M + m;
                        const double2 a = Vp[rs], c = Vm[rs];
                        d.spA = make_double2(ssign * a.x, ssign * a.y);
                        d.smA = make_double2(ssign * c.x, ssign * c.y);
                    }
                }
                in[r] = d;
                fast &= (sp[r] == 0) && (sm[r] == 0);
            }
            for (int i0 = i_start; i0 < nst; i0 += kStage) {
                const int cnt = min(kStage, nst - i0);
                if (lane < cnt) sb.ag[lane] = make_double2(p.alpha[b0 + i0 + lane], p.gamma[b0 + i0 + lane]);
                __syncwarp();
                for (int q0 = 0; q0 < cnt; q0 += kSub) {
                    const int e = lane / LPE;  // entry of this lane's sum: 0..kSub-1 p2, kSub.. m2
                    const int qw = q0 + (e & (kSub - 1));
                    const bool wr = (lane % LPE) == 0 && qw < cnt;
                    double2 *dstw = e >= kSub ? partM : partP;
                    double2 prev = make_double2(0.0, 0.0);
                    if (acc && wr && JHTB_IN(b0 + i0 + qw, p.K, 204)) prev = dstw[b0 + i0 + qw];
                    const bool f = __all_sync(kFull, fast);
                    // The variant is chosen once per group, not per step: a whole group of
                    // representable rings runs one straight sequence of steps (choosing per
                    // step made the two variants' register assignments meet after every step).
                    if (f && q0 + kSub <= cnt) {
#pragma unroll
                        for (int q = 0; q < kSub; q += 2) {
                            double2 op, om;
                            adj2_step<R, false, 1>(sb.ag[q0 + q].x, sb.ag[q0 + q].y, x, p1, p2, sp, m1, m2, sm, in, op, om);
                            rb.v[q][lane] = op;
                            rb.v[kSub + q][lane] = om;
                            adj2_step<R, false, -1>(sb.ag[q0 + q + 1].x, sb.ag[q0 + q + 1].y, x, p1, p2, sp, m1, m2, sm, in, op, om);
                            rb.v[q + 1][lane] = op;
                            rb.v[kSub + q + 1][lane] = om;
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < kSub; q += 2) {
                            double2 op, om;
                            if (q0 + q < cnt) {
                                adj2_step<R, true, 1>(sb.ag[q0 + q].x, sb.ag[q0 + q].y, x, p1, p2, sp, m1, m2, sm, in, op, om);
                                rb.v[q][lane] = op;
                                rb.v[kSub + q][lane] = om;
                            }
                            if (q0 + q + 1 < cnt) {
                                adj2_step<R, true, -1>(sb.ag[q0 + q + 1].x, sb.ag[q0 + q + 1].y, x, p1, p2, sp, m1, m2, sm, in, op, om);
                                rb.v[q + 1][lane] = op;
                                rb.v[kSub + q + 1][lane] = om;
                            }
                        }
                    }
                    if (!f) {
                        fast = true;
#pragma unroll
                        for (int r = 0; r < R; ++r) fast &= (sp[r] == 0) && (sm[r] == 0);
                    }
                    __syncwarp();
                    const double2 tot = red_sum<NV>(rb, lane);
                    __syncwarp();
                    if (wr && JHTB_IN(b0 + i0 + qw, p.K, 204)) dstw[b0 + i0 + qw] = make_double2(tot.x + prev.x, tot.y + prev.y);
                }
                __syncwarp();
            }
            any = true;
        }
        if (!any)
            for (int i = lane; i < nst; i += 32) {
                partP[b0 + i] = make_double2(0.0, 0.0);
                partM[b0 + i] = make_double2(0.0, 0.0);
            }
    }
}

// Final adjoint combine: sum the ring quarters in fixed order, scale by c_l and,
// for spin 2, form aE = (-p2 - m2)/2, aB = i (p2 - m2)/2 (healpix.py:353-354).
template <int SPIN>
__global__ void adj_reduce_kernel(int lmax, long long K, int nsuper, const SeedParam *__restrict__ seed,
                                  const double *__restrict__ cnorm, const double2 *__restrict__ part_all,
                                  double2 *__restrict__ alm_all, int nb) {
    constexpr int NC = SPIN ? 2 : 1;
    const long long total = (long long)nb * K;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(g / K);
        const long long idx = g - (long long)b * K;
        if (!JHTB_IN(idx, K, 205)) continue;
        // (l, m) of the packed index: m from the column base
        int m = (int)floor(((2.0 * lmax + 3.0) - sqrt((2.0 * lmax + 3.0) * (2.0 * lmax + 3.0) - 8.0 * (double)idx)) / 2.0);
        if (m < 0) m = 0;
        while (m > 0 && alm_index(m, m, lmax) > idx) --m;
        while (m < lmax && alm_index(m + 1, m + 1, lmax) <= idx) ++m;
        const int l = (int)(idx - alm_index(0, m, lmax));
        double2 *out = alm_all + (size_t)b * NC * K;
        if (l < seed[m].lmin) {
            out[idx] = make_double2(0.0, 0.0);
            if (SPIN) out[K + idx] = make_double2(0.0, 0.0);
            continue;
        }
        const double2 *part = part_all + (size_t)b * nsuper * NC * K;
        double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
        for (int s = 0; s < nsuper; ++s) {
            const double2 a = part[(size_t)s * NC * K + idx];
            s0.x += a.x;
            s0.y += a.y;
            if (SPIN) {
                const double2 c = part[(size_t)s * NC * K + K + idx];
                s1.x += c.x;
                s1.y += c.y;
            }
        }
        const double c = cnorm[idx];
        if (!SPIN) {
            out[idx] = make_double2(c * s0.x, c * s0.y);
        } else {
            const double pr = c * s0.x, pi = c * s0.y, mr = c * s1.x, mi = c * s1.y;
            out[idx] = make_double2(0.5 * (-pr - mr), 0.5 * (-pi - mi));
            out[K + idx] = make_double2(0.5 * (-(pi - mi)), 0.5 * (pr - mr));
        }
    }
}

int persistent_grid(int blocks_per_sm) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm * blocks_per_sm;
}

template <typename Kern>
int resident_blocks(Kern k) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kWarpsPerBlock * 32, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

// Persistent grid of a Legendre kernel: every resident CTA, or the plan's tuned count.
template <typename Kern>
int leg_grid(const Plan &p, Kern k) {
    const int r = resident_blocks(k);
    return persistent_grid(p.leg_ctas > 0 ? std::min(p.leg_ctas, r) : r);
}

}  // namespace

JHTB_DEBUG_ACCESSOR(legendre)

int launch_start_states(const Plan &p, cudaStream_t s) {
    const int nitems = p.M * p.ntiles;
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    LegParams q = make_params(p);
    if (p.spin == 0) start_state_kernel<0, kR0><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    else start_state_kernel<2, kR2><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_start_states_r(const Plan &p, int R, int ntiles, int *lw, double2 *st, int *stsc, cudaStream_t s) {
    const int nitems = p.M * ntiles;
    const int grid = (nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    LegParams q = make_params(p);
    q.ntiles = ntiles;
    q.lw = lw;
    q.st = st;
    q.stsc = stsc;
    if (p.spin == 0 && R == 4) start_state_kernel<0, 4><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    else if (p.spin == 0 && R == 8) start_state_kernel<0, 8><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    else if (p.spin == 2 && R == 4) start_state_kernel<2, 4><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    else if (p.spin == 2 && R == 2) start_state_kernel<2, 2><<<grid, kWarpsPerBlock * 32, 0, s>>>(q, nitems);
    else return fail(JHTB_ERR_UNSUPPORTED, "start states: unsupported tile width");
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_legendre_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    JHTB_CUDA_TRY(cudaMemsetAsync(p.d_counter, 0, sizeof(unsigned), s));
    LegParams q = make_params(p);
    if (p.spin == 0) {
        auto k = synth0_kernel<kR0>;
        k<<<leg_grid(p, k), kWarpsPerBlock * 32, 0, s>>>(q, alm, F, nb);
    } else {
        auto k = synth2_kernel<kR2>;
        k<<<leg_grid(p, k), kWarpsPerBlock * 32, 0, s>>>(q, alm, F, nb);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

int launch_legendre_adjoint(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    JHTB_CUDA_TRY(cudaMemsetAsync(p.d_counter, 0, sizeof(unsigned), s));
    LegParams q = make_params(p);
    q.ntiles = p.a_ntiles;
    q.lw = p.d_a_lw;
    q.st = p.d_a_st;
    q.stsc = p.d_a_stsc;
    if (p.spin == 0) {
        auto k = adj0_kernel<kRA0>;
        k<<<leg_grid(p, k), kWarpsPerBlock * 32, 0, s>>>(q, F, p.d_part, nb);
    } else {
        auto k = adj2_kernel<kRA2>;
        k<<<leg_grid(p, k), kWarpsPerBlock * 32, 0, s>>>(q, F, p.d_part, nb);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    const long long total = (long long)nb * p.K;
    const int grid = (int)std::min<long long>((total + 255) / 256, 148LL * 32);
    if (p.spin == 0) adj_reduce_kernel<0><<<grid, 256, 0, s>>>(p.lmax, p.K, p.nsuper, p.d_seed, p.d_cnorm, p.d_part, alm, nb);
    else adj_reduce_kernel<2><<<grid, 256, 0, s>>>(p.lmax, p.K, p.nsuper, p.d_seed, p.d_cnorm, p.d_part, alm, nb);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // namespace jhtb
