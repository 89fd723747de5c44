// Batched mixed-precision adjoint Legendre stage on the 5th-generation tensor cores.
//
// The adjoint contracts over rings (jht _recursion.py:472-497 spin 0, :546-572 spin 2),
// while the recursion runs over l.  For one order m and a block of 128 degrees the
// contraction of 16 maps is a GEMM whose reduction dimension is the rings:
//     D[l, n] = sum_t mu_l(t) V[t, n],   l = MMA M (128), n = (map, column) = MMA N (64),
//     t = MMA K (16 rings per instruction), streamed over all live rings of the order.
// Spin 2 runs one GEMM per recursion: D+ = Mu+ [Vpn | s Sm], D- = Mu- [Vmn | s Sp]
// (s = (-1)^(m + lmin), north data and the south mirror's), and the two half-grid sums
// are p2 = D+[Vpn] + (-1)^(l-lmin) D-[Sp], m2 = D-[Vmn] + (-1)^(l-lmin) D+[Sm]; spin 0
// runs D = Mu [Vn | Vs] over two 16-ring halves of a 32-ring chunk, b = D[Vn] + (-1)^(l-lmin) D[Vs].
//
// Work: one item per (order m, block of 128 degrees); items are ordered by m so that the
// CTAs working at one time share the orders' ring data in L2.  A persistent CTA per SM
// runs four roles that meet only at mbarriers:
//   producer warps (one stage each, round robin): thread = (ring, recursion); four
//     independent chains per thread, one per 32-degree segment of the block, each started
//     from the plan's recursion state at its first degree (FP64, the same arithmetic as
//     the FP64 kernels), run the segment's 32 steps, round mu to FP32, split it into three
//     BF16 parts and store them as the A operand in MN-major layout (8 consecutive degrees
//     per 16-byte store);
//   a loader warp: one bulk copy per stage of the chunk's BF16x3 ring-data tiles (B
//     operand, K-major), prepared once per launch by adj_prep_kernel from the FP64 ring
//     spectra;
//   one MMA warp: six split products per GEMM (hh, hm, mh, hl, lh, mm) in four MMAs: hh
//     (N = 64) into a double-buffered FP32 accumulator; the five smaller ones into a
//     correction pair [X | Y] that runs over the whole item (relative size <= 2^-8), two
//     of them with N = 128 over consecutive ring-data splits (h [m | l] and m [h | m]) so
//     each A split is read from shared memory fewer times, and l h into X;
//   four epilogue warps (thread = degree = tensor-memory lane): every 256 rings they fold
//     the hh block sums, already combined into the half-grid sums, into FP64 accumulators
//     in registers (FP32 rounding acts on <= 256 rings); at the item's end they add the
//     correction sums X + Y, scale by c_l and write the item's a_lm (E, B for spin 2).
// The item covers every ring, so no partial sums leave the chip and the result does not
// depend on the order of the work.  Every wait is bounded (poll count and the plan's
// watchdog time); on timeout the kernel records an error, every role leaves its loops,
// and tensor memory is released after the issued MMAs have drained.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"
#include "seed.cuh"
#include "tc_common.cuh"

namespace jhtb {
namespace {
using namespace tc;

constexpr int kLB = kTcaLB;               // degrees per item = MMA M
constexpr int kTK = 16;                   // rings per MMA = K
constexpr int kN = 4 * kTcaMaps;          // 64 columns per GEMM = MMA N
#ifndef JHTB_TCA_NP
#define JHTB_TCA_NP 6
#endif
#ifndef JHTB_TCA_NSA
#define JHTB_TCA_NSA 7
#endif
constexpr int kNP = JHTB_TCA_NP;          // producer warps
constexpr int kNSA = JHTB_TCA_NSA;        // A stages
constexpr int kNSB = 4;                   // B stages
constexpr int kPrefetch = 8;              // ring-data tiles prefetched into L2 ahead of their copy
constexpr int kATile = kLB * kTK * 2;     // one split of one A sub-tile: 4096 bytes
constexpr int kBTile = kN * kTK * 2;      // one split of one B sub-tile: 2048 bytes
constexpr int kAStage = 2 * 3 * kATile;   // 24 KB
constexpr int kBStage = 2 * 3 * kBTile;   // 12 KB
static_assert(kBStage == kTcaBStage, "B stage size");
constexpr int kWLoad = kNP, kWMma = kNP + 1;  // then four epilogue warps
constexpr int kThreads = (kNP + 6) * 32;

template <int SPIN>
struct AdjCfg {
    static constexpr int CR = SPIN ? 16 : 32;      // rings per stage
    static constexpr int NACC = SPIN ? 64 : 32;    // FP64 sums per degree: (p2, m2) or b, per map
    static constexpr int NG = SPIN ? 2 : 1;        // accumulators (GEMMs)
    static constexpr int COL_CORR = 2 * NG * kN;   // hh buffers first: (buf * NG + g) * kN, then the
                                                   // correction pair [X | Y] of GEMM g at COL_CORR + 2 g kN
    static constexpr uint32_t TCOLS = SPIN ? 512 : 256;
};

template <int SPIN>
struct AdjSmem {
    alignas(1024) unsigned char A[kNSA][kAStage];
    alignas(1024) unsigned char B[kNSB][kBStage];
    double2 coef[2][kLB];  // (alpha, gamma) of the item's 128 steps, double-buffered over items
    alignas(8) uint64_t fullA[kNSA], emptyA[kNSA], fullB[kNSB], emptyB[kNSB];
    uint64_t accFull[2], accEmpty[2], corrEmpty, fin, coefFull[2], coefEmpty[2];
    uint32_t taddr;
    int fail;
};

struct AdjParams {
    int lmax, T, nrings;
    long long K;
    const double *x;
    const SeedParam *seed;
    const double2 *ag;      // (alpha, gamma) interleaved, packed like the alm (gamma = 0 for spin 0)
    const double *cnorm;
    const TcaItem *items;
    int nitems;
    const double2 *bst;     // segment-start states, rows [block][chunk - cl][segment][lane]
    const short *bsc;
    const unsigned char *Bt;  // ring-data tiles [M][nchunk][kBStage]
    int nchunk;
    int *err;
    unsigned long long wait_ns;
    int inject;
    int fold;               // stages per FP32 accumulation block
};

// kind::f16 instruction descriptors: FP32 accumulate, BF16 A (MN-major) and B (K-major),
// M = 128, N = 64 (one split of the ring data) or 128 (two consecutive splits).
constexpr uint32_t idesc_adj(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kLB >> 4) << 24);
}
constexpr uint32_t kIdescAdj = idesc_adj(kN), kIdescAdj2 = idesc_adj(2 * kN);
// A sub-tile, MN-major without swizzle: 8 degrees x 8 rings core matrices of 128 bytes,
// degree groups 128 bytes apart (SBO), the two 8-ring halves 2048 bytes apart (LBO).
constexpr uint32_t kALbo = 2048, kASbo = 128;
__device__ __forceinline__ uint32_t amn_off(int lgrp, int ring) {  // 16-byte row of 8 degrees
    return (uint32_t)(lgrp * kASbo + (ring & 7) * 16 + (ring >> 3) * kALbo);
}

__device__ __forceinline__ bool adj_failed(const int *f) { return __any_sync(0xffffffffu, *(volatile const int *)f != 0); }
__device__ __forceinline__ void adj_fail(int *f, int *err) {
    *(volatile int *)f = 1;
    atomicExch(err, 1);
}

__device__ __forceinline__ int item_stages(const TcaItem &q) { return q.c1 > q.c0 ? q.c1 - q.c0 : 0; }

// ---------------------------------------------------------------------------------
// producers: four 32-degree recursion chains per (ring, recursion) -> split A operand
// ---------------------------------------------------------------------------------
constexpr int kSeg = kTcaSeg;        // chains per thread: the block's 32-degree segments
constexpr int kSegLen = kLB / kSeg;  // steps per chain

// One stage of one lane: chain c runs the steps of degrees [32 c, 32 c + 32) of the block
// from its stored segment state; the four chains are independent, so their FP64 steps
// overlap.  Values of a chain in the underflow range (scale exponent < 0) are zero; such a
// chain is rescaled once per 8 steps (8 steps grow a value by far less than the 2^800 of
// headroom above the threshold, so this matches the per-step check of the FP64 kernels in
// every value that reaches FP32).  TAIL: the block runs past lmax (nrem < 128 degrees
// exist); the missing rows are zero.
template <bool TAIL>
__device__ __forceinline__ void adj_stage(const double2 *coef, int nrem, double x, double (&u1)[kSeg],
                                          double (&u2)[kSeg], int (&sc)[kSeg], unsigned char *As, int j, int k) {
    bool low[kSeg];
#pragma unroll
    for (int c = 0; c < kSeg; ++c) low[c] = __any_sync(0xffffffffu, sc[c] != 0);
#pragma unroll 1
    for (int g = 0; g < kSegLen / 8; ++g) {
        double v[kSeg][8];
#pragma unroll
        for (int c = 0; c < kSeg; ++c) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double2 cf = coef[c * kSegLen + g * 8 + q];
                const double u = fma(fma(cf.x, x, cf.y), u1[c], -u2[c]);
                u2[c] = u1[c];
                u1[c] = u;
                v[c][q] = u;
            }
        }
#pragma unroll
        for (int c = 0; c < kSeg; ++c) {
            if (low[c] && sc[c] != 0) {
#pragma unroll
                for (int q = 0; q < 8; ++q) v[c][q] = 0.0;
                if (fabs(u1[c]) > kBig) {
                    u1[c] *= kScaleDown;
                    u2[c] *= kScaleDown;
                    sc[c] += 1;
                }
            }
            if (TAIL) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (c * kSegLen + g * 8 + q >= nrem) v[c][q] = 0.0;
            }
            uint32_t pk[3][4];
            split3_pack8(v[c], pk);
            const uint32_t off = amn_off(c * (kSegLen / 8) + g, k);
#pragma unroll
            for (int sp = 0; sp < 3; ++sp) {
                const uint4 w = make_uint4(pk[sp][0], pk[sp][1], pk[sp][2], pk[sp][3]);
                *reinterpret_cast<uint4 *>(As + j * 3 * kATile + sp * kATile + off) = w;
            }
        }
    }
}

// Lane = (j, k): spin 2 runs recursion h = j (+2 for sub-tile 0, -2 for sub-tile 1) on ring
// k of the 16-ring chunk; spin 0 runs ring 16 j + k of the 32-ring chunk.  The -2
// recursion t_l = alpha_l x - gamma_l runs as w_i = (-1)^i mu_i (i = degree offset in the
// block): w_i = (alpha_i (-x) + gamma_i) w_{i-1} - w_{i-2}, the same arithmetic as the +2
// recursion with x negated and the first state value negated, without a multiply per step;
// the epilogue restores the sign (-1)^i of the row.
template <int SPIN>
__device__ void adj_producer(const AdjParams &p, AdjSmem<SPIN> &sm, int w, int lane) {
    using C = AdjCfg<SPIN>;
    const int j = lane >> 4, k = lane & 15;
    const bool neg = SPIN && j == 1;
    unsigned gc = 0, n = 0;  // stages and items of this CTA so far
    bool ok = true;
    for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x, ++n) {
        if (adj_failed(&sm.fail)) break;
        const TcaItem q = p.items[it];
        const int nstg = item_stages(q);
        const int lmin = __ldg(&p.seed[q.m].lmin);
        const int nst = p.lmax - lmin + 1;
        const int i0 = q.lb * kLB;
        const int nrem = nst - i0;
        const int cb = n & 1;
        if (!mbar_wait_warp(&sm.coefFull[cb], (n >> 1) & 1u, p.wait_ns)) {
            ok = false;
            break;
        }
        // segment states of this lane for stage s, loaded one stage of this warp ahead so the
        // memory latency overlaps the previous stage
        auto load_state = [&](int s, double &x, double (&u1)[kSeg], double (&u2)[kSeg], int (&sc)[kSeg]) {
            const int c = q.c0 + s;
            const int t = SPIN ? c * C::CR + k : c * C::CR + lane;
            x = 0.0;
#pragma unroll
            for (int g = 0; g < kSeg; ++g) {
                u1[g] = u2[g] = 0.0;
                sc[g] = 0;
            }
            if (s < nstg && t < p.T) {
                x = __ldg(&p.x[t]);
                if (neg) x = -x;
                const long long row = q.soff + (long long)(c - q.cl) * (kSeg * 32) + lane;
#pragma unroll
                for (int g = 0; g < kSeg; ++g) {
                    const double2 st = p.bst[row + g * 32];
                    u1[g] = neg ? -st.x : st.x;
                    u2[g] = st.y;
                    sc[g] = p.bsc[row + g * 32];
                }
            }
        };
        double xn, u1n[kSeg], u2n[kSeg];
        int scn[kSeg];
        load_state(w, xn, u1n, u2n, scn);
        for (int s = w; s < nstg; s += kNP) {
            const unsigned g = gc + (unsigned)s;
            const int sA = g % kNSA;
            double x = xn, u1[kSeg], u2[kSeg];
            int sc[kSeg];
#pragma unroll
            for (int c = 0; c < kSeg; ++c) {
                u1[c] = u1n[c];
                u2[c] = u2n[c];
                sc[c] = scn[c];
            }
            load_state(s + kNP, xn, u1n, u2n, scn);
            if (g >= (unsigned)kNSA && !mbar_wait_warp(&sm.emptyA[sA], ((g / kNSA) - 1u) & 1u, p.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();  // the stage's previous MMAs are complete before it is overwritten
            unsigned char *As = sm.A[sA];
            if (nrem >= kLB)
                adj_stage<false>(sm.coef[cb], nrem, x, u1, u2, sc, As, j, k);
            else
                adj_stage<true>(sm.coef[cb], nrem, x, u1, u2, sc, As, j, k);
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&sm.fullA[sA]);
        }
        if (!ok) break;
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.coefEmpty[cb]);  // this warp is done with the item's coefficients
        gc += (unsigned)nstg;
    }
    if (!ok) adj_fail(&sm.fail, p.err);
}

// ---------------------------------------------------------------------------------
// loader: the item's recursion coefficients, then one bulk copy of the chunk's
// ring-data tiles per stage
// ---------------------------------------------------------------------------------
template <int SPIN>
__device__ void adj_loader(const AdjParams &p, AdjSmem<SPIN> &sm, int lane) {
    if (p.inject == kInjectStall) return;  // test hook: no stage is ever published
    if (lane == 0) {  // one thread issues every copy
        unsigned n = 0;
        int sB = 0;
        uint32_t phB = 0;  // parity of the current round of B stages
        bool ok = true, first = true;
        for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x, ++n) {
            if (*(volatile int *)&sm.fail) break;
            const TcaItem q = p.items[it];
            const int nstg = item_stages(q);
            const int cb = n & 1;
            const unsigned char *tiles = p.Bt + ((size_t)q.m * p.nchunk + q.c0) * kBStage;
            (void)JHTB_IN(q.c0 + nstg - 1, p.nchunk, 402);  // the item's tiles lie inside its order's row
            for (int s = 0; s < min(kPrefetch, nstg); ++s) bulk_prefetch_l2(tiles + (size_t)s * kBStage, kBStage);
            if (n >= 2 && !mbar_wait(&sm.coefEmpty[cb], ((n >> 1) - 1u) & 1u, p.wait_ns)) {
                ok = false;
                break;
            }
            const int lmin = __ldg(&p.seed[q.m].lmin);
            const int i0 = q.lb * kLB;
            const uint32_t bytes = (uint32_t)min(kLB, p.lmax - lmin + 1 - i0) * 16u;
            mbar_arrive_tx(&sm.coefFull[cb], bytes);
            bulk_g2s(sm.coef[cb], p.ag + alm_index(lmin, q.m, p.lmax) + i0, bytes, &sm.coefFull[cb]);
            for (int s = 0; s < nstg; ++s) {
                // the stage's previous round has been consumed (the first round starts free)
                if (!first && !mbar_wait(&sm.emptyB[sB], phB ^ 1u, p.wait_ns)) {
                    ok = false;
                    break;
                }
                if (s + kPrefetch < nstg) bulk_prefetch_l2(tiles + (size_t)(s + kPrefetch) * kBStage, kBStage);
                mbar_arrive_tx(&sm.fullB[sB], kBStage);
                bulk_g2s(sm.B[sB], tiles + (size_t)s * kBStage, kBStage, &sm.fullB[sB]);
                if (++sB == kNSB) {
                    sB = 0;
                    phB ^= 1u;
                    first = false;
                }
            }
        }
        if (!ok) adj_fail(&sm.fail, p.err);
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------------
// MMA warp
// ---------------------------------------------------------------------------------
template <int SPIN>
__device__ void adj_mma(const AdjParams &p, AdjSmem<SPIN> &sm, uint32_t tbase, int lane) {
    using C = AdjCfg<SPIN>;
    if (lane == 0) {  // one thread waits and issues; stage indices and parities are counters
        unsigned bk = 0, ncorr = 0;
        int sA = 0, sB = 0;
        uint32_t phA = 0, phB = 0;
        bool ok = true;
        const uint64_t dA0 = smem_desc(sm.A[0], kALbo, kASbo), dB0 = smem_desc(sm.B[0], 128, 256);
        for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x) {
            if (*(volatile int *)&sm.fail) break;
            const TcaItem q = p.items[it];
            const int nstg = item_stages(q);
            int fcount = 0;  // stages of the current FP32 accumulation block so far
            for (int s = 0; s < nstg; ++s) {
                const bool bstart = fcount == 0;
                const bool bend = fcount == p.fold - 1 || s == nstg - 1;
                const unsigned kb = bk & 1u;
                if (!mbar_wait(&sm.fullB[sB], phB, p.wait_ns) || !mbar_wait(&sm.fullA[sA], phA, p.wait_ns) ||
                    (bstart && bk >= 2 && !mbar_wait(&sm.accEmpty[kb], ((bk >> 1) - 1u) & 1u, p.wait_ns)) ||
                    (s == 0 && ncorr > 0 && !mbar_wait(&sm.corrEmpty, (ncorr - 1u) & 1u, p.wait_ns))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const int gg = SPIN ? jj : 0;  // accumulator of this sub-tile
                    const uint32_t dh = tbase + (uint32_t)((kb * C::NG + gg) * kN);
                    const uint32_t dc = tbase + (uint32_t)(C::COL_CORR + gg * 2 * kN);
                    // descriptors: the address field (bits 0-13, bytes / 16) advanced from the
                    // first stage's; shared-memory offsets stay far below 2^18 bytes
                    const uint64_t a0 = dA0 + (uint64_t)((sA * kAStage + jj * 3 * kATile) >> 4);
                    const uint64_t a1 = a0 + (kATile >> 4), a2 = a0 + (2 * kATile >> 4);
                    const uint64_t c0 = dB0 + (uint64_t)((sB * kBStage + jj * 3 * kBTile) >> 4);
                    const uint64_t c1 = c0 + (kBTile >> 4);
                    // first write of each accumulator starts it at zero
                    const uint32_t acc_h = (bstart && (SPIN || jj == 0)) ? 0u : 1u;
                    const uint32_t acc_c = (s == 0 && (SPIN || jj == 0)) ? 0u : 1u;
                    umma_f16_ss(dh, a0, c0, kIdescAdj, acc_h);   // hh
                    umma_f16_ss(dc, a0, c1, kIdescAdj2, acc_c);  // [hm | hl]: B = [m | l] splits
                    umma_f16_ss(dc, a1, c0, kIdescAdj2, 1u);     // [mh | mm]: B = [h | m] splits
                    umma_f16_ss(dc, a2, c0, kIdescAdj, 1u);      // lh into the first half
                }
                umma_commit(&sm.emptyA[sA]);
                umma_commit(&sm.emptyB[sB]);
                if (bend) umma_commit(&sm.accFull[kb]);
                if (++sA == kNSA) {
                    sA = 0;
                    phA ^= 1u;
                }
                if (++sB == kNSB) {
                    sB = 0;
                    phB ^= 1u;
                }
                if (bend) {
                    ++bk;
                    fcount = 0;
                } else {
                    ++fcount;
                }
            }
            if (nstg > 0) ++ncorr;
        }
        if (!ok) adj_fail(&sm.fail, p.err);
        // every issued MMA has completed before tensor memory is released
        umma_commit(&sm.fin);
        if (!mbar_wait(&sm.fin, 0u, p.wait_ns)) adj_fail(&sm.fail, p.err);
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------------
// epilogue: fold the block sums, write the item's a_lm
// ---------------------------------------------------------------------------------
// Adds this lane's (degree's) half-grid sums over all 64 columns of the FP32 accumulators
// at tensor-memory addresses tP (spin 2: D+, spin 0: D) and tM (D-) into the FP64 sums,
// held in registers (every index is fixed at compile time).
template <int SPIN>
__device__ __forceinline__ void adj_fold(double (&acc)[AdjCfg<SPIN>::NACC], uint32_t tP, uint32_t tM, float sgn) {
#pragma unroll
    for (int col = 0; col < kN; col += 8) {
        float vp[8];
        tmem_ld8(tP + (uint32_t)col, vp);
        if (SPIN) {
            float vm[8];
            tmem_ld8(tM + (uint32_t)col, vm);
#pragma unroll
            for (int e = 0; e < 2; ++e) {  // two maps of 4 columns each
                const int b = col / 4 + e;
                const float *P = vp + 4 * e, *Mv = vm + 4 * e;
                // p2 = D+[Vpn] + s D-[Sp],  m2 = D-[Vmn] + s D+[Sm], where the accumulator
                // holds s D- (the producers' sign substitution), s = (-1)^row
                acc[4 * b + 0] += (double)P[0] + (double)Mv[2];
                acc[4 * b + 1] += (double)P[1] + (double)Mv[3];
                acc[4 * b + 2] += (double)sgn * ((double)Mv[0] + (double)P[2]);
                acc[4 * b + 3] += (double)sgn * ((double)Mv[1] + (double)P[3]);
            }
        } else {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int b = col / 4 + e;
                const float *P = vp + 4 * e;
                acc[2 * b + 0] += (double)P[0] + (double)(sgn * P[2]);
                acc[2 * b + 1] += (double)P[1] + (double)(sgn * P[3]);
            }
        }
    }
}

template <int SPIN>
__device__ void adj_epilogue(const AdjParams &p, AdjSmem<SPIN> &sm, double2 *__restrict__ alm, int nb,
                             uint32_t tbase, int warp, int lane) {
    using C = AdjCfg<SPIN>;
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;  // degree offset in the block = tensor-memory lane
    const uint32_t tl = tbase + ((uint32_t)(quarter * 32) << 16);
    double acc[C::NACC];
    unsigned bk = 0;
    bool ok = true;
    for (int it = blockIdx.x; it < p.nitems && ok; it += gridDim.x) {
        if (adj_failed(&sm.fail)) break;
        const TcaItem q = p.items[it];
        const int nstg = item_stages(q);
        const int nfb = (nstg + p.fold - 1) / p.fold;
        const int lmin = __ldg(&p.seed[q.m].lmin);
        const int l = lmin + q.lb * kLB + row;
        const float sgn = (row & 1) ? -1.0f : 1.0f;  // (-1)^(l - lmin): blocks start at even offsets
#pragma unroll
        for (int v = 0; v < C::NACC; ++v) acc[v] = 0.0;
        for (int fb = 0; fb < nfb; ++fb) {
            const unsigned kb = bk & 1u;
            if (!mbar_wait_warp(&sm.accFull[kb], (bk >> 1) & 1u, p.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t hP = tl + (uint32_t)((kb * C::NG + 0) * kN);
            const uint32_t hM = tl + (uint32_t)((kb * C::NG + (SPIN ? 1 : 0)) * kN);
            adj_fold<SPIN>(acc, hP, hM, sgn);
            if (fb == nfb - 1) {  // the item's correction sums: both halves [X | Y] of each GEMM
                const uint32_t cP = tl + (uint32_t)C::COL_CORR, cM = tl + (uint32_t)(C::COL_CORR + (SPIN ? 2 * kN : 0));
                adj_fold<SPIN>(acc, cP, cM, sgn);
                adj_fold<SPIN>(acc, cP + kN, cM + kN, sgn);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&sm.accEmpty[kb]);
                if (fb == nfb - 1) mbar_arrive(&sm.corrEmpty);
            }
            ++bk;
        }
        if (!ok) break;
        // outputs: a_lm of this degree for every map of the group (zero for an item without
        // live rings); spin 2: E = (-p2 - m2) c / 2, B = i (p2 - m2) c / 2 (healpix.py:353-354)
        if (l <= p.lmax) {
            const long long idx = alm_index(l, q.m, p.lmax);
            const bool in = JHTB_IN(idx, p.K, 401);
            const double c = in ? __ldg(&p.cnorm[idx]) : 0.0;
#pragma unroll
            for (int b = 0; b < kTcaMaps; ++b) {
                if (b >= nb || !in) continue;
                if (SPIN) {
                    const double pr = c * acc[4 * b + 0], pi = c * acc[4 * b + 1];
                    const double mr = c * acc[4 * b + 2], mi = c * acc[4 * b + 3];
                    alm[((size_t)b * 2) * p.K + idx] = make_double2(0.5 * (-pr - mr), 0.5 * (-pi - mi));
                    alm[((size_t)b * 2 + 1) * p.K + idx] = make_double2(0.5 * (-(pi - mi)), 0.5 * (pr - mr));
                } else {
                    alm[(size_t)b * p.K + idx] = make_double2(c * acc[2 * b], c * acc[2 * b + 1]);
                }
            }
        }
        // degrees below lmin (spin 2, m < 2) are zero
        if (q.lb == 0 && row < lmin - q.m) {
            const long long idx = alm_index(q.m + row, q.m, p.lmax);
            for (int b = 0; b < nb; ++b)
                for (int cc = 0; cc < (SPIN ? 2 : 1); ++cc)
                    alm[((size_t)b * (SPIN ? 2 : 1) + cc) * p.K + idx] = make_double2(0.0, 0.0);
        }
    }
    if (!ok) adj_fail(&sm.fail, p.err);
}

template <int SPIN>
__global__ void __launch_bounds__(kThreads, 1)
    tc_adjoint_kernel(AdjParams p, double2 *__restrict__ alm, int nb) {
    using C = AdjCfg<SPIN>;
    using S = AdjSmem<SPIN>;
    extern __shared__ unsigned char smem_raw[];
    S &sm = *reinterpret_cast<S *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == kWMma) {
        tmem_alloc(&sm.taddr, C::TCOLS);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kNSA; ++s) {
            mbar_init(&sm.fullA[s], 1);
            mbar_init(&sm.emptyA[s], 1);
        }
        for (int s = 0; s < kNSB; ++s) {
            mbar_init(&sm.fullB[s], 1);
            mbar_init(&sm.emptyB[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.accFull[b], 1);
            mbar_init(&sm.accEmpty[b], 4);
        }
        mbar_init(&sm.corrEmpty, 4);
        mbar_init(&sm.fin, 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.coefFull[b], 1);
            mbar_init(&sm.coefEmpty[b], kNP);
        }
        sm.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sm.taddr;
    if (warp < kNP) {
        adj_producer<SPIN>(p, sm, warp, lane);
    } else if (warp == kWLoad) {
        adj_loader<SPIN>(p, sm, lane);
    } else if (warp == kWMma) {
        adj_mma<SPIN>(p, sm, tbase, lane);
    } else {
        adj_epilogue<SPIN>(p, sm, alm, nb, tbase, warp, lane);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kWMma) tmem_dealloc(tbase, C::TCOLS);
}

// ---------------------------------------------------------------------------------
// ring-data tiles: FP64 ring spectra of a 16-map group -> BF16x3 B operands per
// (order, ring chunk), in the exact shared-memory layout the MMA reads
// ---------------------------------------------------------------------------------
template <int SPIN>
__global__ void __launch_bounds__(256) adj_prep_kernel(int lmax, int T, int nrings, int M, const SeedParam *__restrict__ seed,
                                                       const double2 *__restrict__ F, int nb, int nchunk,
                                                       unsigned char *__restrict__ Bt) {
    __shared__ __align__(16) unsigned char tile[kBStage];
    const long long blk = blockIdx.x;
    const int c = (int)(blk % nchunk), m = (int)(blk / nchunk);
    const int k = threadIdx.x & 15, b = threadIdx.x >> 4;  // ring in the sub-tile, map
    const size_t fmap = (size_t)(SPIN ? 2 : 1) * nrings * M;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        double col[4] = {0.0, 0.0, 0.0, 0.0};
        const int t = SPIN ? c * 16 + k : c * 32 + j * 16 + k;
        if (t < T && b < nb) {
            const int rs = nrings - 1 - t;
            const bool south = t < T - 1;
            if (SPIN) {
                const double ssign = ((m + seed[m].lmin) & 1) ? -1.0 : 1.0;
                // GEMM + (j = 0): [Vpn | s Sm];  GEMM - (j = 1): [Vmn | s Sp]
                const double2 *Fn = F + (size_t)b * fmap + (size_t)j * nrings * M;
                const double2 *Fs = F + (size_t)b * fmap + (size_t)(1 - j) * nrings * M;
                const double2 vn = Fn[(size_t)t * M + m];
                const double2 vs = south ? Fs[(size_t)rs * M + m] : make_double2(0.0, 0.0);
                col[0] = vn.x;
                col[1] = vn.y;
                col[2] = ssign * vs.x;
                col[3] = ssign * vs.y;
            } else {
                const double2 *Fb = F + (size_t)b * fmap;
                const double2 vn = Fb[(size_t)t * M + m];
                const double2 vs = south ? Fb[(size_t)rs * M + m] : make_double2(0.0, 0.0);
                col[0] = vn.x;
                col[1] = vn.y;
                col[2] = vs.x;
                col[3] = vs.y;
            }
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            __nv_bfloat16 vh, vm, vl;
            split3(col[e], vh, vm, vl);
            const uint32_t off = kmaj_off(4 * b + e, k);
            *reinterpret_cast<__nv_bfloat16 *>(tile + j * 3 * kBTile + 0 * kBTile + off) = vh;
            *reinterpret_cast<__nv_bfloat16 *>(tile + j * 3 * kBTile + 1 * kBTile + off) = vm;
            *reinterpret_cast<__nv_bfloat16 *>(tile + j * 3 * kBTile + 2 * kBTile + off) = vl;
        }
    }
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(Bt + (size_t)blk * kBStage);
    const uint4 *src = reinterpret_cast<const uint4 *>(tile);
    for (int i = threadIdx.x; i < kBStage / 16; i += 256) dst[i] = src[i];
}

// ---------------------------------------------------------------------------------
// plan creation: the recursion state at the start of every 32-degree segment of every
// 128-degree block, for the rings of the block's live chunks (the producer lane layout)
// ---------------------------------------------------------------------------------
template <int SPIN>
__global__ void __launch_bounds__(128) tca_segment_state_kernel(int lmax, int T, const double *__restrict__ x,
                                                                const double *__restrict__ logsin,
                                                                const double *__restrict__ logch,
                                                                const double *__restrict__ logsh,
                                                                const SeedParam *__restrict__ seed,
                                                                const double *__restrict__ alpha,
                                                                const double *__restrict__ gamma,
                                                                const int *__restrict__ blk_off,
                                                                const int *__restrict__ blk_cl,
                                                                const long long *__restrict__ blk_soff,
                                                                double2 *__restrict__ bst, short *__restrict__ bsc) {
    constexpr int CR = SPIN ? 16 : 32;
    const int t = blockIdx.x * 128 + threadIdx.x;
    const int h = blockIdx.y, m = blockIdx.z;
    if (t >= T) return;
    const SeedParam sd = seed[m];
    const long long b0 = alm_index(sd.lmin, m, lmax);
    const int nst = lmax - sd.lmin + 1;
    const double xt = x[t];
    double mant = 0.0;
    int sc = 0;
    const double lg = SPIN ? seed_log2(sd, h, logch[t], logsh[t]) : seed_log0(sd, m, logsin[t]);
    make_seed(lg, sd.sign[h], mant, sc);
    double u1 = 0.0, u2 = -mant;
    const double gsg = h ? -1.0 : 1.0;
    const int c = t / CR;
    const int lane = SPIN ? h * 16 + (t & 15) : (t & 31);
    const int nblk = (nst + kLB - 1) / kLB;
    for (int lb = 0; lb < nblk; ++lb) {
        const int blk = blk_off[m] + lb;
        const int cl = blk_cl[blk];
        const long long row = blk_soff[blk] + (long long)(c - cl) * (kTcaSeg * 32) + lane;
        for (int g = 0; g < kTcaSeg; ++g) {
            const int i0 = lb * kLB + g * (kLB / kTcaSeg);
            if (c >= cl) {
                bst[row + g * 32] = i0 < nst ? make_double2(u1, u2) : make_double2(0.0, 0.0);
                bsc[row + g * 32] = i0 < nst ? (short)max(sc, -32768) : (short)0;
            }
            const int i1 = min(nst, i0 + kLB / kTcaSeg);
            for (int i = i0; i < i1; ++i) {
                const double tt = fma(alpha[b0 + i], xt, SPIN ? gsg * gamma[b0 + i] : 0.0);
                double u = fma(tt, u1, -u2);
                double prev = u1;
                rescale(u, prev, sc);
                u2 = prev;
                u1 = u;
            }
        }
    }
}

}  // namespace

JHTB_DEBUG_ACCESSOR(tc_adjoint)

int launch_tca_block_states(const Plan &p, cudaStream_t s) {
    const dim3 grid((p.T + 127) / 128, p.spin ? 2 : 1, p.M);
    if (p.spin)
        tca_segment_state_kernel<2><<<grid, 128, 0, s>>>(p.lmax, p.T, p.d_x, p.d_logsin, p.d_logch, p.d_logsh, p.d_seed,
                                                          p.d_alpha, p.d_gamma, p.d_tca_blk_off, p.d_tca_blk_cl,
                                                          p.d_tca_blk_soff, p.d_tca_st, p.d_tca_sc);
    else
        tca_segment_state_kernel<0><<<grid, 128, 0, s>>>(p.lmax, p.T, p.d_x, p.d_logsin, p.d_logch, p.d_logsh, p.d_seed,
                                                          p.d_alpha, p.d_gamma, p.d_tca_blk_off, p.d_tca_blk_cl,
                                                          p.d_tca_blk_soff, p.d_tca_st, p.d_tca_sc);
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

template <int SPIN>
static int launch_tca_t(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s) {
    auto k = tc_adjoint_kernel<SPIN>;
    const int smem = (int)sizeof(AdjSmem<SPIN>) + 1024;
    int dev = 0, nsm = 148;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    AdjParams q;
    q.lmax = p.lmax;
    q.T = p.T;
    q.nrings = p.nrings;
    q.K = p.K;
    q.x = p.d_x;
    q.seed = p.d_seed;
    q.ag = p.d_ag;
    q.cnorm = p.d_cnorm;
    q.items = p.d_tca_items;
    q.nitems = p.tca_nitems;
    q.bst = p.d_tca_st;
    q.bsc = p.d_tca_sc;
    q.Bt = p.d_tca_B;
    q.nchunk = p.tca_nchunk;
    q.err = p.d_err;
    q.wait_ns = p.tc_wait_ns;
    q.inject = p.inject;
    q.fold = std::max(1, p.tca_fold / (SPIN ? 16 : 32));
    const size_t fmap = (size_t)p.ncomp * p.nrings * p.M, amap = (size_t)p.ncomp * p.K;
    for (int b0 = 0; b0 < nb; b0 += kTcaMaps) {
        const int cnt = std::min(kTcaMaps, nb - b0);
        const long long nblk = (long long)p.M * p.tca_nchunk;
        adj_prep_kernel<SPIN><<<(unsigned)nblk, 256, 0, s>>>(p.lmax, p.T, p.nrings, p.M, p.d_seed, F + b0 * fmap, cnt,
                                                              p.tca_nchunk, p.d_tca_B);
        JHTB_CUDA_TRY(cudaGetLastError());
        k<<<nsm, kThreads, smem, s>>>(q, alm + b0 * amap, cnt);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    return JHTB_OK;
}

int launch_tc_adjoint(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    return p.spin ? launch_tca_t<2>(p, F, alm, nb, s) : launch_tca_t<0>(p, F, alm, nb, s);
}

}  // namespace jhtb
