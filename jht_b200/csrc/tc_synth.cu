// Batched mixed-precision synthesis on the 5th-generation tensor cores (tcgen05).
//
// For one order m and a tile of 128 half-grid rings the l-contraction of B maps is a
// GEMM:  F[t, n] = sum_l mu_l(t) C[l, n],  t = ring (M = 128), l (K, 16 per MMA),
// n = (map, component) (N = 4 B per GEMM).  Spin 2 runs two GEMMs, one per
// recursion (+2 / -2):  D+ = Lambda+ [cp, s cm],  D- = Lambda- [cm, s cp], with
// s = (-1)^(l - lmin) folded into the B rows; jht's four half-grid sums
// (_recursion.py:512-543) are the four column pairs.  Spin 0 runs the same
// contraction for two 128-ring halves of a 256-ring tile, columns [a, s a]
// (_recursion.py:441-469).
//
// The coefficient operand does not depend on the ring, so tc_prep_kernel builds it once
// per launch and map group: for every (order, chunk of 16 degrees) the BF16x3 split of
// c_l a_lm with the N/S sign pattern, in the exact shared-memory layout the MMA reads,
// followed by the chunk's recursion coefficients.  Items are ordered by m, so the CTAs
// working at one time read the same orders' chunks from L2.
//
// The CTA is warp-specialised and its roles meet only at mbarriers:
//   producer warps (one thread per A row = tensor-memory lane and recursion chain) run
//     the FP64 recursion (same normalised form and start states as the FP64 kernels),
//     round mu to FP32, split it into three BF16 parts and store their rows of the A
//     operands straight into tensor memory (tcgen05.st), so the six split products never
//     re-read A through shared memory; every 256 degrees they fold the FP32 block sums
//     into FP64 accumulators in shared memory and at the item's end write the spectra;
//   one loader warp: a bulk copy per chunk of the prepared tiles and coefficients;
//   one MMA warp issues the six split products hh, hm, mh, hl, lh, mm per GEMM
//     (kind::f16, A from tensor memory, B from shared memory, FP32 accumulators in
//     tensor memory) and commits each stage back to its producers.
// hh accumulates in a double-buffered block accumulator (FP32 rounding acts on <= 256
// terms, and the MMAs of the next block run while a block is folded); the five smaller
// products (relative size <= 2^-8) accumulate over the whole item.  Every wait is
// bounded; on timeout the kernel records an error, every role leaves its loop, and
// tensor memory is released after the last MMA has drained.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"
#include "tc_common.cuh"

namespace jhtb {
namespace {
using namespace tc;

constexpr int kTcRows = 128;     // = MMA M = rings per tile
constexpr int kTcK = 16;         // l steps per chunk = MMA K (BF16)
#ifndef JHTB_TC_NSA
#define JHTB_TC_NSA 2
#endif

struct TcParams {
    int lmax, T, nrings, M, nside;
    long long K;
    const double *x;
    const SeedParam *seed;
    int ntiles;  // item tiles per m (128 rings for spin 2, 256 for spin 0)
    int norder;  // entries of order (the items inside the plan's ring range)
    const int *lw;
    const double2 *st;
    const int *stsc;
    const int *order;
    const int *cbase;            // [M] first prepared chunk of each order
    const unsigned char *Bt;     // prepared chunks [chunk][BBYTES]
    int *err;
    unsigned long long wait_ns;  // time limit of every bounded wait
    int inject;                  // fault injection for tests (kInjectStall: the loader publishes nothing)
    int flush;                   // chunks of 16 degrees per FP32 accumulation block
};

template <int SPIN, int BM>
struct TcCfg {
    static constexpr int NG = 2;                    // GEMMs per chunk = recursion chains per producer thread
    static constexpr int NBT = SPIN ? 2 : 1;        // B tiles per chunk (spin 0: both GEMMs share one)
    static constexpr int N = 4 * BM;                // columns per GEMM
    static constexpr int CH = BM >= 16 ? 1 : 2;     // recursion chains (GEMMs) per producer thread
    static constexpr int NPW = 4 * NG / CH;         // producer warps: one thread per A row (TMEM lane) and chain
    static constexpr int LOAD_WARP = NPW;
    static constexpr int MMA_WARP = NPW + 1;
    static constexpr int NTHREADS = (NPW + 2) * 32;
    static constexpr int NSA = JHTB_TC_NSA;         // A stages (in tensor memory)
    static constexpr int NSB = 6;                   // B stages (with the chunk's coefficients): deep enough to cover the bulk copies' latency
    static constexpr int BTILE = N * kTcK * 2;
    static constexpr int BBYTES = NBT * 3 * BTILE + kTcK * 16;  // tiles, then 16 (alpha, gamma) pairs
    static constexpr int BSTRIDE = (BBYTES + 1023) / 1024 * 1024;
    static constexpr int ACOLS = kTcK / 2;          // tensor-memory columns of one A row (16 BF16)
    // tensor memory: hh block sums [buffer][GEMM], correction sums [GEMM], then the A stages
    static constexpr int COL_CORR = 2 * NG * N;
    static constexpr int COL_A = 3 * NG * N;
    static constexpr int NCOL = COL_A + NSA * NG * 3 * ACOLS;
    static constexpr uint32_t TCOLS =
        NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : (NCOL <= 256 ? 256 : 512)));
    static_assert(NCOL <= 512, "tensor memory of one SM");
    static_assert(BBYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
};

template <int SPIN, int BM>
struct TcSmem {
    using C = TcCfg<SPIN, BM>;
    alignas(1024) unsigned char B[C::NSB][C::BSTRIDE];
    double acc[C::NG][C::N][kTcRows];  // FP64 sums [GEMM][column][row]: a warp touches 32 consecutive words
    alignas(8) uint64_t fullA[C::NSA], emptyA[C::NSA], fullB[C::NSB], emptyB[C::NSB];
    uint64_t accFull[2], accEmpty[2], corrEmpty, fin;
    uint32_t taddr;
    int fail;
};

// One (m, ring tile) work item, as every role of the CTA derives it: the chunks run on a
// grid of 16 degrees from lmin; the first live chunk c0 holds the tile's start degree at
// offset `skip` (even), the steps before it are dead (zero) for every ring of the tile.
struct TcItem {
    int m, tile, lmin, nst, i_start, c0, nck, skip;
};

__device__ __forceinline__ TcItem tc_item_of(const TcParams &p, int item) {
    TcItem q;
    q.m = item / p.ntiles;
    q.tile = item - q.m * p.ntiles;
    q.lmin = __ldg(&p.seed[q.m].lmin);
    q.nst = p.lmax - q.lmin + 1;
    q.i_start = __ldg(&p.lw[item]) - q.lmin;
    q.c0 = q.i_start / kTcK;
    q.skip = q.i_start - q.c0 * kTcK;
    q.nck = q.i_start < q.nst ? (q.nst + kTcK - 1) / kTcK - q.c0 : 0;
    return q;
}

// Whether any role has recorded a failure; one verdict per warp (see mbar_wait_warp).
__device__ __forceinline__ bool tc_failed(const int *f) {
    return __any_sync(0xffffffffu, *(volatile const int *)f != 0);
}
__device__ __forceinline__ void tc_fail(int *f, int *err) {
    *(volatile int *)f = 1;
    atomicExch(err, 1);
}

// One step of one recursion, t = alpha_l x + gamma_l precomputed, with the
// scaled-phase bookkeeping (SLOW) or without.
template <bool SLOW>
__device__ __forceinline__ double tc_step(double t, double &u1, double &u2, int &sc) {
    double u = fma(t, u1, -u2);
    double prev = u1;
    if (SLOW) rescale(u, prev, sc);
    u2 = prev;
    u1 = u;
    return (SLOW && sc != 0) ? 0.0 : u;
}

// 16 steps of this thread's CH recursion chains (GEMMs j0 .. j0 + CH - 1), split into
// BF16 parts and stored as its row (= its tensor-memory lane) of those GEMMs' three A
// operands: tA[c] is the lane-offset tensor-memory address of chain c's split-0 operand,
// the splits following at ACOLS columns apart.  Spin 2: GEMM 0 is the +2 recursion
// (+gamma), GEMM 1 the -2 one (-gamma), same ring; spin 0: the GEMMs are rings row and
// 128 + row of the item tile (gamma = 0).  Past the end of the column the
// coefficients are zero, which keeps the state bounded (u_k = -u_{k-2}) while the B
// rows there are zero; rows past the last ring start from a zero state and stay zero.
// In the item's first chunk (FIRST) the `skip` steps before the start state are zero and
// leave the state untouched.  Each half-chunk first loads its eight coefficient pairs
// and forms the multipliers t = alpha x +- gamma, so only one FMA per step stays on the
// dependency chain.
template <bool SLOW, bool FIRST, int CH>
__device__ __forceinline__ void tc_chunk(const double2 *coef, const double (&x)[CH], double (&u1)[CH],
                                         double (&u2)[CH], int (&sc)[CH], const uint32_t (&tA)[CH], int skip,
                                         unsigned long long gflip) {
    constexpr uint32_t AC = kTcK / 2;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        double t[CH][8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 a = coef[half * 8 + k];
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                // GEMM j0 + c runs the +gamma recursion when j0 + c is even, -gamma when odd:
                // gflip holds the sign bit of chain c (bit 63 - c), applied as an exact flip
                const double g = __longlong_as_double(__double_as_longlong(a.y) ^ (long long)((gflip << c) & (1ull << 63)));
                t[c][k] = fma(a.x, x[c], g);
            }
        }
        uint32_t pk[CH][3][4];
        double v[CH][8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const bool dead = FIRST && half * 8 + q < skip;
#pragma unroll
            for (int c = 0; c < CH; ++c) v[c][q] = dead ? 0.0 : tc_step<SLOW>(t[c][q], u1[c], u2[c], sc[c]);
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) split3_pack8(v[c], pk[c]);
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int sp = 0; sp < 3; ++sp)
                tmem_st4(tA[c] + sp * AC + half * 4, pk[c][sp][0], pk[c][sp][1], pk[c][sp][2], pk[c][sp][3]);
    }
}

// Rows of F for one (map, ring): north (healpix.py:250-253) and the signed south mirror.
// Spin 2: GEMM + (H = 0) holds [FpN | FmS], GEMM - (H = 1) holds [FmN | FpS].
template <int SPIN>
__device__ __forceinline__ void tc_store_F(const TcParams &p, double2 *__restrict__ F_all, int b, int H, int t, int m,
                                           int lmin, const double (&v)[4]) {
    const size_t rs = (size_t)(p.nrings - 1 - t);
    if (!JHTB_IN((long long)rs * p.M + m, (long long)p.nrings * p.M, 301)) return;
    if (SPIN) {
        const double ssign = ((m + lmin) & 1) ? -1.0 : 1.0;
        double2 *Fp = F_all + (size_t)b * 2 * p.nrings * p.M;
        double2 *Fm = Fp + (size_t)p.nrings * p.M;
        double2 *Fn = H ? Fm : Fp, *Fs = H ? Fp : Fm;
        Fn[(size_t)t * p.M + m] = make_double2(v[0], v[1]);
        if (t < p.T - 1) Fs[rs * p.M + m] = make_double2(ssign * v[2], ssign * v[3]);
    } else {
        double2 *F = F_all + (size_t)b * p.nrings * p.M;
        F[(size_t)t * p.M + m] = make_double2(v[0], v[1]);
        if (t < p.T - 1) F[rs * p.M + m] = make_double2(v[2], v[3]);
    }
}

// acc[col + e][row] (+)= the 32 FP32 block sums at tensor-memory address ta: one tensor-
// memory load and wait for the 32 columns, then their 32 shared-memory sums.
__device__ __forceinline__ void fold32(double *accj, uint32_t ta, int col, int row, bool first) {
    float v[32];
    tmem_ld32(ta, v);
#pragma unroll
    for (int e = 0; e < 32; ++e) {
        double *a = accj + (size_t)(col + e) * kTcRows + row;
        *a = first ? (double)v[e] : *a + (double)v[e];
    }
}

// ---------------------------------------------------------------------------------
// producer warps: recursion -> A tiles; block folds and the item's output
// ---------------------------------------------------------------------------------
template <int SPIN, int BM>
__device__ void tc_producer(const TcParams &p, TcSmem<SPIN, BM> &sm, double2 *__restrict__ F_all, int nb,
                            uint32_t tbase, int warp, int lane) {
    using C = TcCfg<SPIN, BM>;
    constexpr int N = C::N;
    constexpr int CH = C::CH;
    const int row = (warp & 3) * 32 + lane;  // A row = TMEM lane (warp w reaches lanes 32 (w % 4) ..)
    const int j0 = (warp >> 2) * CH;         // this thread's first GEMM
    // sign bits of gamma for the thread's chains: chain c (GEMM j0 + c) is the -gamma
    // recursion when j0 + c is odd; bit 63 - c of gflip (spin 0 has gamma = 0)
    unsigned long long gflip = 0;
#pragma unroll
    for (int c = 0; c < CH; ++c)
        if ((j0 + c) & 1) gflip |= 1ull << (63 - c);
    const uint32_t tl = tbase + ((uint32_t)((warp & 3) * 32) << 16);
    const int nitems = p.norder;
    unsigned gc = 0, bk = 0;
    bool ok = true;
    // GEMM j's ring (spin 0: two 128-ring halves of the item tile) and start-state slot
    auto ring_of = [&](int tile, int j) { return SPIN ? tile * kTcRows + row : tile * 2 * kTcRows + j * kTcRows + row; };
    auto st_of = [&](int id, int j) { return ((size_t)id * 2 + j) * kTcRows + row; };
    for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        if (tc_failed(&sm.fail)) break;
        const int id = __ldg(&p.order[it]);
        const TcItem q = tc_item_of(p, id);
        int tr[CH];
        double x[CH], u1[CH], u2[CH];
        int sc[CH];
        bool fast = true;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            tr[c] = ring_of(q.tile, j0 + c);
            const double2 st = p.st[st_of(id, j0 + c)];
            x[c] = tr[c] < p.T ? __ldg(&p.x[tr[c]]) : 0.0;
            u1[c] = st.x;
            u2[c] = st.y;
            sc[c] = tr[c] < p.T ? p.stsc[st_of(id, j0 + c)] : 0;
            fast &= sc[c] == 0;
        }
        for (int c = 0; c < q.nck; ++c, ++gc) {
            const int sA = gc % C::NSA, sB = gc % C::NSB;
            if (!mbar_wait_warp(&sm.fullB[sB], (gc / C::NSB) & 1u, p.wait_ns)) { ok = false; break; }
            if (gc >= (unsigned)C::NSA && !mbar_wait_warp(&sm.emptyA[sA], ((gc / C::NSA) - 1u) & 1u, p.wait_ns)) { ok = false; break; }
            tc_fence_after();  // the stage's previous MMAs are complete before it is overwritten
            uint32_t tA[CH];
#pragma unroll
            for (int e = 0; e < CH; ++e) tA[e] = tl + (uint32_t)(C::COL_A + (sA * C::NG + j0 + e) * 3 * C::ACOLS);
            const double2 *coef = reinterpret_cast<const double2 *>(sm.B[sB] + C::NBT * 3 * C::BTILE);
            const bool f = __all_sync(0xffffffffu, fast);
            if (c == 0)  // the first chunk: steps before the start state are dead
                tc_chunk<true, true, CH>(coef, x, u1, u2, sc, tA, q.skip, gflip);
            else if (f)
                tc_chunk<false, false, CH>(coef, x, u1, u2, sc, tA, 0, gflip);
            else
                tc_chunk<true, false, CH>(coef, x, u1, u2, sc, tA, 0, gflip);
            if (!f || c == 0) {
                fast = true;
#pragma unroll
                for (int e = 0; e < CH; ++e) fast &= sc[e] == 0;
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&sm.fullA[sA]);
                mbar_arrive(&sm.emptyB[sB]);
            }
            const bool last = c == q.nck - 1;
            if ((c % p.flush) == p.flush - 1 || last) {
                const unsigned kb = bk & 1u;
                if (!mbar_wait_warp(&sm.accFull[kb], (bk >> 1) & 1u, p.wait_ns)) { ok = false; break; }
                tc_fence_after();
                const bool first_block = c < p.flush;
#pragma unroll 1
                for (int e = 0; e < CH; ++e) {
                    const int j = j0 + e;
                    double *accj = &sm.acc[j][0][0];
                    const uint32_t th = tl + (uint32_t)((kb * C::NG + j) * N);
#pragma unroll 1
                    for (int col = 0; col < N; col += 32) fold32(accj, th + col, col, row, first_block);
                    if (last) {
                        const uint32_t tcorr = tl + (uint32_t)(C::COL_CORR + j * N);
#pragma unroll 1
                        for (int col = 0; col < N; col += 32) fold32(accj, tcorr + col, col, row, false);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&sm.accEmpty[kb]);
                    if (last) mbar_arrive(&sm.corrEmpty);
                }
                ++bk;
                if (last) {
                    // the item's spectra for every map of the group
#pragma unroll 1
                    for (int e = 0; e < CH; ++e) {
                        const int j = j0 + e, t = tr[e];
                        if (t >= p.T) continue;
                        for (int bm = 0; bm < nb; ++bm) {
                            double v[4];
#pragma unroll
                            for (int u = 0; u < 4; ++u) v[u] = sm.acc[j][4 * bm + u][row];
                            tc_store_F<SPIN>(p, F_all, bm, SPIN ? j : 0, t, q.m, q.lmin, v);
                        }
                    }
                }
            }
        }
        if (ok && q.nck == 0) {
            // no representable term in this tile: the rows are exactly zero
            const double z[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int e = 0; e < CH; ++e) {
                const int t = tr[e];
                if (t < p.T)
                    for (int bm = 0; bm < nb; ++bm) tc_store_F<SPIN>(p, F_all, bm, SPIN ? j0 + e : 0, t, q.m, q.lmin, z);
            }
        }
    }
    if (!ok) tc_fail(&sm.fail, p.err);
}

// ---------------------------------------------------------------------------------
// loader warp: one bulk copy per chunk of the prepared tiles and coefficients
// ---------------------------------------------------------------------------------
template <int SPIN, int BM>
__device__ void tc_loader(const TcParams &p, TcSmem<SPIN, BM> &sm, int lane) {
    using C = TcCfg<SPIN, BM>;
    if (p.inject == kInjectStall) return;  // test hook: no stage is ever published
    const int nitems = p.norder;
    unsigned gc = 0;
    bool ok = true;
    for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        if (tc_failed(&sm.fail)) break;
        const TcItem q = tc_item_of(p, __ldg(&p.order[it]));
        const size_t base = (size_t)__ldg(&p.cbase[q.m]) + q.c0;
        for (int c = 0; c < q.nck; ++c, ++gc) {
            const int sB = gc % C::NSB;
            if (gc >= (unsigned)C::NSB && !mbar_wait_warp(&sm.emptyB[sB], ((gc / C::NSB) - 1u) & 1u, p.wait_ns)) {
                ok = false;
                break;
            }
            if (lane == 0) {
                mbar_arrive_tx(&sm.fullB[sB], C::BBYTES);
                bulk_g2s(sm.B[sB], p.Bt + (base + c) * C::BBYTES, C::BBYTES, &sm.fullB[sB]);
            }
            __syncwarp();
        }
    }
    if (!ok) tc_fail(&sm.fail, p.err);
}

// ---------------------------------------------------------------------------------
// MMA warp: one thread issues the split products and the commits
// ---------------------------------------------------------------------------------
template <int SPIN, int BM>
__device__ void tc_mma(const TcParams &p, TcSmem<SPIN, BM> &sm, uint32_t tbase, int lane) {
    using C = TcCfg<SPIN, BM>;
    constexpr int N = C::N;
    constexpr uint32_t IDESC = idesc_bf16(kTcRows, N);
    const int nitems = p.norder;
    unsigned gc = 0, bk = 0, ncorr = 0;
    bool ok = true;
    for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        if (tc_failed(&sm.fail)) break;
        const TcItem q = tc_item_of(p, __ldg(&p.order[it]));
        for (int c = 0; c < q.nck; ++c, ++gc) {
            const int sA = gc % C::NSA, sB = gc % C::NSB;
            const bool bstart = (c % p.flush) == 0;
            const bool bend = (c % p.flush) == p.flush - 1 || c == q.nck - 1;
            const unsigned kb = bk & 1u;
            if (!mbar_wait_warp(&sm.fullA[sA], (gc / C::NSA) & 1u, p.wait_ns) ||
                !mbar_wait_warp(&sm.fullB[sB], (gc / C::NSB) & 1u, p.wait_ns) ||
                (bstart && bk >= 2 && !mbar_wait_warp(&sm.accEmpty[kb], ((bk >> 1) - 1u) & 1u, p.wait_ns)) ||
                (c == 0 && ncorr > 0 && !mbar_wait_warp(&sm.corrEmpty, (ncorr - 1u) & 1u, p.wait_ns))) {
                ok = false;
                break;
            }
            tc_fence_after();
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < C::NG; ++j) {
                    const int jb = SPIN ? j : 0;
                    const uint32_t d = tbase + (uint32_t)((kb * C::NG + j) * N);
                    const uint32_t dc = tbase + (uint32_t)(C::COL_CORR + j * N);
                    const uint32_t a0 = tbase + (uint32_t)(C::COL_A + (sA * C::NG + j) * 3 * C::ACOLS);
                    const uint32_t a1 = a0 + C::ACOLS, a2 = a0 + 2 * C::ACOLS;
                    const unsigned char *Bj = sm.B[sB] + jb * 3 * C::BTILE;
                    const uint64_t c0 = smem_desc(Bj, 128, 256), c1 = smem_desc(Bj + C::BTILE, 128, 256),
                                   c2 = smem_desc(Bj + 2 * C::BTILE, 128, 256);
                    umma_f16_ts(d, a0, c0, IDESC, bstart ? 0u : 1u);  // hh
                    umma_f16_ts(dc, a0, c1, IDESC, c == 0 ? 0u : 1u); // hm
                    umma_f16_ts(dc, a1, c0, IDESC, 1u);               // mh
                    umma_f16_ts(dc, a0, c2, IDESC, 1u);               // hl
                    umma_f16_ts(dc, a2, c0, IDESC, 1u);               // lh
                    umma_f16_ts(dc, a1, c1, IDESC, 1u);               // mm
                }
                umma_commit(&sm.emptyA[sA]);
                umma_commit(&sm.emptyB[sB]);
                if (bend) umma_commit(&sm.accFull[kb]);
            }
            __syncwarp();
            if (bend) ++bk;
        }
        if (ok && q.nck > 0) ++ncorr;
    }
    if (!ok) tc_fail(&sm.fail, p.err);
    // every issued MMA has completed before tensor memory is released
    if (lane == 0) {
        umma_commit(&sm.fin);
        if (!mbar_wait(&sm.fin, 0u, p.wait_ns)) tc_fail(&sm.fail, p.err);  // lane 0 alone
    }
    __syncwarp();
}

template <int SPIN, int BM>
__global__ void __launch_bounds__(TcCfg<SPIN, BM>::NTHREADS, 1)
    tc_synth_kernel(TcParams p, double2 *__restrict__ F_all, int nb) {
    using C = TcCfg<SPIN, BM>;
    using S = TcSmem<SPIN, BM>;
    extern __shared__ unsigned char smem_raw[];
    S &sm = *reinterpret_cast<S *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == C::MMA_WARP) {
        tmem_alloc(&sm.taddr, C::TCOLS);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < C::NSA; ++s) {
            mbar_init(&sm.fullA[s], C::NPW);
            mbar_init(&sm.emptyA[s], 1);
        }
        for (int s = 0; s < C::NSB; ++s) {
            mbar_init(&sm.fullB[s], 1);
            mbar_init(&sm.emptyB[s], 1 + C::NPW);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sm.accFull[b], 1);
            mbar_init(&sm.accEmpty[b], C::NPW);
        }
        mbar_init(&sm.corrEmpty, C::NPW);
        mbar_init(&sm.fin, 1);
        sm.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sm.taddr;
    if (warp < C::NPW) {
        tc_producer<SPIN, BM>(p, sm, F_all, nb, tbase, warp, lane);
    } else if (warp == C::LOAD_WARP) {
        tc_loader<SPIN, BM>(p, sm, lane);
    } else {
        tc_mma<SPIN, BM>(p, sm, tbase, lane);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == C::MMA_WARP) tmem_dealloc(tbase, C::TCOLS);
}

// ---------------------------------------------------------------------------------
// coefficient chunks of one map group: for every (order, chunk of 16 degrees) the B
// tiles (c_l a_lm with the N/S sign pattern, split into three BF16 parts, K-major) and
// the chunk's (alpha, gamma); one CTA of 16 x BM threads (degree, map) per chunk
// ---------------------------------------------------------------------------------
template <int SPIN, int BM>
__global__ void tc_prep_kernel(int lmax, long long K, const SeedParam *__restrict__ seed, const double *__restrict__ alpha,
                               const double *__restrict__ gamma, const double *__restrict__ cnorm,
                               const int *__restrict__ chunk_m, const int *__restrict__ cbase,
                               const double2 *__restrict__ alm_all, int nb, unsigned char *__restrict__ Bt) {
    using C = TcCfg<SPIN, BM>;
    __shared__ __align__(16) unsigned char tile[C::BBYTES];
    const int chunk = blockIdx.x;
    const int m = chunk_m[chunk];
    const int c = chunk - cbase[m];
    const int k = threadIdx.x % kTcK, bm = threadIdx.x / kTcK;
    const int lmin = seed[m].lmin;
    const int nst = lmax - lmin + 1;
    const int i = c * kTcK + k;
    const long long idx = alm_index(lmin, m, lmax) + i;
    const double sg = (i & 1) ? -1.0 : 1.0;  // (-1)^(l - lmin)
    double col[C::NBT][4];
#pragma unroll
    for (int h = 0; h < C::NBT; ++h)
#pragma unroll
        for (int e = 0; e < 4; ++e) col[h][e] = 0.0;
    if (i < nst && bm < nb) {
        const double cn = cnorm[idx];
        if (SPIN) {
            const double2 e = alm_all[((size_t)bm * 2) * K + idx], b = alm_all[((size_t)bm * 2 + 1) * K + idx];
            // cp = -(aE + i aB) c, cm = -(aE - i aB) c   (healpix.py:316-318)
            const double cpr = -(e.x - b.y) * cn, cpi = -(e.y + b.x) * cn;
            const double cmr = -(e.x + b.y) * cn, cmi = -(e.y - b.x) * cn;
            col[0][0] = cpr; col[0][1] = cpi; col[0][2] = sg * cmr; col[0][3] = sg * cmi;
            col[C::NBT - 1][0] = cmr; col[C::NBT - 1][1] = cmi; col[C::NBT - 1][2] = sg * cpr; col[C::NBT - 1][3] = sg * cpi;
        } else {
            const double2 a = alm_all[(size_t)bm * K + idx];
            col[0][0] = a.x * cn; col[0][1] = a.y * cn;
            col[0][2] = sg * a.x * cn; col[0][3] = sg * a.y * cn;
        }
    }
#pragma unroll
    for (int h = 0; h < C::NBT; ++h)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            __nv_bfloat16 vh, vm, vl;
            split3(col[h][e], vh, vm, vl);
            const uint32_t off = kmaj_off(4 * bm + e, k);
            *reinterpret_cast<__nv_bfloat16 *>(tile + (h * 3 + 0) * C::BTILE + off) = vh;
            *reinterpret_cast<__nv_bfloat16 *>(tile + (h * 3 + 1) * C::BTILE + off) = vm;
            *reinterpret_cast<__nv_bfloat16 *>(tile + (h * 3 + 2) * C::BTILE + off) = vl;
        }
    if (bm == 0) {
        double2 ag = make_double2(0.0, 0.0);
        if (i < nst) ag = make_double2(alpha[idx], SPIN ? gamma[idx] : 0.0);
        reinterpret_cast<double2 *>(tile + C::NBT * 3 * C::BTILE)[k] = ag;
    }
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(Bt + (size_t)chunk * C::BBYTES);
    const uint4 *src = reinterpret_cast<const uint4 *>(tile);
    for (int w = threadIdx.x; w < C::BBYTES / 16; w += blockDim.x) dst[w] = src[w];
}

}  // namespace

JHTB_DEBUG_ACCESSOR(tc_synth)

template <int SPIN, int BM>
static int launch_tc_synth_t(const Plan &p, const TcParams &q, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    using C = TcCfg<SPIN, BM>;
    auto k = tc_synth_kernel<SPIN, BM>;
    const int smem = (int)sizeof(TcSmem<SPIN, BM>) + 1024;
    int dev = 0, nsm = 148;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const size_t alm_map = (size_t)p.ncomp * p.K, F_map = (size_t)p.ncomp * p.nrings * p.M;
    for (int b0 = 0; b0 < nb; b0 += BM) {
        const int cnt = std::min(BM, nb - b0);
        tc_prep_kernel<SPIN, BM><<<(unsigned)p.tcs_nchunks, kTcK * BM, 0, s>>>(
            p.lmax, p.K, p.d_seed, p.d_alpha, p.d_gamma, p.d_cnorm, p.d_tcs_chunk_m, p.d_tcs_cbase, alm + b0 * alm_map, cnt,
            p.d_tcs_B);
        JHTB_CUDA_TRY(cudaGetLastError());
        // one CTA per SM (tensor memory and shared memory both size it so)
        k<<<nsm, C::NTHREADS, smem, s>>>(q, F + b0 * F_map, cnt);
        JHTB_CUDA_TRY(cudaGetLastError());
    }
    return JHTB_OK;
}

int launch_tc_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    TcParams q;
    q.lmax = p.lmax;
    q.T = p.T;
    q.nrings = p.nrings;
    q.M = p.M;
    q.nside = p.nside;
    q.K = p.K;
    q.x = p.d_x;
    q.seed = p.d_seed;
    q.ntiles = p.tc_ntiles;
    q.lw = p.d_tc_lw;
    q.st = p.d_tc_st;
    q.stsc = p.d_tc_stsc;
    q.order = p.d_tc_order;
    q.norder = p.tc_norder;
    q.cbase = p.d_tcs_cbase;
    q.Bt = p.d_tcs_B;
    q.err = p.d_err;
    q.wait_ns = p.tc_wait_ns;
    q.inject = p.inject;
    q.flush = std::max(1, p.tc_fold / kTcK);
    // whole groups of kTcMaps maps share one recursion (N = 4 kTcMaps); a remainder runs
    // in groups of 8, so a short batch does not pay for the columns of a full group
    constexpr int kSmall = 8;
    const int nbig = (kTcMaps > kSmall && p.tc_group >= kTcMaps) ? (nb / kTcMaps) * kTcMaps : 0;
    const int nsmall = nb - nbig;
    const size_t alm_map = (size_t)p.ncomp * p.K, F_map = (size_t)p.ncomp * p.nrings * p.M;
    int rc = JHTB_OK;
    if (nbig > 0)
        rc = p.spin ? launch_tc_synth_t<2, kTcMaps>(p, q, alm, F, nbig, s) : launch_tc_synth_t<0, kTcMaps>(p, q, alm, F, nbig, s);
    if (rc == JHTB_OK && nsmall > 0) {
        const double2 *a2 = alm + (size_t)nbig * alm_map;
        double2 *F2 = F + (size_t)nbig * F_map;
        rc = p.spin ? launch_tc_synth_t<2, kSmall>(p, q, a2, F2, nsmall, s) : launch_tc_synth_t<0, kSmall>(p, q, a2, F2, nsmall, s);
    }
    return rc;
}

// Bytes of one prepared coefficient chunk for full (16-map) groups; 8-map groups use less.
size_t tc_synth_chunk_bytes(int spin) { return spin ? TcCfg<2, kTcMaps>::BBYTES : TcCfg<0, kTcMaps>::BBYTES; }

}  // namespace jhtb
