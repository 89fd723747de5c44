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
// The CTA is warp-specialised and its roles meet only at mbarriers:
//   producer warps (one thread per A row = tensor-memory lane, two recursion chains
//     per thread) run the FP64 recursion (same normalised form and start states as
//     the FP64 kernels), round mu to FP32, split it into three BF16 parts and store
//     their rows of the A operands straight into tensor memory (tcgen05.st), so the
//     six split products never re-read A through shared memory;
//   builder warps (one thread per (l, map) of a chunk) load a_lm and c_l two chunks
//     ahead into registers, form the B rows (c_l a_lm with the N/S sign pattern),
//     split them the same way into shared memory, and stage the chunk's recursion
//     coefficients;
//   one MMA warp issues the six split products hh, hm, mh, hl, lh, mm per GEMM
//     (kind::f16, A from tensor memory, B from shared memory, FP32 accumulators in
//     tensor memory) and commits each stage back to its producers.
// hh accumulates apart from the five smaller products (relative size <= 2^-8).
// Every kFlush chunks (256 l) the producers fold the FP32 block sums into per-thread
// double-float (hi, lo) accumulators in shared memory, so FP32 rounding acts on at
// most 256 terms; the item's result is hi + lo in FP64.  Every wait is bounded; on
// timeout the kernel records an error, every role leaves its loop, and tensor memory
// is released after the last MMA has drained.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"
#include "tc_common.cuh"

namespace jhtb {
namespace {

constexpr int kTcRows = 128;     // = MMA M = rings per tile
constexpr int kTcK = 16;         // l steps per chunk = MMA K (BF16)
#ifndef JHTB_TC_FLUSH
#define JHTB_TC_FLUSH 16
#endif
#ifndef JHTB_TC_NSA
#define JHTB_TC_NSA 2
#endif
constexpr int kFlush = JHTB_TC_FLUSH;  // chunks per FP32 accumulation block (256 l)

using namespace tc;

struct TcParams {
    int lmax, T, nrings, M, nside;
    long long K;
    const double *x;
    const SeedParam *seed;
    const double *alpha, *gamma, *cnorm;
    int ntiles;  // item tiles per m (128 rings for spin 2, 256 for spin 0)
    int norder;  // entries of order (the items inside the plan's ring range)
    const int *lw;
    const double2 *st;
    const int *stsc;
    const int *order;
    int *err;
    unsigned long long wait_ns;  // time limit of every bounded wait
    int inject;                  // fault injection for tests (kInjectStall: builders publish nothing)
};

template <int SPIN, int BM>
struct TcCfg {
    static constexpr int NG = 2;                    // GEMMs per chunk = recursion chains per producer thread
    static constexpr int NBT = SPIN ? 2 : 1;        // B tiles per chunk (spin 0: both GEMMs share one)
    static constexpr int N = 4 * BM;                // columns per GEMM
    static constexpr int CH = BM >= 16 ? 1 : 2;     // recursion chains (GEMMs) per producer thread
    static constexpr int NPW = 4 * NG / CH;         // producer warps: one thread per A row (TMEM lane) and chain
    static constexpr int NBW = kTcK * BM / 32;      // builder warps: one thread per (l, map) of a chunk
    static constexpr int MMA_WARP = NPW + NBW;
    static constexpr int NTHREADS = (NPW + NBW + 1) * 32;
    static constexpr int NSA = JHTB_TC_NSA;         // A stages (in tensor memory)
    static constexpr int NSB = 4;                   // B stages (with the chunk's coefficients)
    static constexpr int BTILE = N * kTcK * 2;
    static constexpr int ACOLS = kTcK / 2;          // tensor-memory columns of one A row (16 BF16)
    // tensor memory: per GEMM hh and corr block sums, then the A stages
    static constexpr int COL_A = NG * 2 * N;
    static constexpr int NCOL = COL_A + NSA * NG * 3 * ACOLS;
    static constexpr uint32_t TCOLS =
        NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : (NCOL <= 256 ? 256 : 512)));
    static constexpr int MIN_CTAS = TCOLS <= 256 ? 2 : 1;  // resident CTAs per SM the tensor memory allows
    static_assert(NBW * 32 == kTcK * BM, "one builder thread per (l, map) of a chunk");
    static_assert(NCOL <= 512, "tensor memory of one SM");
};

template <int SPIN, int BM>
struct TcSmem {
    using C = TcCfg<SPIN, BM>;
    alignas(1024) unsigned char B[C::NSB][C::NBT][3][C::BTILE];
    double2 coef[C::NSB][kTcK];  // (alpha, gamma) of the chunk's 16 steps
    // double-float accumulators, [hi/lo][GEMM][column][row]: a warp touches 32 consecutive words
    float acc[2][C::NG][C::N][kTcRows];
    alignas(8) uint64_t fullA[C::NSA], emptyA[C::NSA], fullB[C::NSB], emptyB[C::NSB];
    uint64_t accFull, accEmpty, fin;
    uint32_t taddr;
    int fail;
};

// One (m, ring tile, map group) work item, as every role of the CTA derives it.
struct TcItem {
    int item, m, lmin, i_start, nst, nck, b_lo, b_cnt, tile;
    long long b0;
};

// Item info from its id (the loads of lmin and lw are issued here and consumed later).
__device__ __forceinline__ TcItem tc_item_of(const TcParams &p, int it, int item, int nitems, int nb, int bm) {
    TcItem q;
    const int g = it / nitems;
    q.item = item;
    q.m = item / p.ntiles;
    q.tile = item - q.m * p.ntiles;
    q.lmin = __ldg(&p.seed[q.m].lmin);
    q.b0 = alm_index(q.lmin, q.m, p.lmax);
    q.nst = p.lmax - q.lmin + 1;
    q.i_start = __ldg(&p.lw[item]) - q.lmin;
    q.nck = q.i_start < q.nst ? (q.nst - q.i_start + kTcK - 1) / kTcK : 0;
    q.b_lo = g * bm;
    q.b_cnt = min(bm, nb - q.b_lo);
    return q;
}
__device__ __forceinline__ int tc_order(const TcParams &p, int it, int nitems, int total) {
    return it < total ? __ldg(&p.order[it % nitems]) : 0;
}
__device__ __forceinline__ TcItem tc_item(const TcParams &p, int it, int nitems, int nb, int bm) {
    return tc_item_of(p, it, __ldg(&p.order[it % nitems]), nitems, nb, bm);
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

// 16 steps of this thread's CH recursion chains (GEMMs J0 .. J0 + CH - 1), split into
// BF16 parts and stored as its row (= its tensor-memory lane) of those GEMMs' three A
// operands: tA[c] is the lane-offset tensor-memory address of chain c's split-0 operand,
// the splits following at ACOLS columns apart.  Spin 2: GEMM 0 is the +2 recursion
// (+gamma), GEMM 1 the -2 one (-gamma), same ring; spin 0: the GEMMs are rings row and
// 128 + row of the item tile (gamma = 0).  Past the end of the column the
// coefficients are zero, which keeps the state bounded (u_k = -u_{k-2}) while the B
// rows there are zero; rows past the last ring start from a zero state and stay zero.
// Each half-chunk first loads its eight coefficient pairs and forms the multipliers
// t = alpha x +- gamma, so only one FMA per step stays on the dependency chain.
template <bool SLOW, int CH, int J0>
__device__ __forceinline__ void tc_chunk(const double2 *coef, const double (&x)[CH], double (&u1)[CH],
                                         double (&u2)[CH], int (&sc)[CH], const uint32_t (&tA)[CH]) {
    constexpr uint32_t AC = kTcK / 2;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        double t[CH][8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 a = coef[half * 8 + k];
#pragma unroll
            for (int c = 0; c < CH; ++c) t[c][k] = ((J0 + c) & 1) ? fma(a.x, x[c], -a.y) : fma(a.x, x[c], a.y);
        }
        uint32_t pk[CH][3][4];
#pragma unroll
        for (int q = 0; q < 8; q += 2) {
            double v0[CH], v1[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) v0[c] = tc_step<SLOW>(t[c][q], u1[c], u2[c], sc[c]);
#pragma unroll
            for (int c = 0; c < CH; ++c) v1[c] = tc_step<SLOW>(t[c][q + 1], u1[c], u2[c], sc[c]);
#pragma unroll
            for (int c = 0; c < CH; ++c) split3_pair(v0[c], v1[c], pk[c][0][q / 2], pk[c][1][q / 2], pk[c][2][q / 2]);
        }
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int sp = 0; sp < 3; ++sp)
                tmem_st4(tA[c] + sp * AC + half * 4, pk[c][sp][0], pk[c][sp][1], pk[c][sp][2], pk[c][sp][3]);
    }
}

// (hi, lo) += s in double-float: error-free two-sum of hi + s, then renormalise.
__device__ __forceinline__ void df_add(float &hi, float &lo, float s) {
    const float t = hi + s;
    const float bp = t - hi;
    const float e = (hi - (t - bp)) + (s - bp);
    const float l2 = lo + e;
    hi = t + l2;
    lo = l2 - (hi - t);
}

// Rows of F for one (map, ring): north (healpix.py:250-253) and the signed south mirror.
// Spin 2: GEMM + (H = 0) holds [FpN | FmS], GEMM - (H = 1) holds [FmN | FpS].
template <int SPIN>
__device__ __forceinline__ void tc_store_F(const TcParams &p, double2 *__restrict__ F_all, int b, int H, int t, int m,
                                           int lmin, const double (&v)[4]) {
    const size_t rs = (size_t)(p.nrings - 1 - t);
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
    const uint32_t tl = tbase + ((uint32_t)((warp & 3) * 32) << 16);
    float(&acc)[2][C::NG][N][kTcRows] = sm.acc;
    const int nitems = p.norder;
    const int total = nitems * ((nb + BM - 1) / BM);
    const int stride = gridDim.x;
    unsigned gc = 0, bk = 0;
    bool ok = true;
    // GEMM j's ring (spin 0: two 128-ring halves of the item tile) and start-state slot
    auto ring_of = [&](int tile, int j) { return SPIN ? tile * kTcRows + row : tile * 2 * kTcRows + j * kTcRows + row; };
    auto st_of = [&](int id, int j) { return ((size_t)id * 2 + j) * kTcRows + row; };
    // the next item's id, lmin, lw and start states are loaded one item ahead, the
    // order entry two items ahead
    int it = blockIdx.x;
    int id = tc_order(p, it, nitems, total);
    int id_next = tc_order(p, it + stride, nitems, total);
    int lmin = __ldg(&p.seed[id / p.ntiles].lmin), lwv = __ldg(&p.lw[id]);
    double2 st[CH];
    int stsc[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
        st[c] = p.st[st_of(id, j0 + c)];
        stsc[c] = p.stsc[st_of(id, j0 + c)];
    }
    for (; it < total && ok; it += stride) {
        if (tc_failed(&sm.fail)) break;
        const int id_nn = tc_order(p, it + 2 * stride, nitems, total);
        const int lmin_n = __ldg(&p.seed[id_next / p.ntiles].lmin), lw_n = __ldg(&p.lw[id_next]);
        double2 st_n[CH];
        int stsc_n[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            st_n[c] = p.st[st_of(id_next, j0 + c)];
            stsc_n[c] = p.stsc[st_of(id_next, j0 + c)];
        }

        const int m = id / p.ntiles, tile = id - m * p.ntiles;
        int tr[CH];
        double x[CH], u1[CH], u2[CH];
        int sc[CH];
        bool fast = true;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            tr[c] = ring_of(tile, j0 + c);
            x[c] = tr[c] < p.T ? __ldg(&p.x[tr[c]]) : 0.0;
            u1[c] = st[c].x;
            u2[c] = st[c].y;
            sc[c] = tr[c] < p.T ? stsc[c] : 0;
            fast &= sc[c] == 0;
        }
        const int nst = p.lmax - lmin + 1, i_start = lwv - lmin;
        const int nck = i_start < nst ? (nst - i_start + kTcK - 1) / kTcK : 0;
        for (int c = 0; c < nck; ++c, ++gc) {
            const int sA = gc % C::NSA, sB = gc % C::NSB;
            if (!mbar_wait_warp(&sm.fullB[sB], (gc / C::NSB) & 1u, p.wait_ns)) { ok = false; break; }
            if (gc >= (unsigned)C::NSA && !mbar_wait_warp(&sm.emptyA[sA], ((gc / C::NSA) - 1u) & 1u, p.wait_ns)) { ok = false; break; }
            tc_fence_after();  // the stage's previous MMAs are complete before it is overwritten
            uint32_t tA[CH];
#pragma unroll
            for (int q = 0; q < CH; ++q) tA[q] = tl + (uint32_t)(C::COL_A + (sA * C::NG + j0 + q) * 3 * C::ACOLS);
            const bool f = __all_sync(0xffffffffu, fast);
            if (j0 == 0) {
                if (f) tc_chunk<false, CH, 0>(sm.coef[sB], x, u1, u2, sc, tA);
                else tc_chunk<true, CH, 0>(sm.coef[sB], x, u1, u2, sc, tA);
            } else {
                if (f) tc_chunk<false, CH, 1>(sm.coef[sB], x, u1, u2, sc, tA);
                else tc_chunk<true, CH, 1>(sm.coef[sB], x, u1, u2, sc, tA);
            }
            if (!f) {
                fast = true;
#pragma unroll
                for (int q = 0; q < CH; ++q) fast &= sc[q] == 0;
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&sm.fullA[sA]);
                mbar_arrive(&sm.emptyB[sB]);
            }
            const bool last = c == nck - 1;
            if ((c % kFlush) == kFlush - 1 || last) {
                if (!mbar_wait_warp(&sm.accFull, bk & 1u, p.wait_ns)) { ok = false; break; }
                tc_fence_after();
                const bool first_block = c < kFlush;
                const int b_lo = (it / nitems) * BM, b_cnt = min(BM, nb - b_lo);
#pragma unroll 1
                for (int piece = 0; piece < CH * N / 8; ++piece) {
                    const int q = piece / (N / 8), j = j0 + q, c0 = (piece % (N / 8)) * 8;
                    const uint32_t tg = tl + (uint32_t)(j * 2 * N + c0);
                    float hh[8], co[8];
                    tmem_ld8(tg, hh);
                    tmem_ld8(tg + N, co);
                    float hi[8], lo[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const float sblk = hh[e] + co[e];
                        if (first_block) {
                            hi[e] = sblk;
                            lo[e] = 0.0f;
                        } else {
                            hi[e] = acc[0][j][c0 + e][row];
                            lo[e] = acc[1][j][c0 + e][row];
                            df_add(hi[e], lo[e], sblk);
                        }
                    }
                    if (!last) {
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            acc[0][j][c0 + e][row] = hi[e];
                            acc[1][j][c0 + e][row] = lo[e];
                        }
                    } else {
                        const int t = tr[q];
                        if (t < p.T) {
#pragma unroll
                            for (int jb = 0; jb < 2; ++jb) {
                                const int bm = c0 / 4 + jb;
                                if (bm >= b_cnt) continue;
                                double v[4];
#pragma unroll
                                for (int e = 0; e < 4; ++e) v[e] = (double)hi[4 * jb + e] + (double)lo[4 * jb + e];
                                tc_store_F<SPIN>(p, F_all, b_lo + bm, SPIN ? j : 0, t, m, lmin, v);
                            }
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&sm.accEmpty);
                ++bk;
            }
        }
        if (ok && nck == 0) {
            // no representable term in this tile: the rows are exactly zero
            const int b_lo = (it / nitems) * BM, b_cnt = min(BM, nb - b_lo);
            const double z[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < CH; ++q) {
                const int t = tr[q];
                if (t < p.T)
                    for (int bm = 0; bm < b_cnt; ++bm) tc_store_F<SPIN>(p, F_all, b_lo + bm, SPIN ? j0 + q : 0, t, m, lmin, z);
            }
        }
        id = id_next;
        id_next = id_nn;
        lmin = lmin_n;
        lwv = lw_n;
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            st[q] = st_n[q];
            stsc[q] = stsc_n[q];
        }
    }
    if (!ok) tc_fail(&sm.fail, p.err);
}

// ---------------------------------------------------------------------------------
// builder warps: B tiles (c_l a_lm with the N/S sign pattern) and coefficients
// ---------------------------------------------------------------------------------
struct TcLoad {
    double c;
    double2 e, b, ag;
    bool live;  // a chunk exists (values past the column or the batch are zero)
};

// Walks the CTA's (item, chunk) sequence, skipping items without chunks.
template <int BM>
struct TcCursor {
    int it, c, total, nitems, nb;
    TcItem q;
    __device__ __forceinline__ void settle(const TcParams &p) {
        while (it < total) {
            q = tc_item(p, it, nitems, nb, BM);
            if (q.nck > 0) return;
            it += gridDim.x;
        }
    }
    __device__ __forceinline__ void next(const TcParams &p) {
        if (it >= total) return;
        if (++c >= q.nck) {
            c = 0;
            it += gridDim.x;
            settle(p);
        }
    }
};

template <int SPIN, int BM>
__device__ __forceinline__ TcLoad tc_load(const TcParams &p, const double2 *__restrict__ alm_all,
                                          const TcCursor<BM> &cur, int k, int bm) {
    TcLoad r;
    r.c = 0.0;
    r.e = r.b = r.ag = make_double2(0.0, 0.0);
    r.live = cur.it < cur.total;
    if (!r.live) return r;
    const int i = cur.q.i_start + cur.c * kTcK + k;
    if (i >= cur.q.nst) return r;
    const long long idx = cur.q.b0 + i;
    if (bm == 0) r.ag = make_double2(__ldg(&p.alpha[idx]), SPIN ? __ldg(&p.gamma[idx]) : 0.0);
    if (bm >= cur.q.b_cnt) return r;
    r.c = __ldg(&p.cnorm[idx]);
    if (SPIN) {
        r.e = __ldg(&alm_all[((size_t)(cur.q.b_lo + bm) * 2) * p.K + idx]);
        r.b = __ldg(&alm_all[((size_t)(cur.q.b_lo + bm) * 2 + 1) * p.K + idx]);
    } else {
        r.e = __ldg(&alm_all[(size_t)(cur.q.b_lo + bm) * p.K + idx]);
    }
    return r;
}

template <int SPIN, int BM>
__device__ void tc_builder(const TcParams &p, const double2 *__restrict__ alm_all, TcSmem<SPIN, BM> &sm, int nb,
                           int bt, int lane) {
    using C = TcCfg<SPIN, BM>;
    const int k = bt % kTcK, bm = bt / kTcK;
    const double sg = (k & 1) ? -1.0 : 1.0;  // (-1)^(l - lmin): chunks start at even offsets
    // test hook: no operand stage is ever published, so every wait on one runs out
    if (p.inject == kInjectStall) return;
    const int nitems = p.norder;
    // the loads run two chunks ahead of the stores
    TcCursor<BM> ld{(int)blockIdx.x, 0, nitems * ((nb + BM - 1) / BM), nitems, nb, TcItem{}};
    ld.settle(p);
    TcLoad r0 = tc_load<SPIN, BM>(p, alm_all, ld, k, bm);
    ld.next(p);
    TcLoad r1 = tc_load<SPIN, BM>(p, alm_all, ld, k, bm);
    ld.next(p);
    unsigned gc = 0;
    bool ok = true;
    while (r0.live) {
        if (tc_failed(&sm.fail)) break;
        const int sB = gc % C::NSB;
        if (gc >= (unsigned)C::NSB && !mbar_wait_warp(&sm.emptyB[sB], ((gc / C::NSB) - 1u) & 1u, p.wait_ns)) { ok = false; break; }
        double col[C::NBT][4];
        if (SPIN) {
            // cp = -(aE + i aB) c, cm = -(aE - i aB) c   (healpix.py:316-318)
            const double cpr = -(r0.e.x - r0.b.y) * r0.c, cpi = -(r0.e.y + r0.b.x) * r0.c;
            const double cmr = -(r0.e.x + r0.b.y) * r0.c, cmi = -(r0.e.y - r0.b.x) * r0.c;
            col[0][0] = cpr; col[0][1] = cpi; col[0][2] = sg * cmr; col[0][3] = sg * cmi;
            col[C::NBT - 1][0] = cmr; col[C::NBT - 1][1] = cmi; col[C::NBT - 1][2] = sg * cpr; col[C::NBT - 1][3] = sg * cpi;
        } else {
            col[0][0] = r0.e.x * r0.c; col[0][1] = r0.e.y * r0.c;
            col[0][2] = sg * r0.e.x * r0.c; col[0][3] = sg * r0.e.y * r0.c;
        }
#pragma unroll
        for (int hh = 0; hh < C::NBT; ++hh)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                __nv_bfloat16 vh, vm, vl;
                split3(col[hh][j], vh, vm, vl);
                const uint32_t off = kmaj_off(4 * bm + j, k);
                *reinterpret_cast<__nv_bfloat16 *>(sm.B[sB][hh][0] + off) = vh;
                *reinterpret_cast<__nv_bfloat16 *>(sm.B[sB][hh][1] + off) = vm;
                *reinterpret_cast<__nv_bfloat16 *>(sm.B[sB][hh][2] + off) = vl;
            }
        if (bm == 0) sm.coef[sB][k] = r0.ag;
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.fullB[sB]);
        ++gc;
        r0 = r1;
        r1 = tc_load<SPIN, BM>(p, alm_all, ld, k, bm);
        ld.next(p);
    }
    if (!ok) tc_fail(&sm.fail, p.err);
}

// ---------------------------------------------------------------------------------
// MMA warp: one thread issues the split products and the commits
// ---------------------------------------------------------------------------------
template <int SPIN, int BM>
__device__ void tc_mma(const TcParams &p, TcSmem<SPIN, BM> &sm, int nb, uint32_t tbase, int lane) {
    using C = TcCfg<SPIN, BM>;
    constexpr int N = C::N;
    constexpr uint32_t IDESC = idesc_bf16(kTcRows, N);
    const int nitems = p.norder;
    const int total = nitems * ((nb + BM - 1) / BM);
    unsigned gc = 0, bk = 0;
    bool ok = true;
    const int stride = gridDim.x;
    int it = blockIdx.x;
    int id_next = tc_order(p, it + stride, nitems, total);
    int nck_cur = it < total ? tc_item(p, it, nitems, nb, BM).nck : 0;
    for (; it < total && ok; it += stride) {
        if (tc_failed(&sm.fail)) break;
        const int id_nn = tc_order(p, it + 2 * stride, nitems, total);
        const int nck_next = tc_item_of(p, it + stride < total ? it + stride : it, id_next, nitems, nb, BM).nck;
        const int nck = nck_cur;
        for (int c = 0; c < nck; ++c, ++gc) {
            const int sA = gc % C::NSA, sB = gc % C::NSB;
            const bool bstart = (c % kFlush) == 0;
            const bool bend = (c % kFlush) == kFlush - 1 || c == nck - 1;
            if (!mbar_wait_warp(&sm.fullA[sA], (gc / C::NSA) & 1u, p.wait_ns) || !mbar_wait_warp(&sm.fullB[sB], (gc / C::NSB) & 1u, p.wait_ns) ||
                (bstart && bk > 0 && !mbar_wait_warp(&sm.accEmpty, (bk - 1u) & 1u, p.wait_ns))) {
                ok = false;
                break;
            }
            tc_fence_after();
            if (lane == 0) {
                const uint32_t acc = bstart ? 0u : 1u;
#pragma unroll
                for (int j = 0; j < C::NG; ++j) {
                    const int jb = SPIN ? j : 0;
                    const uint32_t d = tbase + (uint32_t)(j * 2 * N), dc = d + (uint32_t)N;
                    const uint32_t a0 = tbase + (uint32_t)(C::COL_A + (sA * C::NG + j) * 3 * C::ACOLS);
                    const uint32_t a1 = a0 + C::ACOLS, a2 = a0 + 2 * C::ACOLS;
                    const uint64_t c0 = smem_desc(sm.B[sB][jb][0], 128, 256), c1 = smem_desc(sm.B[sB][jb][1], 128, 256),
                                   c2 = smem_desc(sm.B[sB][jb][2], 128, 256);
                    umma_f16_ts(d, a0, c0, IDESC, acc);   // hh
                    umma_f16_ts(dc, a0, c1, IDESC, acc);  // hm
                    umma_f16_ts(dc, a1, c0, IDESC, 1u);   // mh
                    umma_f16_ts(dc, a0, c2, IDESC, 1u);   // hl
                    umma_f16_ts(dc, a2, c0, IDESC, 1u);   // lh
                    umma_f16_ts(dc, a1, c1, IDESC, 1u);   // mm
                }
                umma_commit(&sm.emptyA[sA]);
                umma_commit(&sm.emptyB[sB]);
                if (bend) umma_commit(&sm.accFull);
            }
            __syncwarp();
            if (bend) ++bk;
        }
        nck_cur = nck_next;
        id_next = id_nn;
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
__global__ void __launch_bounds__(TcCfg<SPIN, BM>::NTHREADS, TcCfg<SPIN, BM>::MIN_CTAS)
    tc_synth_kernel(TcParams p, const double2 *__restrict__ alm_all, double2 *__restrict__ F_all, int nb) {
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
            mbar_init(&sm.fullB[s], C::NBW);
            mbar_init(&sm.emptyB[s], 1 + C::NPW);
        }
        mbar_init(&sm.accFull, 1);
        mbar_init(&sm.accEmpty, C::NPW);
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
    } else if (warp < C::NPW + C::NBW) {
        tc_builder<SPIN, BM>(p, alm_all, sm, nb, threadIdx.x - C::NPW * 32, lane);
    } else {
        tc_mma<SPIN, BM>(p, sm, nb, tbase, lane);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == C::MMA_WARP) tmem_dealloc(tbase, C::TCOLS);
}

}  // namespace

template <int SPIN, int BM>
static int launch_tc_synth_t(const TcParams &q, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    using C = TcCfg<SPIN, BM>;
    auto k = tc_synth_kernel<SPIN, BM>;
    const int smem = (int)sizeof(TcSmem<SPIN, BM>) + 1024;
    int dev = 0, nsm = 148, smem_sm = 0, regs_sm = 0, resv = 0;
    JHTB_CUDA_TRY(cudaGetDevice(&dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    JHTB_CUDA_TRY(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    cudaFuncAttributes fa;
    JHTB_CUDA_TRY(cudaFuncGetAttributes(&fa, k));
    // resident CTAs per SM by shared memory, registers and tensor memory (512 columns:
    // a resident CTA must never wait on tensor memory held by another)
    int per_sm = smem_sm / (smem + resv);
    per_sm = std::min(per_sm, regs_sm / std::max(1, fa.numRegs * C::NTHREADS));
    per_sm = std::max(1, std::min(per_sm, (int)(512 / C::TCOLS)));
    k<<<nsm * per_sm, C::NTHREADS, smem, s>>>(q, alm, F, nb);
    JHTB_CUDA_TRY(cudaGetLastError());
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
    q.alpha = p.d_alpha;
    q.gamma = p.d_gamma;
    q.cnorm = p.d_cnorm;
    q.ntiles = p.tc_ntiles;
    q.lw = p.d_tc_lw;
    q.st = p.d_tc_st;
    q.stsc = p.d_tc_stsc;
    q.order = p.d_tc_order;
    q.norder = p.tc_norder;
    q.err = p.d_err;
    q.wait_ns = p.tc_wait_ns;
    q.inject = p.inject;
    // whole groups of kTcMaps maps share one recursion (one CTA per SM, N = 4 kTcMaps);
    // a remainder runs in groups of 8 (two CTAs per SM), so a short batch does not pay
    // for the columns of a full group
    constexpr int kSmall = 8;
    const int nbig = kTcMaps > kSmall ? (nb / kTcMaps) * kTcMaps : 0;
    const int nsmall = nb - nbig;
    const size_t alm_map = (size_t)p.ncomp * p.K, F_map = (size_t)p.ncomp * p.nrings * p.M;
    int rc = JHTB_OK;
    if (nbig > 0)
        rc = p.spin ? launch_tc_synth_t<2, kTcMaps>(q, alm, F, nbig, s) : launch_tc_synth_t<0, kTcMaps>(q, alm, F, nbig, s);
    if (rc == JHTB_OK && nsmall > 0) {
        const double2 *a2 = alm + (size_t)nbig * alm_map;
        double2 *F2 = F + (size_t)nbig * F_map;
        rc = p.spin ? launch_tc_synth_t<2, kSmall>(q, a2, F2, nsmall, s) : launch_tc_synth_t<0, kSmall>(q, a2, F2, nsmall, s);
    }
    return rc;
}

}  // namespace jhtb
