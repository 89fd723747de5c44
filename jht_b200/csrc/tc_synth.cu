// Batched mixed-precision synthesis on the 5th-generation tensor cores (tcgen05).
//
// For one order m and a tile of 128 half-grid rings the l-contraction of B maps is a
// GEMM:  F[t, n] = sum_l mu_l(t) C[l, n],  t = ring (M = 128), l (K, 16 per MMA),
// n = (map, component) (N = 4 B per GEMM).  Spin 2 runs two GEMMs, one per
// recursion (+2 / -2):  D+ = Lambda+ [cp, s cm],  D- = Lambda- [cm, s cp], with
// s = (-1)^(l - lmin) folded into the B rows; jht's four half-grid sums
// (_recursion.py:512-543) are the four column pairs.  Spin 0 runs one GEMM with
// columns [a, s a] (_recursion.py:441-469).
//
// Each thread owns one ring: it runs the FP64 recursion (same normalised form and
// start states as the FP64 kernels), rounds mu to FP32 and splits it into three BF16
// parts, and writes its row of the A tiles (K-major, no swizzle) in shared memory.
// The B tiles (a_lm times c_l, split the same way) are written by all threads.  One
// thread issues the six split products hh, hm, mh, hl, lh, mm per GEMM
// (kind::f16, BF16 x BF16 -> FP32 in tensor memory); a commit to an mbarrier frees
// the double-buffered stage.  Every kFlush chunks the FP32 accumulators are read
// (tcgen05.ld) into FP64 registers and restarted, so FP32 rounding accumulates over
// at most 64 l.  Every wait is bounded; on timeout the kernel records an error,
// releases its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "jhtb_internal.cuh"

namespace jhtb {
namespace {

constexpr int kTcRows = 128;     // = MMA M = rings per tile
constexpr int kTcK = 16;         // l steps per chunk = MMA K (BF16)
constexpr int kFlush = 4;        // chunks per FP32 accumulation block
constexpr int kSuper = 8;        // chunks per staging pass (coefficients + B tiles); multiple of kFlush
constexpr unsigned kWaitLimit = 1u << 26;

// ---------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait (iteration count and ~2 s of wall time); returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const uint64_t t0 = globaltimer_ns();
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 1023u && globaltimer_ns() - t0 > 2000000000ull) return false;
    }
    return false;
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 consecutive FP32 columns -> 32 registers per thread (its own lane's row).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
        "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory descriptor, K-major, no swizzle: 8-row x 16-byte core matrices,
// LBO = byte distance between the two 8-element K halves, SBO = between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo) {
    const uint32_t a = smem_u32(p);
    return (uint64_t)((a >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1 (sm100), swizzle none
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with LBO 128, SBO 256
// (K = 16): core matrix (row/8, k/8) at (row/8)*256 + (k/8)*128, row-in-core * 16 + k%8 * 2.
__device__ __forceinline__ uint32_t kmaj_off(int row, int k) {
    return (uint32_t)((row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// x ~ h + m + l with h, m, l BF16: x is rounded to FP32, then each part keeps the top
// 16 bits of the remaining residual (a truncation, exact in FP32), so h + m + l differs
// from x by less than 2^-24 |x|.  Returns the three parts as FP32 bit patterns whose
// low halves are zero (the BF16 value is the high half).
__device__ __forceinline__ void split3_bits(double xd, uint32_t &h, uint32_t &m, uint32_t &l) {
    const float x = (float)xd;
    h = __float_as_uint(x) & 0xFFFF0000u;
    const float r1 = x - __uint_as_float(h);
    m = __float_as_uint(r1) & 0xFFFF0000u;
    const float r2 = r1 - __uint_as_float(m);
    l = __float_as_uint(r2) & 0xFFFF0000u;
}
// two BF16 high halves -> one packed word (first value in the low half)
__device__ __forceinline__ uint32_t pack_hi(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x7632); }

// BF16 of FP32 value x by truncation (used for the B tiles, same split as split3_bits)
__device__ __forceinline__ void split3(double xd, __nv_bfloat16 &h, __nv_bfloat16 &m, __nv_bfloat16 &l) {
    uint32_t hb, mb, lb;
    split3_bits(xd, hb, mb, lb);
    h = __ushort_as_bfloat16((unsigned short)(hb >> 16));
    m = __ushort_as_bfloat16((unsigned short)(mb >> 16));
    l = __ushort_as_bfloat16((unsigned short)(lb >> 16));
}


__device__ __forceinline__ void rescale(double &u, double &prev, int &sc) {
    if (sc < 0 && fabs(u) > kBig) {
        u *= kScaleDown;
        prev *= kScaleDown;
        sc += 1;
    }
}

struct TcParams {
    int lmax, T, nrings, M, nside;
    long long K;
    const double *x;
    const SeedParam *seed;
    const double *alpha, *gamma, *cnorm;
    int ntiles;  // 128-ring tiles per m
    const int *lw;
    const double2 *st;
    const int *stsc;
    const int *order;
    unsigned *counter;
    int *err;
};

template <int SPIN, int BM>
struct TcSmem {
    static constexpr int NG = SPIN ? 2 : 1;
    static constexpr int N = 4 * BM;
    // per stage: A tiles [NG][3 splits][128 x 16 bf16], B tiles [NG][3][N x 16 bf16]
    alignas(1024) unsigned char A[2][NG][3][kTcRows * kTcK * 2];
    // B tiles for all kSuper chunks of a 128-step super-chunk, built in one pass
    alignas(128) unsigned char B[kSuper][NG][3][N * kTcK * 2];
    double2 coef[kSuper * kTcK];  // (alpha, gamma) for the super-chunk's steps
    alignas(8) uint64_t mbar[2];
    uint32_t taddr;
    int err;
};

// One step of one recursion with the scaled-phase bookkeeping (SLOW) or without.
template <bool SLOW>
__device__ __forceinline__ double tc_step(double al, double ga, double x, double &u1, double &u2, int &sc) {
    double u = fma(fma(al, x, ga), u1, -u2);
    double prev = u1;
    if (SLOW) rescale(u, prev, sc);
    u2 = prev;
    u1 = u;
    return (SLOW && sc != 0) ? 0.0 : u;
}

// 16 steps -> packed BF16 rows (pk[split][word]) of this thread's ring.
template <bool SLOW>
__device__ __forceinline__ void tc_chunk(const double2 *coef, int ncnt, double x, double gsign, bool valid, double &u1,
                                         double &u2, int &sc, uint32_t (&pk)[3][kTcK / 2]) {
#pragma unroll
    for (int q = 0; q < kTcK; q += 2) {
        double v0 = 0.0, v1 = 0.0;
        if (q < ncnt) {
            const double2 ag = coef[q];
            v0 = tc_step<SLOW>(ag.x, gsign * ag.y, x, u1, u2, sc);
        }
        if (q + 1 < ncnt) {
            const double2 ag = coef[q + 1];
            v1 = tc_step<SLOW>(ag.x, gsign * ag.y, x, u1, u2, sc);
        }
        if (!valid) v0 = v1 = 0.0;
        uint32_t h0, m0, l0, h1, m1, l1;
        split3_bits(v0, h0, m0, l0);
        split3_bits(v1, h1, m1, l1);
        pk[0][q / 2] = pack_hi(h0, h1);
        pk[1][q / 2] = pack_hi(m0, m1);
        pk[2][q / 2] = pack_hi(l0, l1);
    }
}

template <int SPIN, int BM>
__global__ void __launch_bounds__(kTcRows * (SPIN ? 2 : 1), SPIN ? 2 : 3) tc_synth_kernel(TcParams p, const double2 *__restrict__ alm_all,
                                                                           double2 *__restrict__ F_all, int nb) {
    using S = TcSmem<SPIN, BM>;
    constexpr int NG = S::NG, N = S::N;
    constexpr int NTH = kTcRows * NG;           // one thread per (ring, recursion)
    constexpr int NCOL = 2 * NG * N;            // per GEMM: hh accumulator + correction accumulator
    constexpr uint32_t TCOLS = NCOL <= 32 ? 32 : (NCOL <= 64 ? 64 : (NCOL <= 128 ? 128 : 256));
    constexpr uint32_t IDESC = idesc_bf16(kTcRows, N);
    extern __shared__ unsigned char smem_raw[];
    S &sm = *reinterpret_cast<S *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ int s_it;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = tid % kTcRows;  // ring within the tile = A row = TMEM lane
    const int h = tid / kTcRows;    // recursion: 0 = +spin (or spin 0), 1 = -spin
    const double gsign = h ? -1.0 : 1.0;

    if (warp == 0) {
        tmem_alloc(&sm.taddr, TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&sm.mbar[0], 1);
        mbar_init(&sm.mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sm.taddr;
    const uint32_t tlane = (uint32_t)((warp & 3) * 32) << 16;
    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};
    bool failed = false;

    const int L = p.lmax;
    const int ngroups = (nb + BM - 1) / BM;
    const int nitems = p.M * p.ntiles;
    for (;;) {
        if (tid == 0) s_it = (int)atomicAdd(p.counter, 1u);
        __syncthreads();
        const int it = s_it;
        __syncthreads();
        if (it >= nitems * ngroups || failed) break;
        const int g = it / nitems;
        const int item = p.order[it - g * nitems];
        const int m = item / p.ntiles, tile = item % p.ntiles;
        const int b_lo = g * BM, b_cnt = min(BM, nb - b_lo);
        const SeedParam sd = p.seed[m];
        const long long b0 = alm_index(sd.lmin, m, L);
        const int nst = L - sd.lmin + 1;
        const int i_start = p.lw[item] - sd.lmin;
        const int t = tile * kTcRows + row;
        const bool valid = t < p.T;
        const double x = valid ? p.x[t] : 0.0;
        double u1, u2;
        int sc;
        {
            // start-state layout [item][h][r][lane], ring = r * 32 + lane within the tile
            const size_t o = ((size_t)item * NG + h) * kTcRows + row;
            const double2 st = p.st[o];
            u1 = st.x;
            u2 = st.y;
            sc = valid ? p.stsc[o] : 0;
        }
        bool fast = sc == 0;
        double acc[N];
#pragma unroll
        for (int n = 0; n < N; ++n) acc[n] = 0.0;
        bool fresh = true;
        int kc = 0;
        for (int i0 = i_start; i0 < nst; i0 += kTcK, ++kc) {
            const int s = kc & 1;
            if (pending[s]) {
                if (!mbar_wait(&sm.mbar[s], phase[s])) failed = true;
                phase[s] ^= 1u;
                pending[s] = false;
            }
            if (kc % kSuper == 0) {
                // ---- staging pass for kSuper chunks; the pipeline is drained here (the
                //      previous chunk closed a flush block). ----
                for (int w = tid; w < kSuper * kTcK; w += NTH) {
                    const int i = i0 + w;
                    sm.coef[w] = i < nst ? make_double2(p.alpha[b0 + i], SPIN ? p.gamma[b0 + i] : 0.0)
                                         : make_double2(0.0, 0.0);
                }
                for (int w = tid; w < kSuper * kTcK * BM; w += NTH) {
                    const int st = w % (kSuper * kTcK), bm = w / (kSuper * kTcK);
                    const int k = st % kTcK, cix = st / kTcK;
                    const int i = i0 + st;
                    const double sg = (k & 1) ? -1.0 : 1.0;  // (-1)^(l - lmin): chunks start at even i
                    double col[NG][4];
                    if (i < nst && bm < b_cnt) {
                        const long long idx = b0 + i;
                        const double c = p.cnorm[idx];
                        if (SPIN) {
                            const double2 e = alm_all[((size_t)(b_lo + bm) * 2) * p.K + idx];
                            const double2 bb = alm_all[((size_t)(b_lo + bm) * 2 + 1) * p.K + idx];
                            // cp = -(aE + i aB) c, cm = -(aE - i aB) c   (healpix.py:316-318)
                            const double cpr = -(e.x - bb.y) * c, cpi = -(e.y + bb.x) * c;
                            const double cmr = -(e.x + bb.y) * c, cmi = -(e.y - bb.x) * c;
                            col[0][0] = cpr; col[0][1] = cpi; col[0][2] = sg * cmr; col[0][3] = sg * cmi;
                            col[NG - 1][0] = cmr; col[NG - 1][1] = cmi; col[NG - 1][2] = sg * cpr; col[NG - 1][3] = sg * cpi;
                        } else {
                            const double2 a = alm_all[(size_t)(b_lo + bm) * p.K + idx];
                            col[0][0] = a.x * c; col[0][1] = a.y * c; col[0][2] = sg * a.x * c; col[0][3] = sg * a.y * c;
                        }
                    } else {
#pragma unroll
                        for (int hh = 0; hh < NG; ++hh)
#pragma unroll
                            for (int j = 0; j < 4; ++j) col[hh][j] = 0.0;
                    }
#pragma unroll
                    for (int hh = 0; hh < NG; ++hh)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            __nv_bfloat16 vh, vm, vl;
                            split3(col[hh][j], vh, vm, vl);
                            const uint32_t off = kmaj_off(4 * bm + j, k);
                            *reinterpret_cast<__nv_bfloat16 *>(sm.B[cix][hh][0] + off) = vh;
                            *reinterpret_cast<__nv_bfloat16 *>(sm.B[cix][hh][1] + off) = vm;
                            *reinterpret_cast<__nv_bfloat16 *>(sm.B[cix][hh][2] + off) = vl;
                        }
                }
            }
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            // ---- A: 16 steps of this thread's recursion, split into BF16 parts ----
            const int ncnt = min(kTcK, nst - i0);
            const double2 *coef = sm.coef + (kc % kSuper) * kTcK;
            uint32_t pk[3][kTcK / 2];
            if (__all_sync(0xffffffffu, fast)) {
                tc_chunk<false>(coef, ncnt, x, gsign, valid, u1, u2, sc, pk);
            } else {
                tc_chunk<true>(coef, ncnt, x, gsign, valid, u1, u2, sc, pk);
                fast = sc == 0;
            }
#pragma unroll
            for (int sp = 0; sp < 3; ++sp) {
                unsigned char *Ab = sm.A[s][h][sp];
                *reinterpret_cast<uint4 *>(Ab + kmaj_off(row, 0)) = make_uint4(pk[sp][0], pk[sp][1], pk[sp][2], pk[sp][3]);
                *reinterpret_cast<uint4 *>(Ab + kmaj_off(row, 8)) = make_uint4(pk[sp][4], pk[sp][5], pk[sp][6], pk[sp][7]);
            }
            fence_async_smem();
            __syncthreads();
            // ---- one thread issues the split products; a commit frees stage s ----
            if (tid == 0) {
                tc_fence_after();
                const int bs = kc % kSuper;
#pragma unroll
                for (int hh = 0; hh < NG; ++hh) {
                    // hh into its own accumulator; the five smaller products (relative size
                    // <= 2^-8) into a second one, so hh sees 4 FP32 roundings per block
                    const uint32_t d = tbase + (uint32_t)(hh * 2 * N), dc = d + (uint32_t)N;
                    const uint64_t a0 = smem_desc(sm.A[s][hh][0], 128, 256), a1 = smem_desc(sm.A[s][hh][1], 128, 256),
                                   a2 = smem_desc(sm.A[s][hh][2], 128, 256);
                    const uint64_t c0 = smem_desc(sm.B[bs][hh][0], 128, 256), c1 = smem_desc(sm.B[bs][hh][1], 128, 256),
                                   c2 = smem_desc(sm.B[bs][hh][2], 128, 256);
                    umma_f16(d, a0, c0, IDESC, fresh ? 0u : 1u);   // hh
                    umma_f16(dc, a0, c1, IDESC, fresh ? 0u : 1u);  // hm
                    umma_f16(dc, a1, c0, IDESC, 1u);               // mh
                    umma_f16(dc, a0, c2, IDESC, 1u);               // hl
                    umma_f16(dc, a2, c0, IDESC, 1u);               // lh
                    umma_f16(dc, a1, c1, IDESC, 1u);               // mm
                }
                umma_commit(&sm.mbar[s]);
            }
            pending[s] = true;
            fresh = false;
            const bool last = i0 + kTcK >= nst;
            if ((kc % kFlush) == kFlush - 1 || last) {
                // drain both stages (older first), then fold the FP32 block into FP64
                const int so = s ^ 1;
                if (pending[so]) {
                    if (!mbar_wait(&sm.mbar[so], phase[so])) failed = true;
                    phase[so] ^= 1u;
                    pending[so] = false;
                }
                if (!mbar_wait(&sm.mbar[s], phase[s])) failed = true;
                phase[s] ^= 1u;
                pending[s] = false;
                tc_fence_after();
                if (__syncthreads_or(failed)) {
                    failed = true;
                    break;
                }
#pragma unroll
                for (int part = 0; part < 2; ++part)
#pragma unroll
                    for (int c0 = 0; c0 < N; c0 += 32) {
                        float v[32];
                        tmem_ld32(tbase + tlane + (uint32_t)(h * 2 * N + part * N + c0), v);
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (c0 + j < N) acc[c0 + j] += (double)v[j];
                    }
                tc_fence_before();
                __syncthreads();
                fresh = true;
            }
        }
        if (failed) break;
        // ---- outputs: F_north / F_south per map (healpix.py:250-253) ----
        if (valid) {
            const double ssign = ((m + sd.lmin) & 1) ? -1.0 : 1.0;
            const size_t rs = (size_t)(4 * p.nside - 2 - t);
            for (int bm = 0; bm < b_cnt; ++bm) {
                if (SPIN) {
                    // GEMM + (h = 0): [FpN | FmS signed];  GEMM - (h = 1): [FmN | FpS signed]
                    double2 *Fp = F_all + (size_t)(b_lo + bm) * 2 * p.nrings * p.M;
                    double2 *Fm = Fp + (size_t)p.nrings * p.M;
                    double2 *Fn = h ? Fm : Fp, *Fs = h ? Fp : Fm;
                    Fn[(size_t)t * p.M + m] = make_double2(acc[4 * bm], acc[4 * bm + 1]);
                    if (t < p.T - 1) Fs[rs * p.M + m] = make_double2(ssign * acc[4 * bm + 2], ssign * acc[4 * bm + 3]);
                } else {
                    double2 *F = F_all + (size_t)(b_lo + bm) * p.nrings * p.M;
                    F[(size_t)t * p.M + m] = make_double2(acc[4 * bm], acc[4 * bm + 1]);
                    if (t < p.T - 1) F[rs * p.M + m] = make_double2(acc[4 * bm + 2], acc[4 * bm + 3]);
                }
            }
        }
    }
    if (failed && tid == 0) atomicExch(p.err, 1);
    // release tensor memory once every issued MMA has completed (bounded)
    for (int s = 0; s < 2; ++s)
        if (pending[s]) {
            mbar_wait(&sm.mbar[s], phase[s]);
            pending[s] = false;
        }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tbase, TCOLS);
}

}  // namespace

int tc_smem_bytes(int spin) {
    return (spin ? (int)sizeof(TcSmem<2, kTcMaps>) : (int)sizeof(TcSmem<0, kTcMaps>)) + 1024;
}

int launch_tc_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s) {
    if (nb <= 0) return JHTB_OK;
    JHTB_CUDA_TRY(cudaMemsetAsync(p.d_counter, 0, sizeof(unsigned), s));
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
    q.counter = p.d_counter;
    q.err = p.d_err;
    const int smem = tc_smem_bytes(p.spin);
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (p.spin) {
        auto k = tc_synth_kernel<2, kTcMaps>;
        JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 2 * kTcRows, smem);
        k<<<nsm * std::max(2, per_sm), 2 * kTcRows, smem, s>>>(q, alm, F, nb);
    } else {
        auto k = tc_synth_kernel<0, kTcMaps>;
        JHTB_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTcRows, smem);
        k<<<nsm * std::max(2, per_sm), kTcRows, smem, s>>>(q, alm, F, nb);
    }
    JHTB_CUDA_TRY(cudaGetLastError());
    return JHTB_OK;
}

}  // namespace jhtb
