// Internal definitions shared by the jhtb CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/jhtb.h"

namespace jhtb {

// ---------------------------------------------------------------------------------
// error reporting (thread-local last error, int status codes; never abort)
// ---------------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

#define JHTB_CUDA_TRY(expr)                                   \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return ::jhtb::cuda_fail(_e, #expr); \
    } while (0)

// ---------------------------------------------------------------------------------
// scaled representation of the recursion: value = mant * 2^(800 * sc), sc <= 0.
// While sc < 0 the value is far below any contribution that matters and is not
// accumulated; when |mant| exceeds 2^400 it is rescaled by 2^-800 and sc steps up.
// ---------------------------------------------------------------------------------
constexpr double kBig = 0x1p400;
constexpr double kScaleDown = 0x1p-800;
constexpr double kLogScaleHi = 554.5177444475703;     // 800 ln 2, 41 significant bits
constexpr double kLogScaleLo = 3.85953392016288e-10;  // 800 ln 2 - kLogScaleHi
constexpr double kLn2x400 = 277.25887222397812;       // 400 ln 2

// Legendre kernels: half-grid rings per lane (a warp tile is 32 * R consecutive rings).
#ifndef JHTB_R0
#define JHTB_R0 4
#endif
#ifndef JHTB_R2
#define JHTB_R2 2
#endif
constexpr int kR0 = JHTB_R0;  // spin 0
constexpr int kR2 = JHTB_R2;  // spin 2
// The adjoint sums each l over the rings of a warp tile: wider tiles (more rings per
// lane) spend fewer instructions on the cross-lane sum per ring.
#ifndef JHTB_RA0
#define JHTB_RA0 4
#endif
#ifndef JHTB_RA2
#define JHTB_RA2 4
#endif
constexpr int kRA0 = JHTB_RA0;  // adjoint, spin 0
constexpr int kRA2 = JHTB_RA2;  // adjoint, spin 2
#ifndef JHTB_TC_MAPS
#define JHTB_TC_MAPS 16
#endif
constexpr int kTcMaps = JHTB_TC_MAPS;  // maps per tensor-core pass (N = 4 * maps per GEMM)

// FFT: largest power-of-two length handled in one CTA's shared memory.
constexpr int kFftMax = 8192;    // largest power-of-two ring handled by the direct path per piece plan
constexpr int kTwLen = 32768;    // twiddle table length: every FFT and split length divides it
constexpr int kFftPiece = 4096;  // largest FFT held in shared memory; longer ones run in pieces
constexpr int kFftLogMax = 13;

// Ring FFT modes: kDirect (N a power of two), kBluestein (chirp-z of length N), kSplit4
// (N = 4 i: four chirp-z transforms of length i and a radix-4 combination).
enum RingMode : int { kDirect = 0, kBluestein = 1, kSplit4 = 2 };

struct RingDesc {
    int N;          // pixels in the ring
    int mode;       // RingMode
    int P;          // FFT length: N (direct), Bluestein length (power of two >= 2N-1), or for
                    // kSplit4 the Bluestein length of the quarter ring (power of two >= N/2-1)
    int Q;          // pieces of P / Q <= kFftPiece points (1, 2, 4 or 8) in the piecewise path
    long long start;   // first pixel
    long long bh_off;  // offset (complex units) of this length's chirp spectrum
    double phi0;       // azimuth of the first pixel
};

// Pieces a ring's transform runs in, one CTA each (1: the whole ring in one CTA): a
// power-of-two ring above kFftPiece points in N / kFftPiece pieces, a kSplit4 ring in 4.
__host__ __device__ __forceinline__ int ring_pieces(const RingDesc &rd) {
    if (rd.mode == kSplit4) return 4;
    if (rd.mode == kDirect && rd.N > kFftPiece && 2 * rd.N <= kTwLen) return rd.N / kFftPiece;
    return 1;
}

// Per-m seed parameters.  Spin 0: lf = theta-independent log|lambda_mm|,
// sign = (-1)^m, pc = ps = 0.  Spin +-2: log|d^{lmin}_{-m,+-2}| = lf + pc log cos(t/2)
// + ps log sin(t/2) with sign (_recursion.py:166-188).
struct SeedParam {
    double lf[2];
    double sign[2];
    int pc[2];
    int ps[2];
    int lmin;
    int pad;
};

// One work item of the tensor-core adjoint: order m, block lb of 128 degrees (l from
// lmin + 128 lb), the ring chunks [c0, c1) it streams, the block's first live ring chunk
// cl (<= c0) and the offset soff of its rows in the segment-state table.
struct TcaItem {
    int m, lb, c0, c1, cl, pad;
    long long soff;
};

struct Plan {
    int nside, lmax, spin, precision, max_batch;
    int T;         // half-grid rings (north cap + equator) = 2 nside
    int nrings;    // 4 nside - 1
    int M;         // lmax + 1
    long long K;   // packed alm size
    long long npix;
    bool rings_only;    // ring-set plan (no pixel grid): the Legendre stage only
    int ncomp;     // 1 (spin 0) or 2 (spin 2)
    int npairs;    // m-pairs (m, lmax - m)

    // geometry (device)
    double *d_x;        // [T] cos theta
    double *d_logsin;   // [T] log sin theta       (spin 0 seeds)
    double *d_logch;    // [T] log cos(theta/2)    (spin 2 seeds)
    double *d_logsh;    // [T] log sin(theta/2)
    RingDesc *d_rings;  // [nrings]
    double2 *d_tw;      // [kTwLen] exp(-2 pi i k / kTwLen)
    double2 *d_bh;      // Bluestein chirp spectra, FFT_P(conj(w))/P, per distinct length
    long long bh_len;

    // recursion tables (device), packed like the alm
    SeedParam *d_seed;  // [M]
    double *d_alpha;    // [K]
    double *d_gamma;    // [K] (spin 2)
    double *d_cnorm;    // [K]

    // Legendre work items (plan creation): start l and recursion state per (m, warp tile),
    // cost-sorted item orders for the persistent kernels
    int ntiles;          // synthesis warp tiles per m (32 kR rings)
    int *d_lw;           // [M * ntiles]
    double2 *d_st;       // [M * ntiles][nrec][R][32]
    int *d_stsc;         // [M * ntiles][nrec][R][32]
    int *d_synth_order;  // [M * ntiles]
    // adjoint warp tiles (32 kRA rings): the synthesis tables when kRA == kR
    int a_ntiles;
    int nsuper, tps;     // ring quarters per m, adjoint warp tiles per quarter
    int *d_a_lw;
    double2 *d_a_st;
    int *d_a_stsc;
    bool a_owns_tables;
    int *d_adj_order;    // [M * nsuper]
    int *d_adj_tiles;    // [M * nsuper][tps]
    unsigned *d_counter; // work-queue counter
    double2 *d_part;     // [chunk][nsuper][ncomp][K] adjoint partial sums

    // tensor-core path (precision BF16X3): 128-ring (spin 2) or 256-ring (spin 0) tiles;
    // the start tables are the adjoint's when their tile widths agree
    int tc_ntiles;
    int *d_tc_lw;
    double2 *d_tc_st;
    int *d_tc_stsc;
    int *d_tc_order;
    bool tc_owns_tables;
    int *d_err;           // device error flag
    // tensor-core adjoint (precision BF16X3): recursion state at the start of every
    // 32-degree segment of every 128-degree block, for the block's live ring chunks only
    // (rows [block][chunk - cl][segment][32 lanes], lane = recursion x 16 rings for spin 2,
    // 32 rings for spin 0), the items, and the BF16x3 ring-data tiles of one 16-map group
    // [M][nchunk][12 KB]
    long long tca_nblk;
    long long tca_nstate;   // rows of the segment-state table
    int *d_tca_blk_off;     // [M] first block of each order
    int *d_tca_blk_cl;      // [block] first live ring chunk
    long long *d_tca_blk_soff;  // [block] first row in the segment-state table
    double2 *d_tca_st;      // (mu_{l-1}, mu_{l-2}) before the segment's first step
    short *d_tca_sc;        // the state's scale exponent
    TcaItem *d_tca_items;
    int tca_nitems;
    int tca_nchunk;         // ring chunks of the half grid (16 rings spin 2, 32 spin 0)
    unsigned char *d_tca_B;
    double2 *d_ag;          // (alpha, gamma) interleaved, packed like the alm (spin 2)
    std::vector<int> h_tca_blk_off, h_tca_blk_cl;
    std::vector<long long> h_tca_blk_soff;
    // tensor-core synthesis (precision BF16X3): prepared coefficient chunks of one map
    // group, one per (order, 16 degrees from lmin) [chunk][bytes]
    long long tcs_nchunks;
    int *d_tcs_chunk_m;     // [tcs_nchunks] order of each chunk
    int *d_tcs_cbase;       // [M] first chunk of each order
    unsigned char *d_tcs_B;
    unsigned long long tc_wait_ns = 2000000000ull;  // time limit of the tensor-core kernels' waits
    // tuning (jhtb_plan_set_tuning): FP32 accumulation block of the tensor-core synthesis
    // (degrees) and adjoint (rings), maps per tensor-core synthesis group, CTAs per SM of
    // the FP64 persistent kernels (0 = as many as fit)
    int tc_fold = 256, tca_fold = 256, tc_group = 16, leg_ctas = 0;
    int inject = 0;       // fault injection for tests (kInjectStall)

    // ring-pair range of the plan (sharding over devices): half-grid rings
    // [ring_t0, ring_t1) and their southern mirrors; the whole grid by default
    int ring_t0, ring_t1;
    int nsynth;           // entries of d_synth_order (items inside the range)
    int tc_norder;        // entries of d_tc_order
    // rings of the plan's range by kernel: ring_small (one 256-thread CTA per ring, pieces
    // through global scratch above kFftPiece points) and ring_piece ((ring << 3 | piece)
    // work units of the rings that run in pieces, ring_pieces() > 1)
    int *d_ring_small, *d_ring_piece;
    int nring_small, nring_piece;
    std::vector<unsigned char> h_ring_pieces;  // [ring] pieces of its transform (1: the one-CTA kernel)
    std::vector<int> h_lw, h_a_lw, h_tc_lw;  // start l per item, kept for re-sorting

    // workspace
    double2 *d_F;       // [chunk][nchan][nrings][M] ring spectra
    double2 *d_W;       // [chunk][npix] ring scratch rows of the split transforms
    double2 *d_W2;      // [chunk][npix] second scratch row (phased input / piece sums)
    double *d_scratch;  // small reduction scratch
    int chunk;          // maps per workspace pass
    size_t bytes;

    // optional per-stage timing (CUDA events recorded on the launch stream)
    bool timing;
    struct StageEvent {
        cudaEvent_t start, stop;
        int stage;
    };
    std::vector<StageEvent> events;
};

// Fault injection (tests of the failure path; no GPU fault is raised): the tensor-core
// kernels' builder warps publish no operand stage, so the waits on them run out.
constexpr int kInjectStall = JHTB_FAULT_STALL;

enum Stage : int { kStageLegSynth = 0, kStageRingSynth = 1, kStageRingAdj = 2, kStageLegAdj = 3, kNumStages = 4 };

// kernels launchers (return 0 or a jhtb status)
int launch_legendre_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s);
int launch_legendre_adjoint(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s);
int launch_ring_synth(const Plan &p, const double2 *F, double *maps, int nb, cudaStream_t s);
int launch_ring_adjoint(const Plan &p, const double *maps, double2 *F, double2 *W, int nb,
                        cudaStream_t s);
int launch_start_states(const Plan &p, cudaStream_t s);
int launch_start_states_r(const Plan &p, int R, int ntiles, int *lw, double2 *st, int *stsc, cudaStream_t s);
int launch_tc_synth(const Plan &p, const double2 *alm, double2 *F, int nb, cudaStream_t s);
int launch_tc_adjoint(const Plan &p, const double2 *F, double2 *alm, int nb, cudaStream_t s);
size_t tc_synth_chunk_bytes(int spin);
int launch_tca_block_states(const Plan &p, cudaStream_t s);
constexpr int kTcaLB = 128;       // degrees per tensor-core adjoint item (= MMA M)
constexpr int kTcaSeg = 4;        // recursion segments per item (independent chains per thread)
constexpr int kTcaMaps = 16;      // maps per tensor-core adjoint group
constexpr int kTcaBStage = 12288; // bytes of one ring chunk's BF16x3 tiles (2 x 3 x 64 x 16 x 2)
int launch_bluestein_setup(const Plan &p, const int *lengths, const long long *offs, int nlen,
                           cudaStream_t s);
constexpr int kRingGranule = 256;  // alignment of ring ranges: a multiple of every tile width

__host__ __device__ inline long long alm_index(long long l, long long m, long long lmax) {
    return m * (2 * lmax + 1 - m) / 2 + l;
}

// ---------------------------------------------------------------------------------
// Debug bounds checks (a library built with -DJHTB_DEBUG: `make debug`).  Every checked
// gather or scatter tests its index against the extent of its buffer; an access out of
// range is skipped (a load reads zero), and the number of failures with the first one's
// site, index and extent is kept in a device record per translation unit, which
// jhtb_debug_bounds() collects.  Without JHTB_DEBUG a check is the constant true and the
// access is unchanged.  Site numbers: 1xx azimuthal stage, 2xx FP64 Legendre kernels,
// 3xx tensor-core synthesis, 4xx tensor-core adjoint, 5xx vector kernels.
// ---------------------------------------------------------------------------------
struct DebugRecord {
    unsigned long long count;
    long long index, extent;
    int site, pad;
};
#ifdef JHTB_DEBUG
static __device__ DebugRecord g_debug_record;
__device__ __forceinline__ bool debug_in_range(long long i, long long n, int site) {
    if (i >= 0 && i < n) return true;
    if (atomicAdd(&g_debug_record.count, 1ull) == 0ull) {
        g_debug_record.site = site;
        g_debug_record.index = i;
        g_debug_record.extent = n;
    }
    return false;
}
#define JHTB_IN(i, n, site) ::jhtb::debug_in_range((long long)(i), (long long)(n), (site))
// the record of this translation unit: copied out and, with reset, cleared
#define JHTB_DEBUG_ACCESSOR(name)                                                            \
    int debug_record_##name(::jhtb::DebugRecord *out, bool reset) {                          \
        if (cudaMemcpyFromSymbol(out, g_debug_record, sizeof(::jhtb::DebugRecord)) != cudaSuccess) \
            return 1;                                                                         \
        if (reset) {                                                                          \
            const ::jhtb::DebugRecord z{};                                                    \
            if (cudaMemcpyToSymbol(g_debug_record, &z, sizeof(z)) != cudaSuccess) return 1;   \
        }                                                                                     \
        return 0;                                                                             \
    }
#else
#define JHTB_IN(i, n, site) true
#define JHTB_DEBUG_ACCESSOR(name)
#endif
int debug_record_legendre(DebugRecord *out, bool reset);
int debug_record_ringfft(DebugRecord *out, bool reset);
int debug_record_tc_synth(DebugRecord *out, bool reset);
int debug_record_tc_adjoint(DebugRecord *out, bool reset);
int debug_record_vecops(DebugRecord *out, bool reset);

}  // namespace jhtb
