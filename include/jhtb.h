/*
 * jhtb -- B200 (sm_100a) on-grid HEALPix spherical-harmonic transforms.
 *
 * Plain C ABI: opaque plan handle, device pointers, sizes, a CUDA stream passed
 * as void*.  No C++ or torch types cross this boundary.  Every function returns
 * an int status (JHTB_OK == 0); on failure jhtb_last_error() describes it.
 * Nothing aborts or traps.
 *
 * Conventions (those of jht, src/jht/healpix.py:1-24):
 *   - a_lm: healpy m-major packing, idx(l,m) = m(2 lmax + 1 - m)/2 + l, m >= 0 only,
 *     K = (lmax+1)(lmax+2)/2 complex128 per component;
 *   - orthonormal Y_lm with the Condon-Shortley phase, map = sum a_lm Y_lm;
 *   - spin 2: components (E, B) <-> (Q, U), COSMO convention;
 *   - maps: RING order, Npix = 12 nside^2 float64 per component.
 * Batched layouts: alm [batch][ncomp][K] complex128, maps [batch][ncomp][Npix]
 * float64, with ncomp = 1 (spin 0) or 2 (spin 2).
 *
 * Each entry point replaces one jht function (file:line in jht v0.2.0):
 *   jhtb_plan_create        healpix.py:184-357  (_prepare: geometry, recursion plan, FFT plan)
 *   jhtb_synthesis          healpix.py:363-387  (synthesis)
 *   jhtb_adjoint_synthesis  healpix.py:390-412  (adjoint_synthesis)
 *   jhtb_weighted_residual  _analysis.py:49-52, :58-60 (W * m and W * (m - S a))
 *   jhtb_axpy               _analysis.py:60  (a + bare_analysis(...)), masked.py:313 (CG updates)
 *   jhtb_dot                masked.py:313  (the inner products of the CG solve)
 *   jhtb_plan_create_rings  offgrid.py:60-88  (recursion plan at the Clenshaw-Curtis rings)
 *   jhtb_legendre_synthesis offgrid.py:155-160 (synth_contract at those rings)
 *   jhtb_legendre_adjoint   offgrid.py:163-168 (adjoint_contract at those rings)
 *   jhtb_nufft_interp       _nufft.py:164-178 (nufft2d2's window sums)
 *   jhtb_nufft_spread       _nufft.py:181-188 (nufft2d1's scatter-add)
 *   jhtb_nufft_spread_tiles _nufft.py:181-188 (the same, for points grouped by grid tile)
 */
#ifndef JHTB_H
#define JHTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JHTB_OK 0
#define JHTB_ERR_INVALID (-1)     /* bad argument (size, spin, precision, null pointer) */
#define JHTB_ERR_UNSUPPORTED (-2) /* valid request the library does not implement */
#define JHTB_ERR_CUDA (-3)        /* a CUDA runtime call failed */
#define JHTB_ERR_NOMEM (-4)       /* device allocation failed */

/* Arithmetic used by the contraction.  The recursion, seeds, coefficients and
 * the ring FFTs are FP64 in every mode. */
#define JHTB_PREC_FP64 0 /* plain FP64 everywhere */
#define JHTB_PREC_FP32 1 /* FP32 contraction, FP32 accumulation (not available yet) */
#define JHTB_PREC_BF16X3 2 /* batched: mu and a_lm rounded to FP32 and split into three BF16
                              parts; six split products per tile on the tensor cores (tcgen05),
                              FP32 accumulation folded into FP64 every 256 l */

typedef struct jhtb_plan jhtb_plan;

/* Optional host-computed seed inputs (host pointers; any member may be NULL, in
 * which case the library computes it itself in FP64).  They let a caller hand
 * over bit-identical copies of the tables its own reference implementation
 * uses, e.g. jht's NumPy plan (_recursion.py:305-333):
 *   x            [2 nside]   cos(theta) of the north-cap + equator rings
 *   logsin       [2 nside]   log sin(theta)                (spin 0 seeds)
 *   logcos_half  [2 nside]   log cos(theta/2)              (spin 2 seeds)
 *   logsin_half  [2 nside]   log sin(theta/2)              (spin 2 seeds)
 *   seed_logc    spin 0: [lmax+1] theta-independent log|lambda_mm|;
 *                spin 2: [2][lmax+1] log-factor of d^{lmin}_{-m,+2}, then of d^{lmin}_{-m,-2} */
typedef struct jhtb_host_tables {
    const double *x;
    const double *logsin;
    const double *logcos_half;
    const double *logsin_half;
    const double *seed_logc;
} jhtb_host_tables;

/* Library version, e.g. 100 for 0.1.0. */
int jhtb_version(void);

/* Copy the calling thread's last error message into buf (NUL-terminated). */
int jhtb_last_error(char *buf, size_t len);

/* Build all geometry, recursion and FFT tables for (nside, lmax, spin) on the
 * current CUDA device and allocate workspace for up to max_batch maps per
 * launch (larger batches are processed in chunks).  spin must be 0 or 2;
 * nside in [1, 4096]; lmax in [0, 16383].  tables may be NULL.
 * Replaces healpix.py:184 _prepare. */
int jhtb_plan_create(int nside, int lmax, int spin, int precision, int max_batch,
                     const jhtb_host_tables *tables, jhtb_plan **out);

/* Ring-set plan: the Legendre stage only, on nrings iso-latitude rings symmetric about
 * the equator (nrings odd; ring t and ring nrings-1-t at cos theta = +-x[t], the middle
 * ring on the equator).  tables->x (required) holds x[t] >= 0 for the northern rings
 * t < (nrings + 1) / 2, non-increasing; the other tables fields may be NULL (then
 * derived from x).  Used for the Clenshaw-Curtis rings of the off-grid transforms
 * (offgrid.py:60-88: build_recursion_plan at x_cc).  jhtb_synthesis /
 * jhtb_adjoint_synthesis reject such a plan; use jhtb_legendre_synthesis / _adjoint. */
int jhtb_plan_create_rings(int nrings, int lmax, int spin, int precision, int max_batch,
                           const jhtb_host_tables *tables, jhtb_plan **out);

/* Release every device allocation owned by the plan. */
int jhtb_plan_destroy(jhtb_plan *plan);

/* Device bytes held by the plan (tables + workspace). */
int jhtb_plan_bytes(const jhtb_plan *plan, int64_t *bytes);

/* Calls on one plan share its workspace: issue them in order on one stream (or
 * synchronise between streams).  Different plans are independent. */

/* S: alm (device, complex128 [batch][ncomp][K]) -> maps (device, float64
 * [batch][ncomp][Npix]).  Stream-ordered on `stream` (a cudaStream_t, NULL =
 * legacy default stream).  Inputs are not modified.  healpix.py:363-387. */
int jhtb_synthesis(jhtb_plan *plan, const void *alm, void *maps, int batch, void *stream);

/* S^T: maps (device float64) -> alm (device complex128), the exact transpose of
 * jhtb_synthesis in the (2 - delta_m0)-weighted alm inner product.
 * healpix.py:390-412. */
int jhtb_adjoint_synthesis(jhtb_plan *plan, const void *maps, void *alm, int batch, void *stream);

/* The Legendre stage of S alone: alm (device complex128 [batch][ncomp][K]) -> ring
 * coefficients (device complex128 [batch][ncomp][nrings][lmax+1]),
 * F[c][r][m] = sum_l lambda^{s_c}_lm(x_r) alm_c[l, m], with the spin-2 channels
 * -(E + iB) (+2) and -(E - iB) (-2).  offgrid.py:155-160 (synth_contract at the
 * Clenshaw-Curtis rings); for a HEALPix plan these are healpix.py:280-291's F before
 * the phase and the ring FFT. */
int jhtb_legendre_synthesis(jhtb_plan *plan, const void *alm, void *rings, int batch, void *stream);

/* Transpose of jhtb_legendre_synthesis over all rings: rings (complex128
 * [batch][ncomp][nrings][lmax+1]) -> alm (complex128 [batch][ncomp][K]); spin 0:
 * a_lm = sum_r lambda_lm(x_r) V[r][m]; spin 2: (1/2)(-p - n), (i/2)(p - n) with p, n the
 * +2 / -2 channel sums (healpix.py:353-354).  offgrid.py:163-168 (adjoint_contract). */
int jhtb_legendre_adjoint(jhtb_plan *plan, const void *rings, void *alm, int batch, void *stream);

/* out[i] = w(pix i) * (maps[i] - synth[i]) for every component and map in the
 * batch (synth may be NULL: out = w * maps).  w(pix) = (4 pi / Npix)(1 + ring_w[r'])
 * with r' the north partner of the pixel's ring, or 4 pi / Npix when ring_w is NULL
 * (weights.py:86-106).  ring_w: device float64 [2 nside]. */
int jhtb_weighted_residual(const jhtb_plan *plan, const double *maps, const double *synth,
                           const double *ring_w, double *out, int batch, void *stream);

/* y[i] += alpha * x[i] over n float64 values (complex data: pass 2*count). */
int jhtb_axpy(int64_t n, double alpha, const double *x, double *y, void *stream);

/* *result (device float64) = sum_i x[i] y[i] over n values, FP64, fixed reduction
 * order (bitwise reproducible).  Uses the plan's small reduction scratch, so calls
 * on one plan must be ordered on one stream. */
int jhtb_dot(const jhtb_plan *plan, int64_t n, const double *x, const double *y, double *result,
             void *stream);

/* Spin-0 FP64 synthesis that allocates nothing, for callers that cannot call
 * cudaMalloc (a host framework or plugin that owns every device allocation, or a
 * process whose device memory is already reserved).  No counterpart in jht.
 * alm: device complex128 [K]; map: device float64 [12 nside^2].  Needs no plan:
 * its only scratch is a fixed 2 MiB __device__ array inside the library, which
 * limits it to nside <= 64, lmax <= 1023 and (4 nside - 1)(lmax + 1) <= 131072
 * (larger sizes are rejected with JHTB_ERR_INVALID).  All calls share that array:
 * calls that overlap on the GPU race, so order them on one stream.  The first call
 * on each device looks up the array's address (and looks it up again when the device's
 * CUDA context has changed, e.g. after cudaDeviceReset); make it before any stream
 * capture. */
int jhtb_synthesis_noalloc(int nside, int lmax, const void *alm, void *map, void *stream);

/* ---- 2D NUFFT stages of the off-grid transforms (_nufft.py:150-191) ----
 * grid: device complex128 [nk][nm] on the (theta, phi) torus; theta, phi: device
 * float64 [npts]; W: kernel width (6, 8, 10, 14 or 16); beta: the exponential-of-
 * semicircle shape.  Point (theta, phi) reads or writes the W x W window starting at
 * ceil(coord n / 2pi - W / 2) on each axis (mod n), weights
 * exp(beta (sqrt(1 - (2t/W)^2) - 1)).  Any finite or non-finite coordinate stays
 * inside the grid. */

/* out[j] = sum of the window's weighted cells (complex128 [npts]); with dtheta and
 * dphi non-NULL also the derivatives of out[j] in theta and phi.  nufft2d2's gather
 * and window sum (_nufft.py:164-178). */
int jhtb_nufft_interp(const void *grid, int nk, int nm, int W, double beta, const double *theta,
                      const double *phi, int64_t npts, void *out, void *dtheta, void *dphi, void *stream);

/* grid += the transpose of jhtb_nufft_interp applied to vals (complex128 [npts]); the
 * caller zeroes grid first.  FP64 atomic adds: the order of the sums over points is
 * not fixed.  nufft2d1's scatter-add (_nufft.py:181-188). */
int jhtb_nufft_spread(const void *vals, const double *theta, const double *phi, int64_t npts, int nk,
                      int nm, int W, double beta, void *grid, void *stream);

/* jhtb_nufft_spread for points grouped by 32 x 32-cell tiles of the grid: segment i covers
 * points [seg_start[i], seg_start[i] + seg_count[i]) (inside [0, npts)), all keyed to tile
 * seg_tile[i] = kb * tiles_m + mb (rows kb = floor(theta nk / (64 pi)), columns
 * mb = floor(phi nm / (64 pi))).  Each segment's windows are summed in on-chip memory and
 * added to the grid once per cell; a point outside its segment's tile is added directly.
 * Same result as jhtb_nufft_spread up to the order of the sums. */
int jhtb_nufft_spread_tiles(const void *vals, const double *theta, const double *phi, int64_t npts,
                            int64_t nseg, const int64_t *seg_start, const int *seg_count,
                            const int64_t *seg_tile, int tiles_m, int nk, int nm, int W, double beta,
                            void *grid, void *stream);

/* ---- sharding over devices (no counterpart in jht, which runs on one device) ----
 * A plan can be restricted to the ring pairs of half-grid rings [t0, t1) (the
 * northern rings t0..t1-1, the equator included when t1 = 2 nside, and their
 * southern mirrors).  Synthesis then writes only the pixels of those rings (other
 * pixels of the output are left as they were) and the adjoint returns only their
 * contribution, so the adjoints of plans whose ranges cover [0, 2 nside) once sum to
 * the full adjoint.  Ranges are aligned to 256 rings. */

/* Legendre work of each group of `granule` half-grid rings (granule a positive
 * multiple of 256), in ring-recursion steps: cost[g] for g < ceil(2 nside / granule). */
int jhtb_plan_ring_costs(const jhtb_plan *plan, int granule, int64_t *cost, int ncost);

/* Restrict the plan to half-grid rings [t0, t1): 0 <= t0 < t1 <= 2 nside, t0 and t1
 * multiples of 256 (t1 may be 2 nside).  Synchronises the device. */
int jhtb_plan_set_ring_range(jhtb_plan *plan, int t0, int t1);

/* ---- diagnostics (no counterpart in jht; its profiling is by stage-timing scripts,
 * scripts/profile_adjoint.py) ---------------------------------------------------- */

/* Stages reported by jhtb_plan_timings. */
#define JHTB_STAGE_LEGENDRE_SYNTH 0 /* fused recursion + contraction, synthesis   */
#define JHTB_STAGE_RING_SYNTH 1     /* phase, fold and inverse ring DFTs           */
#define JHTB_STAGE_RING_ADJOINT 2   /* forward ring DFTs, gather and phase         */
#define JHTB_STAGE_LEGENDRE_ADJOINT 3 /* fused recursion + contraction, adjoint    */

/* When enabled, every stage launch of this plan is bracketed by CUDA events on its
 * stream.  Adds no synchronisation. */
int jhtb_plan_set_timing(jhtb_plan *plan, int enable);

/* Sum of recorded stage times (ms[4], milliseconds) and launch counts (counts[4]);
 * waits for the recorded events.  reset != 0 drops the records. */
int jhtb_plan_timings(jhtb_plan *plan, double *ms, int64_t *counts, int reset);

/* Device-side error status of the plan's kernels (0 = none, 1 = a bounded wait in a
 * tensor-core kernel timed out).  Synchronises the device to read it; resets it. */
int jhtb_plan_status(jhtb_plan *plan, int *device_error);

/* Time limit of every bounded wait inside the tensor-core kernels (mbarrier hand-offs
 * between their warp roles), in nanoseconds, 1e6 .. 6e10; default 2e9.  A wait that runs
 * out makes the kernel record status 1 (jhtb_plan_status), leave its loops, wait for its
 * own tensor-core operations in flight and release its tensor memory: the call's output
 * is then undefined but the context stays usable. */
int jhtb_plan_set_watchdog(jhtb_plan *plan, int64_t timeout_ns);

/* Tuning knobs (no counterpart in jht; chosen per configuration by jht_b200.autotune and
 * kept in its table).  None changes the transform, only the speed and, for the
 * tensor-core folds, the rounding (every allowed value keeps it within the tested bound):
 *   JHTB_TUNE_TC_FOLD   degrees per FP32 accumulation block of the tensor-core synthesis
 *                       (multiple of 16, default 256);
 *   JHTB_TUNE_TCA_FOLD  rings per FP32 accumulation block of the tensor-core adjoint
 *                       (multiple of 32, default 256);
 *   JHTB_TUNE_TC_GROUP  maps per tensor-core synthesis group, 8 or 16 (default 16);
 *   JHTB_TUNE_LEG_CTAS  CTAs per SM of the FP64 Legendre kernels, 0 = all that fit (default). */
#define JHTB_TUNE_TC_FOLD 1
#define JHTB_TUNE_TCA_FOLD 2
#define JHTB_TUNE_TC_GROUP 3
#define JHTB_TUNE_LEG_CTAS 4
int jhtb_plan_set_tuning(jhtb_plan *plan, int key, int value);

/* Fault injection for tests of that failure path (no GPU fault is raised).
 * JHTB_FAULT_STALL: the tensor-core kernels' operand builders publish nothing, so the
 * waits on them run out after the watchdog limit.  0 switches injection off. */
#define JHTB_FAULT_STALL 1
int jhtb_plan_inject_fault(jhtb_plan *plan, int kind);

/* Batched complex FP64 FFT of a 2,3,5-smooth length n <= 10240 (replaces the jnp.fft calls of
 * jht's off-grid transforms, _nufft.py:164-191; longer transforms are composed by the caller
 * from two calls, four-step).  Transform b = o * inner + t (o < howmany / inner, t < inner)
 * reads x[i] = in[o * in_dist_outer + t * in_dist_inner + i * in_stride] (complex128
 * elements) and writes out[o * out_dist_outer + t * out_dist_inner + k * out_stride] =
 * scale * w_k * sum_i x[i] e^{sign 2 pi i i k / n}, with w_k = e^{sign 2 pi i (t k mod
 * twiddle_n) / twiddle_n} when twiddle_n > 0 (the four-step twiddle), else 1.  sign = -1
 * (forward) or +1.  roots: device table of e^{-2 pi i k / n} for k < n (complex128), or NULL
 * to compute each butterfly's root.  In place (out == in) only with the same input and
 * output layout. */
int jhtb_fft_c2c(const void *in, void *out, int n, int64_t howmany, int64_t inner, int64_t in_stride,
                 int64_t in_dist_outer, int64_t in_dist_inner, int64_t out_stride, int64_t out_dist_outer,
                 int64_t out_dist_inner, int sign, double scale, int64_t twiddle_n, const void *roots, void *stream);

/* Bounds-check record of a debug library (no counterpart in jht; the replacement for a
 * memory checker on machines where none can run).  A library built with `make debug`
 * (jht_b200/_lib_debug/libjhtb.so, -DJHTB_DEBUG) tests every checked gather and scatter
 * index of its kernels against the extent of its buffer and skips an access out of range;
 * this call waits for the device, returns the number of such accesses since the last call
 * and the first one's site code, index and extent, and clears the record.  The release
 * library compiles no checks and returns JHTB_ERR_UNSUPPORTED. */
int jhtb_debug_bounds(int64_t *count, int *site, int64_t *index, int64_t *extent);

/* FP64 FMA throughput probe: a grid of 148*blocks_per_sm CTAs x 256 threads, each
 * running 8 independent FMA chains for `iters` steps.  Writes the elapsed time of
 * the launch (CUDA events on `stream`) to *ms and the FLOP count (2 per FMA) to
 * *flops; sink (device, >= 1 double) keeps the result live. */
int jhtb_probe_fp64_fma(int blocks_per_sm, int iters, double *sink, double *ms, double *flops, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* JHTB_H */
