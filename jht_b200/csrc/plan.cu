// Plan construction and the C ABI entry points.
//
// A plan holds, on the device, everything that depends only on (nside, lmax,
// spin): the RING geometry (jht healpix.py:107-140), per-m recursion seeds
// (_recursion.py:53-56, :166-188), the normalised three-term recursion
// coefficients, the per-ring FFT descriptors with Bluestein chirp spectra, and
// the ring-spectrum workspace.  It replaces jht's lru-cached _prepare
// (healpix.py:184-357), which builds the same information as NumPy constants.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "jhtb_internal.cuh"

namespace jhtb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    set_error(m);
    // a failed allocation (or other non-sticky error) also sets the runtime's per-thread
    // last error; clear it so that the caller's next CUDA call does not report it again
    (void)cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? JHTB_ERR_NOMEM : JHTB_ERR_CUDA;
}

namespace {

bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

long long next_pow2(long long n) {
    long long p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Compensated sum, for the theta-independent log of the sectoral seed.
double kahan_log_const(int m) {
    double s = -0.5 * std::log(4.0 * M_PI), c = 0.0;
    for (int k = 1; k <= m; ++k) {
        double y = 0.5 * std::log((2.0 * k + 1.0) / (2.0 * k)) - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
    return s;
}

// log|d^{lmin}_{M,M'}| constant, sign and the powers of cos(t/2), sin(t/2)
// (_recursion.py:166-188).
void wigner_seed_param(int M, int Mp, int lmin, double &lf, double &sign, int &pc, int &ps) {
    int k0 = std::max(0, M - Mp);
    lf = 0.5 * (std::lgamma(lmin + M + 1.0) + std::lgamma(lmin - M + 1.0) +
                std::lgamma(lmin + Mp + 1.0) + std::lgamma(lmin - Mp + 1.0)) -
         (std::lgamma(k0 + 1.0) + std::lgamma(lmin + M - k0 + 1.0) +
          std::lgamma(lmin - Mp - k0 + 1.0) + std::lgamma(k0 - M + Mp + 1.0));
    sign = (k0 % 2) ? -1.0 : 1.0;
    pc = 2 * lmin - 2 * k0 + M - Mp;
    ps = 2 * k0 - M + Mp;
}

template <typename T>
int upload(T **dptr, const std::vector<T> &h, size_t &bytes) {
    size_t n = h.size() * sizeof(T);
    if (n == 0) n = sizeof(T);
    JHTB_CUDA_TRY(cudaMalloc((void **)dptr, n));
    bytes += n;
    if (!h.empty()) JHTB_CUDA_TRY(cudaMemcpy(*dptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return JHTB_OK;
}

void free_plan(Plan *p) {
    if (!p) return;
    void *ptrs[] = {p->d_x,     p->d_logsin, p->d_logch, p->d_logsh,   p->d_rings, p->d_tw,
                    p->d_bh,    p->d_seed,   p->d_alpha, p->d_gamma,   p->d_cnorm, p->d_F,
                    p->d_W,     p->d_W2,     p->d_scratch, p->d_lw, p->d_st, p->d_stsc, p->d_synth_order,
                    p->d_adj_order, p->d_adj_tiles, p->d_counter, p->d_part, p->d_err, p->d_ring_small, p->d_ring_piece};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (p->a_owns_tables) {
        void *a[] = {p->d_a_lw, p->d_a_st, p->d_a_stsc};
        for (void *q : a)
            if (q) cudaFree(q);
    }
    if (p->tc_owns_tables) {
        void *tc[] = {p->d_tc_lw, p->d_tc_st, p->d_tc_stsc};
        for (void *q : tc)
            if (q) cudaFree(q);
    }
    if (p->d_tc_order) cudaFree(p->d_tc_order);
    void *tca[] = {p->d_tca_blk_off, p->d_tca_blk_cl, p->d_tca_blk_soff, p->d_tca_st, p->d_tca_sc, p->d_tca_items,
                   p->d_tca_B, p->d_ag, p->d_tcs_chunk_m, p->d_tcs_cbase, p->d_tcs_B};
    for (void *q : tca)
        if (q) cudaFree(q);
    for (auto &e : p->events) {
        cudaEventDestroy(e.start);
        cudaEventDestroy(e.stop);
    }
    delete p;
}

// Cost-sorted item orders of the persistent kernels, restricted to the items whose
// tile lies inside the plan's ring range, and the ring list of the azimuthal stage.
// Called at plan creation and again whenever the range changes.
int build_ring_lists(Plan *p, size_t &bytes);

int build_orders(Plan *p) {
    const int L = p->lmax, M = p->M;
    const int t0 = p->ring_t0, t1 = p->ring_t1;
    size_t bytes = 0;
    auto refresh = [&](int **dptr, const std::vector<int> &h) -> int {
        if (*dptr) cudaFree(*dptr);
        *dptr = nullptr;
        return upload(dptr, h, bytes);
    };
    int rc;
    // FP64 synthesis: tiles of 32 kR rings, one item each
    {
        const int tw = 32 * (p->spin ? kR2 : kR0);
        const std::vector<int> &lw = p->h_lw;
        auto cost = [&](long long it) { return std::max(0, L + 1 - lw[it]); };
        std::vector<int> so;
        for (long long i = 0; i < (long long)M * p->ntiles; ++i) {
            const int tile = (int)(i % p->ntiles);
            if (tile * tw >= t0 && tile * tw < t1) so.push_back((int)i);
        }
        std::stable_sort(so.begin(), so.end(), [&](int a, int b) { return cost(a) > cost(b); });
        p->nsynth = (int)so.size();
        if ((rc = refresh(&p->d_synth_order, so))) return rc;
    }
    // FP64 adjoint: tiles of 32 kRA rings grouped into ring quarters (one item each)
    {
        const int tw = 32 * (p->spin ? kRA2 : kRA0);
        const int nt = p->a_ntiles;
        const std::vector<int> &lw = p->h_a_lw;
        auto in_range = [&](int tile) { return tile * tw >= t0 && tile * tw < t1; };
        auto cost = [&](long long it) { return std::max(0, L + 1 - lw[it]); };
        const long long nsup = (long long)M * p->nsuper;
        std::vector<int> at((size_t)nsup * p->tps, -1), ao(nsup);
        std::vector<long long> acost(nsup, 0);
        for (int m = 0; m < M; ++m)
            for (int s = 0; s < p->nsuper; ++s) {
                std::vector<int> tl;
                for (int t = s * p->tps; t < std::min((s + 1) * p->tps, nt); ++t)
                    if (in_range(t)) tl.push_back(t);
                std::stable_sort(tl.begin(), tl.end(), [&](int a, int b) {
                    return lw[(long long)m * nt + a] < lw[(long long)m * nt + b];
                });
                const long long si = (long long)m * p->nsuper + s;
                for (size_t j = 0; j < tl.size(); ++j) {
                    at[si * p->tps + j] = tl[j];
                    acost[si] += cost((long long)m * nt + tl[j]);
                }
                ao[si] = (int)si;
            }
        std::stable_sort(ao.begin(), ao.end(), [&](int a, int b) { return acost[a] > acost[b]; });
        if ((rc = refresh(&p->d_adj_order, ao))) return rc;
        if ((rc = refresh(&p->d_adj_tiles, at))) return rc;
    }
    // tensor-core kernel: tiles of 128 (spin 2) or 256 (spin 0) rings
    if (p->precision == JHTB_PREC_BF16X3) {
        const int tw = p->spin ? 128 : 256;
        const std::vector<int> &lw = p->h_tc_lw;
        std::vector<int> so;
        for (long long i = 0; i < (long long)M * p->tc_ntiles; ++i) {
            const int tile = (int)(i % p->tc_ntiles);
            if (tile * tw >= t0 && tile * tw < t1) so.push_back((int)i);
        }
        // in order of m: the CTAs working at one time share the orders' coefficient chunks in L2
        (void)lw;
        p->tc_norder = (int)so.size();
        if ((rc = refresh(&p->d_tc_order, so))) return rc;
    }
    // tensor-core adjoint: items (order, 128-degree block) in order of m, each streaming the
    // ring chunks from the first 128-ring tile that is live in the block to the equator,
    // clipped to the plan's ring range
    if (p->precision == JHTB_PREC_BF16X3) {
        const int CR = p->spin ? 16 : 32;
        const int nt = p->a_ntiles, tw = 32 * (p->spin ? kRA2 : kRA0);
        const std::vector<int> &lw = p->h_a_lw;
        std::vector<TcaItem> items;
        const int clo = t0 / CR, chi = std::min(p->tca_nchunk, (t1 + CR - 1) / CR);
        (void)nt;
        (void)tw;
        (void)lw;
        for (int m = 0; m < M; ++m) {
            const int lmin = p->spin ? std::max(m, 2) : m;
            const int nblk = (L - lmin + 1 + kTcaLB - 1) / kTcaLB;
            for (int lb = 0; lb < nblk; ++lb) {
                const int blk = p->h_tca_blk_off[m] + lb;
                TcaItem it;
                it.m = m;
                it.lb = lb;
                it.cl = p->h_tca_blk_cl[blk];
                it.c0 = std::max(clo, std::min(chi, it.cl));
                it.c1 = chi;
                it.pad = 0;
                it.soff = p->h_tca_blk_soff[blk];
                items.push_back(it);
            }
        }
        p->tca_nitems = (int)items.size();
        if (p->d_tca_items) cudaFree(p->d_tca_items);
        p->d_tca_items = nullptr;
        if ((rc = upload(&p->d_tca_items, items, bytes))) return rc;
    }
    if (!p->h_ring_pieces.empty() && (rc = build_ring_lists(p, bytes))) return rc;
    return JHTB_OK;
}

// Azimuthal stage: the range's northern rings and their southern mirrors, split by the
// kernel that transforms them (whole rings in one CTA; (ring << 3 | piece) units of the
// rings that run in pieces, a ring's pieces adjacent so that they read its data from L2
// together); within each list the rings keep their order.
int build_ring_lists(Plan *p, size_t &bytes) {
    const int T = p->T, t0 = p->ring_t0, t1 = p->ring_t1;
    int rc;
    for (int **q : {&p->d_ring_small, &p->d_ring_piece})
        if (*q) cudaFree(*q);
    p->d_ring_small = p->d_ring_piece = nullptr;
    std::vector<int> small, whole;
    auto add = [&](int r) { (p->h_ring_pieces[r] > 1 ? whole : small).push_back(r); };
    for (int t = t0; t < t1; ++t) {
        add(t);
        if (t < T - 1) add(p->nrings - 1 - t);
    }
    std::sort(small.begin(), small.end());
    std::sort(whole.begin(), whole.end());
    std::vector<int> pieces;
    for (int r : whole)
        for (int s = 0; s < p->h_ring_pieces[r]; ++s) pieces.push_back(r << 3 | s);
    p->nring_small = (int)small.size();
    p->nring_piece = (int)pieces.size();
    if ((rc = upload(&p->d_ring_small, small, bytes))) return rc;
    if ((rc = upload(&p->d_ring_piece, pieces, bytes))) return rc;
    return JHTB_OK;
}

int build_plan(Plan *p, const jhtb_host_tables *ht) {
    const int nside = p->nside, L = p->lmax, spin = p->spin;
    const int T = p->T, M = p->M, nr = p->nrings;
    size_t &bytes = p->bytes;

    // ---- RING geometry (healpix.py:107-140) -----------------------------------------
    std::vector<double> z(nr), phi0(nr);
    std::vector<long long> npr(nr), start(nr);
    const double ns2 = 3.0 * (double)((long long)nside * nside);
    for (int r = 0; r < (p->rings_only ? 0 : nr); ++r) {
        long long i = r + 1;
        if (i < nside) {
            npr[r] = 4 * i;
            z[r] = 1.0 - (double)(i * i) / ns2;
            phi0[r] = M_PI / (4.0 * (double)i);
        } else if (i > 3LL * nside) {
            long long ii = 4LL * nside - i;
            npr[r] = 4 * ii;
            z[r] = -(1.0 - (double)(ii * ii) / ns2);
            phi0[r] = M_PI / (4.0 * (double)ii);
        } else {
            npr[r] = 4LL * nside;
            z[r] = 4.0 / 3.0 - (2.0 * (double)i) / (3.0 * (double)nside);
            phi0[r] = ((i - nside) % 2 == 0) ? M_PI / (4.0 * (double)nside) : 0.0;
        }
        start[r] = r == 0 ? 0 : start[r - 1] + npr[r - 1];
    }

    // ---- half-grid seed inputs ----------------------------------------------------------
    std::vector<double> x(T), lsin(T), lch(T), lsh(T);
    for (int t = 0; t < T; ++t) {
        x[t] = ht && ht->x ? ht->x[t] : z[t];
        double xx = x[t];
        double s2 = std::min(std::max(1.0 - xx * xx, 0.0), 1.0);
        double c2 = std::min(std::max((1.0 + xx) / 2.0, 0.0), 1.0);
        double h2 = std::min(std::max((1.0 - xx) / 2.0, 0.0), 1.0);
        lsin[t] = ht && ht->logsin ? ht->logsin[t] : std::log(std::sqrt(s2));
        lch[t] = ht && ht->logcos_half ? ht->logcos_half[t] : std::log(std::sqrt(c2));
        lsh[t] = ht && ht->logsin_half ? ht->logsin_half[t] : std::log(std::sqrt(h2));
    }
    int rc;
    if ((rc = upload(&p->d_x, x, bytes))) return rc;
    if ((rc = upload(&p->d_logsin, lsin, bytes))) return rc;
    if ((rc = upload(&p->d_logch, lch, bytes))) return rc;
    if ((rc = upload(&p->d_logsh, lsh, bytes))) return rc;

    // ---- per-m seeds ---------------------------------------------------------------------
    std::vector<SeedParam> seeds(M);
    for (int m = 0; m < M; ++m) {
        SeedParam &sp = seeds[m];
        std::memset(&sp, 0, sizeof(sp));
        if (spin == 0) {
            sp.lmin = m;
            sp.lf[0] = ht && ht->seed_logc ? ht->seed_logc[m] : kahan_log_const(m);
            sp.sign[0] = (m % 2) ? -1.0 : 1.0;
        } else {
            sp.lmin = std::max(m, 2);
            for (int h = 0; h < 2; ++h) {
                int s = h == 0 ? 2 : -2;
                wigner_seed_param(-m, s, sp.lmin, sp.lf[h], sp.sign[h], sp.pc[h], sp.ps[h]);
                if (ht && ht->seed_logc) sp.lf[h] = ht->seed_logc[h * M + m];
            }
        }
    }
    if ((rc = upload(&p->d_seed, seeds, bytes))) return rc;

    // ---- normalised recursion coefficients ------------------------------------------------
    // y_l = (P_l x + Q_l) y_{l-1} - R_l y_{l-2} with y = lambda / f (f = 1 for spin 0,
    // (-1)^m sqrt((2l+1)/4pi) for spin 2).  Writing y_l = g_l mu_l with g_lmin = g_lmin+1 = 1,
    // g_l = R_l g_{l-2}, gives mu_l = (alpha_l x + gamma_l) mu_{l-1} - mu_{l-2} and
    // lambda_l = c_l mu_l, c_l = f_l g_l.  alpha = gamma = 0 at l = lmin (the seed step).
    // The tables are computed in long double (64-bit significand) and rounded once: the
    // running product g_l would otherwise carry ~sqrt(l) FP64 roundings into c_l, and at
    // degree 4096 that is a visible part of the transform's error near the poles.
    const long long K = p->K;
    std::vector<double> alpha(K, 0.0), gamma(spin ? K : 0, 0.0), cnorm(K, 0.0);
    typedef long double xr;
    const xr kPi = 3.14159265358979323846264338327950288L;
    for (int m = 0; m <= L; ++m) {
        const int lmin = seeds[m].lmin;
        xr g2 = 1.0L, g1 = 1.0L;  // g_{l-2}, g_{l-1}
        const xr fsign = (spin && (m % 2)) ? -1.0L : 1.0L;
        for (int l = lmin; l <= L; ++l) {
            const long long idx = alm_index(l, m, L);
            xr P = 0, Q = 0, R = 0;
            if (l > lmin) {
                if (spin == 0) {
                    const xr dl = l;
                    P = sqrtl((2 * dl - 1) * (2 * dl + 1) / ((dl - m) * (dl + m)));
                    R = sqrtl((2 * dl + 1) * ((dl - 1) * (dl - 1) - (xr)m * m) / ((2 * dl - 3) * (dl - m) * (dl + m)));
                } else {
                    // Wigner-d coefficients at l-1 producing d^l (_recursion.py:136-143)
                    const xr Lp = l - 1, Mm = -m, Mp = 2;
                    const xr D = Lp * sqrtl(((Lp + 1) * (Lp + 1) - Mm * Mm) * ((Lp + 1) * (Lp + 1) - Mp * Mp));
                    P = (2 * Lp + 1) * Lp * (Lp + 1) / D;
                    Q = -(2 * Lp + 1) * Mm * Mp / D;
                    R = (Lp + 1) * sqrtl((Lp * Lp - Mm * Mm) * (Lp * Lp - Mp * Mp)) / D;
                }
            }
            const xr g = (l <= lmin + 1) ? 1.0L : R * g2;
            if (l > lmin) {
                alpha[idx] = (double)(P * g1 / g);
                if (spin) gamma[idx] = (double)(Q * g1 / g);
            }
            const xr f = spin ? fsign * sqrtl((2.0L * l + 1.0L) / (4.0L * kPi)) : 1.0L;
            cnorm[idx] = (double)(f * g);
            if (l > lmin) { g2 = g1; g1 = g; } else { g2 = 1.0L; g1 = 1.0L; }
        }
    }
    if ((rc = upload(&p->d_alpha, alpha, bytes))) return rc;
    if (spin && (rc = upload(&p->d_gamma, gamma, bytes))) return rc;
    if ((rc = upload(&p->d_cnorm, cnorm, bytes))) return rc;

    // ---- Legendre work items: start states at the first representable l per warp tile,
    //      cost-sorted orders for the persistent synthesis / adjoint kernels ----------------
    {
        const int R = spin ? kR2 : kR0;
        const int nrec = spin ? 2 : 1;
        p->ntiles = (T + 32 * R - 1) / (32 * R);
        const long long nitems = (long long)M * p->ntiles;
        const size_t nst_el = (size_t)nitems * nrec * R * 32;
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_lw, sizeof(int) * nitems));
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_st, sizeof(double2) * nst_el));
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_stsc, sizeof(int) * nst_el));
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_counter, 4 * sizeof(unsigned)));
        bytes += sizeof(int) * nitems + (sizeof(double2) + sizeof(int)) * nst_el + 4 * sizeof(unsigned);
        if ((rc = launch_start_states(*p, 0))) return rc;
        JHTB_CUDA_TRY(cudaDeviceSynchronize());
        p->h_lw.resize(nitems);
        JHTB_CUDA_TRY(cudaMemcpy(p->h_lw.data(), p->d_lw, sizeof(int) * nitems, cudaMemcpyDeviceToHost));
    }
    {
        // adjoint tiles of 32 kRA rings (the synthesis tables when the widths agree)
        const int R = spin ? kR2 : kR0, RA = spin ? kRA2 : kRA0;
        const int nrec = spin ? 2 : 1;
        p->a_ntiles = (T + 32 * RA - 1) / (32 * RA);
        p->nsuper = std::min(4, p->a_ntiles);
        p->tps = (p->a_ntiles + p->nsuper - 1) / p->nsuper;
        if (RA == R) {
            p->a_owns_tables = false;
            p->d_a_lw = p->d_lw;
            p->d_a_st = p->d_st;
            p->d_a_stsc = p->d_stsc;
            p->h_a_lw = p->h_lw;
        } else {
            const long long nitems = (long long)M * p->a_ntiles;
            const size_t nel = (size_t)nitems * nrec * RA * 32;
            p->a_owns_tables = true;
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_a_lw, sizeof(int) * nitems));
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_a_st, sizeof(double2) * nel));
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_a_stsc, sizeof(int) * nel));
            bytes += sizeof(int) * nitems + (sizeof(double2) + sizeof(int)) * nel;
            if ((rc = launch_start_states_r(*p, RA, p->a_ntiles, p->d_a_lw, p->d_a_st, p->d_a_stsc, 0))) return rc;
            JHTB_CUDA_TRY(cudaDeviceSynchronize());
            p->h_a_lw.resize(nitems);
            JHTB_CUDA_TRY(cudaMemcpy(p->h_a_lw.data(), p->d_a_lw, sizeof(int) * nitems, cudaMemcpyDeviceToHost));
        }
    }

    // ---- tensor-core path: 128-ring tiles ---------------------------------------------------
    JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_err, sizeof(int)));
    JHTB_CUDA_TRY(cudaMemset(p->d_err, 0, sizeof(int)));
    if (p->precision == JHTB_PREC_BF16X3) {
        // tensor-core tiles: 128 rings x both recursions (spin 2) or 256 rings (spin 0),
        // so each producer thread of the batched kernel runs two recursion chains
        const int Rt = spin ? 4 : 8;
        const int nrec = spin ? 2 : 1;
        p->tc_ntiles = (T + 32 * Rt - 1) / (32 * Rt);
        if (Rt == (spin ? kRA2 : kRA0)) {
            p->tc_owns_tables = false;
            p->d_tc_lw = p->d_a_lw;
            p->d_tc_st = p->d_a_st;
            p->d_tc_stsc = p->d_a_stsc;
            p->h_tc_lw = p->h_a_lw;
        } else {
            const long long nitems = (long long)M * p->tc_ntiles;
            const size_t nel = (size_t)nitems * nrec * Rt * 32;
            p->tc_owns_tables = true;
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tc_lw, sizeof(int) * nitems));
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tc_st, sizeof(double2) * nel));
            JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tc_stsc, sizeof(int) * nel));
            bytes += sizeof(int) * nitems + (sizeof(double2) + sizeof(int)) * nel;
            if ((rc = launch_start_states_r(*p, Rt, p->tc_ntiles, p->d_tc_lw, p->d_tc_st, p->d_tc_stsc, 0))) return rc;
            JHTB_CUDA_TRY(cudaDeviceSynchronize());
            p->h_tc_lw.resize(nitems);
            JHTB_CUDA_TRY(cudaMemcpy(p->h_tc_lw.data(), p->d_tc_lw, sizeof(int) * nitems, cudaMemcpyDeviceToHost));
        }
    }
    if (p->precision == JHTB_PREC_BF16X3) {
        // tensor-core adjoint: recursion state at every 32-degree segment start of every
        // 128-degree block, for the block's live ring chunks
        std::vector<int> off(M);
        long long nblk = 0;
        for (int m = 0; m < M; ++m) {
            off[m] = (int)nblk;
            nblk += (L - seeds[m].lmin + 1 + kTcaLB - 1) / kTcaLB;
        }
        p->tca_nblk = nblk;
        p->h_tca_blk_off = off;
        if ((rc = upload(&p->d_tca_blk_off, off, bytes))) return rc;
        // the block's first live ring chunk: the first chunk of the first ring tile of the
        // FP64 adjoint whose first live degree lies below the block's end (tiles nearer the
        // equator start no later); segment states are kept from that chunk to the equator
        p->tca_nchunk = (T + (spin ? 16 : 32) - 1) / (spin ? 16 : 32);
        {
            const int CR = spin ? 16 : 32, nt = p->a_ntiles, tw = 32 * (spin ? kRA2 : kRA0);
            std::vector<int> cl(nblk);
            std::vector<long long> soff(nblk);
            long long rows = 0;
            for (int m = 0; m < M; ++m) {
                const int lmin = seeds[m].lmin;
                const int nb = (L - lmin + 1 + kTcaLB - 1) / kTcaLB;
                for (int lb = 0; lb < nb; ++lb) {
                    const int l0 = lmin + lb * kTcaLB;
                    int first = nt;
                    for (int tile = 0; tile < nt; ++tile)
                        if (p->h_a_lw[(long long)m * nt + tile] < l0 + kTcaLB) {
                            first = tile;
                            break;
                        }
                    const long long b = off[m] + lb;
                    cl[b] = std::min(p->tca_nchunk, (int)((long long)first * tw / CR));
                    soff[b] = rows;
                    rows += (long long)(p->tca_nchunk - cl[b]) * kTcaSeg * 32;
                }
            }
            p->tca_nstate = rows;
            p->h_tca_blk_cl = cl;
            p->h_tca_blk_soff = soff;
            if ((rc = upload(&p->d_tca_blk_cl, cl, bytes))) return rc;
            if ((rc = upload(&p->d_tca_blk_soff, soff, bytes))) return rc;
        }
        const size_t nel = (size_t)std::max(1LL, p->tca_nstate);
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tca_st, sizeof(double2) * nel));
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tca_sc, sizeof(short) * nel));
        bytes += (sizeof(double2) + sizeof(short)) * nel;
        {
            std::vector<double2> ag(K);
            for (long long i = 0; i < K; ++i) ag[i] = make_double2(alpha[i], spin ? gamma[i] : 0.0);
            if ((rc = upload(&p->d_ag, ag, bytes))) return rc;
        }
        if ((rc = launch_tca_block_states(*p, 0))) return rc;
        JHTB_CUDA_TRY(cudaDeviceSynchronize());
        // tensor-core synthesis: prepared coefficient chunks of 16 degrees per order
        std::vector<int> cbase(M), chunk_m;
        for (int m = 0; m < M; ++m) {
            cbase[m] = (int)chunk_m.size();
            const int nck = (L - seeds[m].lmin + 1 + 15) / 16;
            for (int c = 0; c < nck; ++c) chunk_m.push_back(m);
        }
        p->tcs_nchunks = (long long)chunk_m.size();
        if ((rc = upload(&p->d_tcs_cbase, cbase, bytes))) return rc;
        if ((rc = upload(&p->d_tcs_chunk_m, chunk_m, bytes))) return rc;
        const size_t cb = (size_t)p->tcs_nchunks * tc_synth_chunk_bytes(spin);
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tcs_B, cb));
        bytes += cb;
        const size_t bt = (size_t)M * p->tca_nchunk * kTcaBStage;
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_tca_B, bt));
        bytes += bt;
    }
    p->ring_t0 = 0;
    p->ring_t1 = T;
    if ((rc = build_orders(p))) return rc;

    // ---- ring FFT descriptors (HEALPix plans; a ring-set plan stops at the ring spectra) ----
    std::vector<RingDesc> rings(p->rings_only ? 0 : nr);
    std::map<long long, long long> bh_offset;  // Bluestein length -> offset
    std::vector<int> blens;
    std::vector<long long> boffs;
    long long bh_len = 0;
    if (!p->rings_only) {
        for (int r = 0; r < nr; ++r) {
            RingDesc &d = rings[r];
            d.N = (int)npr[r];
            d.start = start[r];
            d.phi0 = phi0[r];
            if (is_pow2(d.N) && d.N <= 8 * kFftPiece) {
                d.mode = kDirect;
                d.P = d.N;
                d.Q = std::max(1, d.N / kFftPiece);
                d.bh_off = 0;
            } else if (d.N % 4 == 0 && 2LL * d.N - 1 > kFftPiece && 2LL * (d.N / 4) - 1 <= kFftPiece) {
                // too long for one shared-memory chirp-z: four of length N / 4 (polar cap rings)
                const int qn = d.N / 4;
                d.mode = kSplit4;
                d.P = (int)next_pow2(2LL * qn - 1);
                d.Q = 1;
                auto it = bh_offset.find(qn);
                if (it == bh_offset.end()) {
                    bh_offset[qn] = bh_len;
                    blens.push_back(qn);
                    boffs.push_back(bh_len);
                    d.bh_off = bh_len;
                    bh_len += d.P;
                } else {
                    d.bh_off = it->second;
                }
            } else {
                d.mode = kBluestein;
                d.P = (int)next_pow2(2LL * d.N - 1);
                d.Q = std::max(1, d.P / kFftPiece);
                if (d.Q > 8) return fail(JHTB_ERR_UNSUPPORTED, "ring length too large (nside > 4096)");
                auto it = bh_offset.find(d.N);
                if (it == bh_offset.end()) {
                    bh_offset[d.N] = bh_len;
                    blens.push_back(d.N);
                    boffs.push_back(bh_len);
                    d.bh_off = bh_len;
                    bh_len += d.P;
                } else {
                    d.bh_off = it->second;
                }
            }
        }
        if ((rc = upload(&p->d_rings, rings, bytes))) return rc;
        p->h_ring_pieces.assign(nr, 1);
        for (int r = 0; r < nr; ++r) p->h_ring_pieces[r] = (unsigned char)ring_pieces(rings[r]);
        if ((rc = build_ring_lists(p, bytes))) return rc;

        std::vector<double2> tw(kTwLen);
        for (int k = 0; k < kTwLen; ++k) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)kTwLen;
            tw[k] = make_double2((double)cosl(a), (double)sinl(a));
        }
        if ((rc = upload(&p->d_tw, tw, bytes))) return rc;

        p->bh_len = bh_len;
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_bh, sizeof(double2) * std::max(bh_len, 1LL)));
        bytes += sizeof(double2) * std::max(bh_len, 1LL);
    }

    // ---- workspace --------------------------------------------------------------------------
    const size_t f_per_map = sizeof(double2) * (size_t)p->ncomp * nr * M;
    p->chunk = std::max(1, p->max_batch);
    JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_F, f_per_map * p->chunk));
    bytes += f_per_map * p->chunk;
    if (p->precision == JHTB_PREC_FP64) {  // partial rows of the FP64 adjoint (the tensor-core one needs none)
        const size_t part = sizeof(double2) * (size_t)p->nsuper * p->ncomp * p->K * p->chunk;
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_part, part));
        bytes += part;
    }
    bool need_w = false;
    for (int r = 0; r < (int)rings.size(); ++r) need_w |= p->h_ring_pieces[r] == 1 && rings[r].Q > 1;
    if (need_w) {
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_W, sizeof(double2) * (size_t)p->npix * p->chunk));
        JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_W2, sizeof(double2) * (size_t)p->npix * p->chunk));
        bytes += 2 * sizeof(double2) * (size_t)p->npix * p->chunk;
    }
    JHTB_CUDA_TRY(cudaMalloc((void **)&p->d_scratch, 4096 * sizeof(double)));
    bytes += 4096 * sizeof(double);

    // ---- Bluestein chirp spectra (device) -------------------------------------------------------
    if (!blens.empty()) {
        int *d_len = nullptr;
        long long *d_off = nullptr;
        JHTB_CUDA_TRY(cudaMalloc((void **)&d_len, sizeof(int) * blens.size()));
        JHTB_CUDA_TRY(cudaMalloc((void **)&d_off, sizeof(long long) * boffs.size()));
        JHTB_CUDA_TRY(cudaMemcpy(d_len, blens.data(), sizeof(int) * blens.size(), cudaMemcpyHostToDevice));
        JHTB_CUDA_TRY(cudaMemcpy(d_off, boffs.data(), sizeof(long long) * boffs.size(), cudaMemcpyHostToDevice));
        rc = launch_bluestein_setup(*p, d_len, d_off, (int)blens.size(), 0);
        cudaError_t e = cudaDeviceSynchronize();
        cudaFree(d_len);
        cudaFree(d_off);
        if (rc) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "bluestein setup");
    }
    return JHTB_OK;
}

}  // namespace

// One stage launch: an NVTX range named after the stage (seen by Nsight Systems /
// Nsight Compute range filters; a no-op without a tool attached), and, when the
// plan's timing is on, a CUDA event pair around the launch.
static const char *const kStageNames[kNumStages] = {"jhtb:legendre_synth", "jhtb:ring_synth", "jhtb:ring_adjoint",
                                                    "jhtb:legendre_adjoint"};

struct StageTimer {
    Plan &p;
    cudaStream_t s;
    Plan::StageEvent ev{};
    bool on;
    StageTimer(Plan &plan, cudaStream_t stream, int stage) : p(plan), s(stream), on(plan.timing) {
        nvtxRangePushA(kStageNames[stage]);
        if (!on) return;
        ev.stage = stage;
        if (cudaEventCreate(&ev.start) != cudaSuccess || cudaEventCreate(&ev.stop) != cudaSuccess) {
            on = false;
            return;
        }
        cudaEventRecord(ev.start, s);
    }
    ~StageTimer() {
        if (on) {
            cudaEventRecord(ev.stop, s);
            p.events.push_back(ev);
        }
        nvtxRangePop();
    }
};

}  // namespace jhtb

using namespace jhtb;

extern "C" {

int jhtb_version(void) { return 100; }

int jhtb_last_error(char *buf, size_t len) {
    if (!buf || len == 0) return JHTB_ERR_INVALID;
    std::snprintf(buf, len, "%s", g_last_error.c_str());
    return JHTB_OK;
}

int jhtb_plan_create(int nside, int lmax, int spin, int precision, int max_batch,
                     const jhtb_host_tables *tables, jhtb_plan **out) {
    if (!out) return fail(JHTB_ERR_INVALID, "jhtb_plan_create: out is NULL");
    *out = nullptr;
    if (spin != 0 && spin != 2)
        return fail(JHTB_ERR_UNSUPPORTED, "spin=" + std::to_string(spin) + " unsupported (only 0 and 2)");
    if (nside < 1 || nside > 4096)
        return fail(JHTB_ERR_INVALID, "nside must be in [1, 4096], got " + std::to_string(nside));
    if (lmax < 0 || lmax > 16383) return fail(JHTB_ERR_INVALID, "lmax must be in [0, 16383]");
    if (precision == JHTB_PREC_FP32)
        return fail(JHTB_ERR_UNSUPPORTED, "FP32 contraction is not implemented (use JHTB_PREC_FP64 or JHTB_PREC_BF16X3)");
    if (precision != JHTB_PREC_FP64 && precision != JHTB_PREC_BF16X3)
        return fail(JHTB_ERR_INVALID, "unknown precision " + std::to_string(precision));
    if (max_batch < 1) return fail(JHTB_ERR_INVALID, "max_batch must be >= 1");
    Plan *p = new (std::nothrow) Plan();  // value-initialised: pointers null, counters zero
    if (!p) return fail(JHTB_ERR_NOMEM, "host allocation failed");
    p->nside = nside;
    p->lmax = lmax;
    p->spin = spin;
    p->precision = precision;
    p->max_batch = max_batch;
    p->T = 2 * nside;
    p->nrings = 4 * nside - 1;
    p->M = lmax + 1;
    p->K = (long long)(lmax + 1) * (lmax + 2) / 2;
    p->npix = 12LL * nside * nside;
    p->ncomp = spin ? 2 : 1;
    p->npairs = lmax / 2 + 1;
    int rc = build_plan(p, tables);
    if (rc) {
        free_plan(p);
        return rc;
    }
    *out = reinterpret_cast<jhtb_plan *>(p);
    return JHTB_OK;
}

int jhtb_plan_create_rings(int nrings, int lmax, int spin, int precision, int max_batch,
                           const jhtb_host_tables *tables, jhtb_plan **out) {
    if (!out) return fail(JHTB_ERR_INVALID, "jhtb_plan_create_rings: out is NULL");
    *out = nullptr;
    if (spin != 0 && spin != 2)
        return fail(JHTB_ERR_UNSUPPORTED, "spin=" + std::to_string(spin) + " unsupported (only 0 and 2)");
    if (nrings < 1 || nrings > 65535 || nrings % 2 == 0)
        return fail(JHTB_ERR_INVALID, "nrings must be odd and in [1, 65535], got " + std::to_string(nrings));
    if (lmax < 0 || lmax > 16383) return fail(JHTB_ERR_INVALID, "lmax must be in [0, 16383]");
    if (precision == JHTB_PREC_FP32)
        return fail(JHTB_ERR_UNSUPPORTED, "FP32 contraction is not implemented (use JHTB_PREC_FP64 or JHTB_PREC_BF16X3)");
    if (precision != JHTB_PREC_FP64 && precision != JHTB_PREC_BF16X3)
        return fail(JHTB_ERR_INVALID, "unknown precision " + std::to_string(precision));
    if (max_batch < 1) return fail(JHTB_ERR_INVALID, "max_batch must be >= 1");
    if (!tables || !tables->x)
        return fail(JHTB_ERR_INVALID, "jhtb_plan_create_rings: tables->x (the northern rings' cos theta) is required");
    const int T = (nrings + 1) / 2;
    for (int t = 0; t < T; ++t) {
        const double x = tables->x[t];
        if (!(x >= 0.0 && x <= 1.0) || (t > 0 && x > tables->x[t - 1]))
            return fail(JHTB_ERR_INVALID, "jhtb_plan_create_rings: x must be non-increasing in [0, 1]");
    }
    Plan *p = new (std::nothrow) Plan();
    if (!p) return fail(JHTB_ERR_NOMEM, "host allocation failed");
    p->rings_only = true;
    p->nside = 0;
    p->lmax = lmax;
    p->spin = spin;
    p->precision = precision;
    p->max_batch = max_batch;
    p->T = T;
    p->nrings = nrings;
    p->M = lmax + 1;
    p->K = (long long)(lmax + 1) * (lmax + 2) / 2;
    p->npix = 0;
    p->ncomp = spin ? 2 : 1;
    p->npairs = lmax / 2 + 1;
    int rc = build_plan(p, tables);
    if (rc) {
        free_plan(p);
        return rc;
    }
    *out = reinterpret_cast<jhtb_plan *>(p);
    return JHTB_OK;
}

int jhtb_legendre_synthesis(jhtb_plan *plan, const void *alm, void *rings, int batch, void *stream) {
    if (!plan || !alm || !rings) return fail(JHTB_ERR_INVALID, "jhtb_legendre_synthesis: NULL argument");
    if (batch < 0) return fail(JHTB_ERR_INVALID, "jhtb_legendre_synthesis: negative batch");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    cudaStream_t s = (cudaStream_t)stream;
    const double2 *a = (const double2 *)alm;
    double2 *F = (double2 *)rings;
    const size_t f_map = (size_t)p.ncomp * p.nrings * p.M;
    for (int b0 = 0; b0 < batch; b0 += p.chunk) {
        const int nb = std::min(p.chunk, batch - b0);
        StageTimer t(p, s, kStageLegSynth);
        const int rc = p.precision == JHTB_PREC_BF16X3
                           ? launch_tc_synth(p, a + (size_t)b0 * p.ncomp * p.K, F + (size_t)b0 * f_map, nb, s)
                           : launch_legendre_synth(p, a + (size_t)b0 * p.ncomp * p.K, F + (size_t)b0 * f_map, nb, s);
        if (rc) return rc;
    }
    return JHTB_OK;
}

int jhtb_legendre_adjoint(jhtb_plan *plan, const void *rings, void *alm, int batch, void *stream) {
    if (!plan || !alm || !rings) return fail(JHTB_ERR_INVALID, "jhtb_legendre_adjoint: NULL argument");
    if (batch < 0) return fail(JHTB_ERR_INVALID, "jhtb_legendre_adjoint: negative batch");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    cudaStream_t s = (cudaStream_t)stream;
    const double2 *F = (const double2 *)rings;
    double2 *a = (double2 *)alm;
    const size_t f_map = (size_t)p.ncomp * p.nrings * p.M;
    for (int b0 = 0; b0 < batch; b0 += p.chunk) {
        const int nb = std::min(p.chunk, batch - b0);
        StageTimer t(p, s, kStageLegAdj);
        const int rc = p.precision == JHTB_PREC_BF16X3
                           ? launch_tc_adjoint(p, F + (size_t)b0 * f_map, a + (size_t)b0 * p.ncomp * p.K, nb, s)
                           : launch_legendre_adjoint(p, F + (size_t)b0 * f_map, a + (size_t)b0 * p.ncomp * p.K, nb, s);
        if (rc) return rc;
    }
    return JHTB_OK;
}

int jhtb_plan_destroy(jhtb_plan *plan) {
    free_plan(reinterpret_cast<Plan *>(plan));
    return JHTB_OK;
}

int jhtb_plan_bytes(const jhtb_plan *plan, int64_t *bytes) {
    if (!plan || !bytes) return fail(JHTB_ERR_INVALID, "jhtb_plan_bytes: NULL argument");
    *bytes = (int64_t) reinterpret_cast<const Plan *>(plan)->bytes;
    return JHTB_OK;
}

int jhtb_synthesis(jhtb_plan *plan, const void *alm, void *maps, int batch, void *stream) {
    if (!plan || !alm || !maps) return fail(JHTB_ERR_INVALID, "jhtb_synthesis: NULL argument");
    if (batch < 0) return fail(JHTB_ERR_INVALID, "jhtb_synthesis: negative batch");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    if (p.rings_only)
        return fail(JHTB_ERR_INVALID, "jhtb_synthesis: a ring-set plan has no pixel grid (use the jhtb_legendre_* calls)");
    cudaStream_t s = (cudaStream_t)stream;
    const double2 *a = (const double2 *)alm;
    double *m = (double *)maps;
    for (int b0 = 0; b0 < batch; b0 += p.chunk) {
        int nb = std::min(p.chunk, batch - b0);
        int rc;
        {
            StageTimer t(p, s, kStageLegSynth);
            rc = p.precision == JHTB_PREC_BF16X3 ? launch_tc_synth(p, a + (size_t)b0 * p.ncomp * p.K, p.d_F, nb, s)
                                                 : launch_legendre_synth(p, a + (size_t)b0 * p.ncomp * p.K, p.d_F, nb, s);
        }
        if (rc) return rc;
        {
            StageTimer t(p, s, kStageRingSynth);
            rc = launch_ring_synth(p, p.d_F, m + (size_t)b0 * p.ncomp * p.npix, nb, s);
        }
        if (rc) return rc;
    }
    return JHTB_OK;
}

int jhtb_adjoint_synthesis(jhtb_plan *plan, const void *maps, void *alm, int batch, void *stream) {
    if (!plan || !alm || !maps) return fail(JHTB_ERR_INVALID, "jhtb_adjoint_synthesis: NULL argument");
    if (batch < 0) return fail(JHTB_ERR_INVALID, "jhtb_adjoint_synthesis: negative batch");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    if (p.rings_only)
        return fail(JHTB_ERR_INVALID, "jhtb_adjoint_synthesis: a ring-set plan has no pixel grid (use the jhtb_legendre_* calls)");
    cudaStream_t s = (cudaStream_t)stream;
    const double *m = (const double *)maps;
    double2 *a = (double2 *)alm;
    for (int b0 = 0; b0 < batch; b0 += p.chunk) {
        int nb = std::min(p.chunk, batch - b0);
        int rc;
        {
            StageTimer t(p, s, kStageRingAdj);
            rc = launch_ring_adjoint(p, m + (size_t)b0 * p.ncomp * p.npix, p.d_F, p.d_W, nb, s);
        }
        if (rc) return rc;
        {
            StageTimer t(p, s, kStageLegAdj);
            rc = p.precision == JHTB_PREC_BF16X3 ? launch_tc_adjoint(p, p.d_F, a + (size_t)b0 * p.ncomp * p.K, nb, s)
                                                 : launch_legendre_adjoint(p, p.d_F, a + (size_t)b0 * p.ncomp * p.K, nb, s);
        }
        if (rc) return rc;
    }
    return JHTB_OK;
}

int jhtb_plan_status(jhtb_plan *plan, int *device_error) {
    if (!plan || !device_error) return fail(JHTB_ERR_INVALID, "jhtb_plan_status: NULL argument");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    JHTB_CUDA_TRY(cudaDeviceSynchronize());
    JHTB_CUDA_TRY(cudaMemcpy(device_error, p.d_err, sizeof(int), cudaMemcpyDeviceToHost));
    JHTB_CUDA_TRY(cudaMemset(p.d_err, 0, sizeof(int)));
    return JHTB_OK;
}

int jhtb_plan_set_watchdog(jhtb_plan *plan, int64_t timeout_ns) {
    if (!plan) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_watchdog: NULL plan");
    if (timeout_ns < 1000000 || timeout_ns > 60000000000LL)
        return fail(JHTB_ERR_INVALID, "jhtb_plan_set_watchdog: timeout_ns must be in [1e6, 6e10]");
    reinterpret_cast<Plan *>(plan)->tc_wait_ns = (unsigned long long)timeout_ns;
    return JHTB_OK;
}

int jhtb_plan_set_tuning(jhtb_plan *plan, int key, int value) {
    if (!plan) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: NULL plan");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    switch (key) {
        case JHTB_TUNE_TC_FOLD:
            if (value < 16 || value > 4096 || value % 16)
                return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: TC_FOLD must be a multiple of 16 in [16, 4096]");
            p.tc_fold = value;
            return JHTB_OK;
        case JHTB_TUNE_TCA_FOLD:
            if (value < 32 || value > 8192 || value % 32)
                return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: TCA_FOLD must be a multiple of 32 in [32, 8192]");
            p.tca_fold = value;
            return JHTB_OK;
        case JHTB_TUNE_TC_GROUP:
            if (value != 8 && value != 16) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: TC_GROUP must be 8 or 16");
            p.tc_group = value;
            return JHTB_OK;
        case JHTB_TUNE_LEG_CTAS:
            if (value < 0 || value > 16) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: LEG_CTAS must be in [0, 16]");
            p.leg_ctas = value;
            return JHTB_OK;
        default:
            return fail(JHTB_ERR_INVALID, "jhtb_plan_set_tuning: unknown key " + std::to_string(key));
    }
}

int jhtb_plan_inject_fault(jhtb_plan *plan, int kind) {
    if (!plan) return fail(JHTB_ERR_INVALID, "jhtb_plan_inject_fault: NULL plan");
    if (kind != 0 && kind != JHTB_FAULT_STALL)
        return fail(JHTB_ERR_INVALID, "jhtb_plan_inject_fault: kind must be 0 or JHTB_FAULT_STALL");
    reinterpret_cast<Plan *>(plan)->inject = kind;
    return JHTB_OK;
}

int jhtb_debug_bounds(int64_t *count, int *site, int64_t *index, int64_t *extent) {
    if (!count || !site || !index || !extent) return fail(JHTB_ERR_INVALID, "jhtb_debug_bounds: NULL argument");
    *count = 0;
    *site = 0;
    *index = *extent = 0;
#ifdef JHTB_DEBUG
    JHTB_CUDA_TRY(cudaDeviceSynchronize());
    int (*const readers[])(DebugRecord *, bool) = {debug_record_legendre, debug_record_ringfft, debug_record_tc_synth,
                                                   debug_record_tc_adjoint, debug_record_vecops};
    for (auto rd : readers) {
        DebugRecord r{};
        if (rd(&r, true)) return fail(JHTB_ERR_CUDA, "jhtb_debug_bounds: reading a bounds record failed");
        if (r.count && !*count) {
            *site = r.site;
            *index = r.index;
            *extent = r.extent;
        }
        *count += (int64_t)r.count;
    }
    return JHTB_OK;
#else
    return fail(JHTB_ERR_UNSUPPORTED, "jhtb_debug_bounds: bounds checks are compiled into the debug library only (make debug)");
#endif
}

int jhtb_plan_ring_costs(const jhtb_plan *plan, int granule, int64_t *cost, int ncost) {
    if (!plan || !cost) return fail(JHTB_ERR_INVALID, "jhtb_plan_ring_costs: NULL argument");
    const Plan &p = *reinterpret_cast<const Plan *>(plan);
    if (p.rings_only) return fail(JHTB_ERR_INVALID, "jhtb_plan_ring_costs: HEALPix plans only");
    if (granule <= 0 || granule % kRingGranule)
        return fail(JHTB_ERR_INVALID, "jhtb_plan_ring_costs: granule must be a positive multiple of " +
                                          std::to_string(kRingGranule));
    const int ng = (p.T + granule - 1) / granule;
    if (ncost < ng) return fail(JHTB_ERR_INVALID, "jhtb_plan_ring_costs: need " + std::to_string(ng) + " entries");
    for (int g = 0; g < ng; ++g) cost[g] = 0;
    const int tw = 32 * (p.spin ? kR2 : kR0);
    for (long long i = 0; i < (long long)p.M * p.ntiles; ++i) {
        const int tile = (int)(i % p.ntiles);
        const int t_lo = tile * tw, t_hi = std::min(p.T, t_lo + tw);
        cost[t_lo / granule] += (int64_t)std::max(0, p.lmax + 1 - p.h_lw[i]) * (t_hi - t_lo);
    }
    return JHTB_OK;
}

int jhtb_plan_set_ring_range(jhtb_plan *plan, int t0, int t1) {
    if (!plan) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_ring_range: NULL plan");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    if (p.rings_only) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_ring_range: HEALPix plans only");
    if (t0 < 0 || t1 > p.T || t0 >= t1 || t0 % kRingGranule || (t1 % kRingGranule && t1 != p.T))
        return fail(JHTB_ERR_INVALID, "jhtb_plan_set_ring_range: need 0 <= t0 < t1 <= 2 nside = " +
                                          std::to_string(p.T) + " with t0 and t1 (unless 2 nside) multiples of " +
                                          std::to_string(kRingGranule));
    JHTB_CUDA_TRY(cudaDeviceSynchronize());  // no launch of this plan may still read the old orders
    p.ring_t0 = t0;
    p.ring_t1 = t1;
    return build_orders(&p);
}

int jhtb_plan_set_timing(jhtb_plan *plan, int enable) {
    if (!plan) return fail(JHTB_ERR_INVALID, "jhtb_plan_set_timing: NULL plan");
    reinterpret_cast<Plan *>(plan)->timing = enable != 0;
    return JHTB_OK;
}

int jhtb_plan_timings(jhtb_plan *plan, double *ms, int64_t *counts, int reset) {
    if (!plan || !ms || !counts) return fail(JHTB_ERR_INVALID, "jhtb_plan_timings: NULL argument");
    Plan &p = *reinterpret_cast<Plan *>(plan);
    for (int i = 0; i < kNumStages; ++i) {
        ms[i] = 0.0;
        counts[i] = 0;
    }
    for (auto &e : p.events) {
        JHTB_CUDA_TRY(cudaEventSynchronize(e.stop));
        float t = 0.f;
        JHTB_CUDA_TRY(cudaEventElapsedTime(&t, e.start, e.stop));
        ms[e.stage] += t;
        counts[e.stage] += 1;
    }
    if (reset) {
        for (auto &e : p.events) {
            cudaEventDestroy(e.start);
            cudaEventDestroy(e.stop);
        }
        p.events.clear();
    }
    return JHTB_OK;
}

}  // extern "C"
