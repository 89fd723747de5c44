/*
 * CPU oracle, C part: the Legendre / Wigner-d recursion + l-contraction of
 * jht's on-grid transform in FP64, parallel over m with OpenMP.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle checks the CUDA path and times the CPU
 * baseline; the product never links it).  It is the same algorithm as the
 * NumPy oracle (jht_oracle.py) and as the reference:
 *   - coefficients: _recursion.py:37-50 (spin 0), :136-143 (Wigner, spin +-2)
 *   - seeds:        _recursion.py:53-56 (sectoral), :166-188 (Wigner single term)
 *   - one step:     _recursion.py:352-369, the per-step log-renormalisation
 *                   raw = (A x + C) p - B q; r = |(raw, p)|; p,q,s <- raw/r, p/r, s+log r
 *   - contraction:  _recursion.py:441-497 (spin 0 N/S parity), :512-572 (spin 2)
 * Outputs are (M, T) half-grid arrays, row m = order, column t = ring.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

/* flat index of a_{m,m} (healpix.py:53-55) */
static long alm_base(long m, long lmax) { return m * (2 * lmax + 1 - m) / 2 + m; }

/* Per-m coefficient columns for l = 0..lmax (zero where l <= lmin). */
static void coeffs(int spin, int m, int lmax, double *A, double *B, double *C, double *pref) {
    int lmin = m > abs(spin) ? m : abs(spin);
    for (int l = 0; l <= lmax; ++l) { A[l] = B[l] = C[l] = 0.0; }
    if (spin == 0) {
        for (int l = m + 1; l <= lmax; ++l) {
            double L = l;
            A[l] = sqrt((2 * L - 1) * (2 * L + 1) / ((L - m) * (L + m)));
            B[l] = sqrt((2 * L + 1) * ((L - 1) * (L - 1) - (double)m * m) /
                        ((2 * L - 3) * (L - m) * (L + m)));
        }
        for (int l = 0; l <= lmax; ++l) pref[l] = 1.0;
    } else {
        double M = -m, Mp = spin;
        for (int l = lmin + 1; l <= lmax; ++l) {
            double L = l - 1; /* coefficients at l-1 produce d^l */
            double D = L * sqrt(((L + 1) * (L + 1) - M * M) * ((L + 1) * (L + 1) - Mp * Mp));
            A[l] = (2 * L + 1) * L * (L + 1) / D;
            C[l] = -(2 * L + 1) * M * Mp / D;
            B[l] = (L + 1) * sqrt((L * L - M * M) * (L * L - Mp * Mp)) / D;
        }
        double sg = (m % 2) ? -1.0 : 1.0;
        for (int l = 0; l <= lmax; ++l) pref[l] = sg * sqrt((2.0 * l + 1.0) / (4.0 * M_PI));
    }
}

/* Seed (sign, log|value|) at l = lmin for every ring. */
static void seed(int spin, int m, int T, const double *x, double *sign, double *slog) {
    if (spin == 0) {
        double c = -0.5 * log(4.0 * M_PI);
        for (int k = 1; k <= m; ++k) c += 0.5 * log((2.0 * k + 1.0) / (2.0 * k));
        *sign = (m % 2) ? -1.0 : 1.0;
        for (int t = 0; t < T; ++t) {
            double s2 = 1.0 - x[t] * x[t];
            s2 = s2 < 0 ? 0 : (s2 > 1 ? 1 : s2);
            slog[t] = (m == 0) ? c : c + m * log(sqrt(s2));
        }
        return;
    }
    int M = -m, Mp = spin;
    int lmin = m > abs(spin) ? m : abs(spin);
    int k0 = M - Mp > 0 ? M - Mp : 0;
    double lf = 0.5 * (lgamma(lmin + M + 1.0) + lgamma(lmin - M + 1.0) + lgamma(lmin + Mp + 1.0) +
                       lgamma(lmin - Mp + 1.0)) -
                (lgamma(k0 + 1.0) + lgamma(lmin + M - k0 + 1.0) + lgamma(lmin - Mp - k0 + 1.0) +
                 lgamma(k0 - M + Mp + 1.0));
    *sign = (k0 % 2) ? -1.0 : 1.0;
    int pc = 2 * lmin - 2 * k0 + M - Mp, ps = 2 * k0 - M + Mp;
    for (int t = 0; t < T; ++t) {
        double ch = (1.0 + x[t]) / 2.0, sh = (1.0 - x[t]) / 2.0;
        ch = sqrt(ch < 0 ? 0 : (ch > 1 ? 1 : ch));
        sh = sqrt(sh < 0 ? 0 : (sh > 1 ? 1 : sh));
        double v = lf;
        if (pc > 0) v += pc * log(ch);
        if (ps > 0) v += ps * log(sh);
        slog[t] = v;
    }
}

/* One recursion state: mantissa p, previous q, log-scale s (per ring). */
typedef struct { double *p, *q, *s; } state_t;

static inline double step(double A, double B, double C, double x, double *p, double *q, double *s) {
    double raw = (A * x + C) * (*p) - B * (*q);
    double r = sqrt(raw * raw + (*p) * (*p));
    if (r == 0.0) r = 1.0;
    double np_ = raw / r, nq = (*p) / r;
    *s = *s + log(r);
    *p = np_;
    *q = nq;
    return np_ * exp(*s);
}

/* Advance to degree l and return lambda_l(t) (no pref) for all rings. */
static void advance(int l, int lmin, const double *A, const double *B, const double *C, int T,
                    const double *x, double sg, const double *slog, state_t st, double *lam) {
    if (l < lmin) {
        for (int t = 0; t < T; ++t) lam[t] = 0.0;
    } else if (l == lmin) {
        for (int t = 0; t < T; ++t) {
            st.p[t] = sg; st.q[t] = 0.0; st.s[t] = slog[t];
            lam[t] = sg * exp(slog[t]);
        }
    } else {
        for (int t = 0; t < T; ++t) lam[t] = step(A[l], B[l], C[l], x[t], &st.p[t], &st.q[t], &st.s[t]);
    }
}

/*
 * Spin-0 synthesis contraction for m in [m_lo, m_hi):
 *   Ft[m,t] = sum_l a_lm lambda_lm(t),  Fs[m,t] = sum_l (-1)^l a_lm lambda_lm(t).
 * Spin-2 (E,B in alm[0..K), alm[K..2K)): FpN, FpS, FmN, FmS as _recursion.py:512-543.
 * out holds nout = (spin==0 ? 2 : 4) arrays of shape (lmax+1, T).
 */
void oracle_synth(int spin, int lmax, int T, const double *x, const cplx *alm, cplx *out, int m_lo,
                  int m_hi) {
    long K = (long)(lmax + 1) * (lmax + 2) / 2;
    long MT = (long)(lmax + 1) * T;
#pragma omp parallel
    {
        int L1 = lmax + 1;
        double *A = malloc(sizeof(double) * L1 * 8), *B = A + L1, *C = B + L1, *pref = C + L1;
        double *A2 = pref + L1, *B2 = A2 + L1, *C2 = B2 + L1, *pref2 = C2 + L1;
        double *buf = malloc(sizeof(double) * T * 10);
        state_t s1 = {buf, buf + T, buf + 2 * T}, s2 = {buf + 3 * T, buf + 4 * T, buf + 5 * T};
        double *lam1 = buf + 6 * T, *lam2 = buf + 7 * T, *slog1 = buf + 8 * T, *slog2 = buf + 9 * T;
#pragma omp for schedule(dynamic, 1)
        for (int m = m_lo; m < m_hi; ++m) {
            int lmin = m > abs(spin) ? m : abs(spin);
            double sg1, sg2;
            if (spin == 0) {
                coeffs(0, m, lmax, A, B, C, pref);
                seed(0, m, T, x, &sg1, slog1);
                cplx *Ft = out + (long)m * T, *Fs = out + MT + (long)m * T;
                for (int t = 0; t < T; ++t) Ft[t] = Fs[t] = 0;
                for (int l = 0; l <= lmax; ++l) {
                    advance(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    if (l < lmin) continue;
                    cplx a = alm[alm_base(m, lmax) + l - m];
                    double par = (l % 2) ? -1.0 : 1.0;
                    for (int t = 0; t < T; ++t) {
                        cplx c = a * lam1[t];
                        Ft[t] += c;
                        Fs[t] += par * c;
                    }
                }
            } else {
                coeffs(2, m, lmax, A, B, C, pref);
                coeffs(-2, m, lmax, A2, B2, C2, pref2);
                seed(2, m, T, x, &sg1, slog1);
                seed(-2, m, T, x, &sg2, slog2);
                cplx *FpN = out + (long)m * T, *FpS = FpN + MT, *FmN = FpS + MT, *FmS = FmN + MT;
                for (int t = 0; t < T; ++t) FpN[t] = FpS[t] = FmN[t] = FmS[t] = 0;
                for (int l = 0; l <= lmax; ++l) {
                    advance(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    advance(l, lmin, A2, B2, C2, T, x, sg2, slog2, s2, lam2);
                    if (l < lmin) continue;
                    long i = alm_base(m, lmax) + l - m;
                    cplx e = alm[i], b = alm[K + i];
                    cplx cp = -(e + I * b) * pref[l], cm = -(e - I * b) * pref[l];
                    double par = (l % 2) ? -1.0 : 1.0;
                    for (int t = 0; t < T; ++t) {
                        FpN[t] += cp * lam1[t];
                        FpS[t] += par * cp * lam2[t];
                        FmN[t] += cm * lam2[t];
                        FmS[t] += par * cm * lam1[t];
                    }
                }
            }
        }
        free(buf);
        free(A);
    }
}

/*
 * Adjoint contraction for m in [m_lo, m_hi).
 * spin 0: in = [Vn, Vs] (each (M,T)); out[0..K) = b_lm = sum_t lambda (Vn + (-1)^l Vs).
 * spin 2: in = [Vpn, Sp, Vmn, Sm]; out[0..K) = p2, out[K..2K) = m2 (_recursion.py:546-572).
 */
void oracle_adjoint(int spin, int lmax, int T, const double *x, const cplx *in, cplx *out, int m_lo,
                    int m_hi) {
    long K = (long)(lmax + 1) * (lmax + 2) / 2;
    long MT = (long)(lmax + 1) * T;
#pragma omp parallel
    {
        int L1 = lmax + 1;
        double *A = malloc(sizeof(double) * L1 * 8), *B = A + L1, *C = B + L1, *pref = C + L1;
        double *A2 = pref + L1, *B2 = A2 + L1, *C2 = B2 + L1, *pref2 = C2 + L1;
        double *buf = malloc(sizeof(double) * T * 10);
        state_t s1 = {buf, buf + T, buf + 2 * T}, s2 = {buf + 3 * T, buf + 4 * T, buf + 5 * T};
        double *lam1 = buf + 6 * T, *lam2 = buf + 7 * T, *slog1 = buf + 8 * T, *slog2 = buf + 9 * T;
#pragma omp for schedule(dynamic, 1)
        for (int m = m_lo; m < m_hi; ++m) {
            int lmin = m > abs(spin) ? m : abs(spin);
            double sg1, sg2;
            long base = alm_base(m, lmax);
            if (spin == 0) {
                coeffs(0, m, lmax, A, B, C, pref);
                seed(0, m, T, x, &sg1, slog1);
                const cplx *Vn = in + (long)m * T, *Vs = in + MT + (long)m * T;
                for (int l = 0; l <= lmax; ++l) {
                    advance(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    if (l < m) continue;
                    cplx sn = 0, ss = 0;
                    for (int t = 0; t < T; ++t) { sn += lam1[t] * Vn[t]; ss += lam1[t] * Vs[t]; }
                    double par = (l % 2) ? -1.0 : 1.0;
                    out[base + l - m] = pref[l] * (sn + par * ss);
                }
            } else {
                coeffs(2, m, lmax, A, B, C, pref);
                coeffs(-2, m, lmax, A2, B2, C2, pref2);
                seed(2, m, T, x, &sg1, slog1);
                seed(-2, m, T, x, &sg2, slog2);
                const cplx *Vpn = in + (long)m * T, *Sp = Vpn + MT, *Vmn = Sp + MT, *Sm = Vmn + MT;
                for (int l = 0; l <= lmax; ++l) {
                    advance(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    advance(l, lmin, A2, B2, C2, T, x, sg2, slog2, s2, lam2);
                    if (l < m) continue;
                    cplx a1 = 0, a2 = 0, a3 = 0, a4 = 0;
                    for (int t = 0; t < T; ++t) {
                        a1 += lam1[t] * Vpn[t];
                        a2 += lam2[t] * Sp[t];
                        a3 += lam2[t] * Vmn[t];
                        a4 += lam1[t] * Sm[t];
                    }
                    double par = (l % 2) ? -1.0 : 1.0;
                    out[base + l - m] = pref[l] * (a1 + par * a2);
                    out[K + base + l - m] = pref[l] * (a3 + par * a4);
                }
            }
        }
        free(buf);
        free(A);
    }
}

/*
 * ---------------------------------------------------------------------------------
 * Extended-precision arbiter: the same algorithm (coefficients, seeds, per-step
 * log-renormalised recursion, N/S contraction) carried out in x87 80-bit long double
 * (64-bit significand, 11 bits more than FP64).  It decides which of two FP64
 * evaluations -- this oracle's and the CUDA kernels' -- carries a given difference:
 * its own rounding is ~2^-64 per operation, 2048 times below FP64's.  The ring
 * positions x are the FP64 values both FP64 evaluations use.
 * ---------------------------------------------------------------------------------
 */
typedef long double xreal;
typedef long double _Complex xcplx;
static const xreal XPI = 3.14159265358979323846264338327950288L;

static void coeffs_ld(int spin, int m, int lmax, xreal *A, xreal *B, xreal *C, xreal *pref) {
    int lmin = m > abs(spin) ? m : abs(spin);
    for (int l = 0; l <= lmax; ++l) { A[l] = B[l] = C[l] = 0.0L; }
    if (spin == 0) {
        for (int l = m + 1; l <= lmax; ++l) {
            xreal L = l;
            A[l] = sqrtl((2 * L - 1) * (2 * L + 1) / ((L - m) * (L + m)));
            B[l] = sqrtl((2 * L + 1) * ((L - 1) * (L - 1) - (xreal)m * m) / ((2 * L - 3) * (L - m) * (L + m)));
        }
        for (int l = 0; l <= lmax; ++l) pref[l] = 1.0L;
    } else {
        xreal M = -m, Mp = spin;
        for (int l = lmin + 1; l <= lmax; ++l) {
            xreal L = l - 1;
            xreal D = L * sqrtl(((L + 1) * (L + 1) - M * M) * ((L + 1) * (L + 1) - Mp * Mp));
            A[l] = (2 * L + 1) * L * (L + 1) / D;
            C[l] = -(2 * L + 1) * M * Mp / D;
            B[l] = (L + 1) * sqrtl((L * L - M * M) * (L * L - Mp * Mp)) / D;
        }
        xreal sg = (m % 2) ? -1.0L : 1.0L;
        for (int l = 0; l <= lmax; ++l) pref[l] = sg * sqrtl((2.0L * l + 1.0L) / (4.0L * XPI));
    }
}

static void seed_ld(int spin, int m, int T, const double *x, xreal *sign, xreal *slog) {
    if (spin == 0) {
        xreal c = -0.5L * logl(4.0L * XPI);
        for (int k = 1; k <= m; ++k) c += 0.5L * logl((2.0L * k + 1.0L) / (2.0L * k));
        *sign = (m % 2) ? -1.0L : 1.0L;
        for (int t = 0; t < T; ++t) {
            xreal xt = x[t];
            xreal s2 = 1.0L - xt * xt;
            s2 = s2 < 0 ? 0 : (s2 > 1 ? 1 : s2);
            slog[t] = (m == 0) ? c : c + m * logl(sqrtl(s2));
        }
        return;
    }
    int M = -m, Mp = spin;
    int lmin = m > abs(spin) ? m : abs(spin);
    int k0 = M - Mp > 0 ? M - Mp : 0;
    xreal lf = 0.5L * (lgammal(lmin + M + 1.0L) + lgammal(lmin - M + 1.0L) + lgammal(lmin + Mp + 1.0L) +
                       lgammal(lmin - Mp + 1.0L)) -
               (lgammal(k0 + 1.0L) + lgammal(lmin + M - k0 + 1.0L) + lgammal(lmin - Mp - k0 + 1.0L) +
                lgammal(k0 - M + Mp + 1.0L));
    *sign = (k0 % 2) ? -1.0L : 1.0L;
    int pc = 2 * lmin - 2 * k0 + M - Mp, ps = 2 * k0 - M + Mp;
    for (int t = 0; t < T; ++t) {
        xreal xt = x[t];
        xreal ch = (1.0L + xt) / 2.0L, sh = (1.0L - xt) / 2.0L;
        ch = sqrtl(ch < 0 ? 0 : (ch > 1 ? 1 : ch));
        sh = sqrtl(sh < 0 ? 0 : (sh > 1 ? 1 : sh));
        xreal v = lf;
        if (pc > 0) v += pc * logl(ch);
        if (ps > 0) v += ps * logl(sh);
        slog[t] = v;
    }
}

typedef struct { xreal *p, *q, *s; } xstate_t;

static inline xreal step_ld(xreal A, xreal B, xreal C, xreal x, xreal *p, xreal *q, xreal *s) {
    xreal raw = (A * x + C) * (*p) - B * (*q);
    xreal r = sqrtl(raw * raw + (*p) * (*p));
    if (r == 0.0L) r = 1.0L;
    xreal np_ = raw / r, nq = (*p) / r;
    *s = *s + logl(r);
    *p = np_;
    *q = nq;
    return np_ * expl(*s);
}

static void advance_ld(int l, int lmin, const xreal *A, const xreal *B, const xreal *C, int T, const double *x,
                       xreal sg, const xreal *slog, xstate_t st, xreal *lam) {
    if (l < lmin) {
        for (int t = 0; t < T; ++t) lam[t] = 0.0L;
    } else if (l == lmin) {
        for (int t = 0; t < T; ++t) {
            st.p[t] = sg; st.q[t] = 0.0L; st.s[t] = slog[t];
            lam[t] = sg * expl(slog[t]);
        }
    } else {
        for (int t = 0; t < T; ++t) lam[t] = step_ld(A[l], B[l], C[l], (xreal)x[t], &st.p[t], &st.q[t], &st.s[t]);
    }
}

/* oracle_synth in long double; same arguments and output layout (rounded to FP64 at the end). */
void oracle_synth_ld(int spin, int lmax, int T, const double *x, const cplx *alm, cplx *out, int m_lo,
                     int m_hi) {
    long K = (long)(lmax + 1) * (lmax + 2) / 2;
    long MT = (long)(lmax + 1) * T;
#pragma omp parallel
    {
        int L1 = lmax + 1;
        xreal *A = malloc(sizeof(xreal) * L1 * 8), *B = A + L1, *C = B + L1, *pref = C + L1;
        xreal *A2 = pref + L1, *B2 = A2 + L1, *C2 = B2 + L1, *pref2 = C2 + L1;
        xreal *buf = malloc(sizeof(xreal) * T * 10);
        xcplx *acc = malloc(sizeof(xcplx) * T * 4);
        xstate_t s1 = {buf, buf + T, buf + 2 * T}, s2 = {buf + 3 * T, buf + 4 * T, buf + 5 * T};
        xreal *lam1 = buf + 6 * T, *lam2 = buf + 7 * T, *slog1 = buf + 8 * T, *slog2 = buf + 9 * T;
#pragma omp for schedule(dynamic, 1)
        for (int m = m_lo; m < m_hi; ++m) {
            int lmin = m > abs(spin) ? m : abs(spin);
            xreal sg1, sg2;
            for (int t = 0; t < 4 * T; ++t) acc[t] = 0;
            if (spin == 0) {
                coeffs_ld(0, m, lmax, A, B, C, pref);
                seed_ld(0, m, T, x, &sg1, slog1);
                for (int l = 0; l <= lmax; ++l) {
                    advance_ld(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    if (l < lmin) continue;
                    xcplx a = alm[alm_base(m, lmax) + l - m];
                    xreal par = (l % 2) ? -1.0L : 1.0L;
                    for (int t = 0; t < T; ++t) {
                        xcplx c = a * lam1[t];
                        acc[t] += c;
                        acc[T + t] += par * c;
                    }
                }
                for (int t = 0; t < T; ++t) {
                    out[(long)m * T + t] = (cplx)acc[t];
                    out[MT + (long)m * T + t] = (cplx)acc[T + t];
                }
            } else {
                coeffs_ld(2, m, lmax, A, B, C, pref);
                coeffs_ld(-2, m, lmax, A2, B2, C2, pref2);
                seed_ld(2, m, T, x, &sg1, slog1);
                seed_ld(-2, m, T, x, &sg2, slog2);
                for (int l = 0; l <= lmax; ++l) {
                    advance_ld(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    advance_ld(l, lmin, A2, B2, C2, T, x, sg2, slog2, s2, lam2);
                    if (l < lmin) continue;
                    long i = alm_base(m, lmax) + l - m;
                    xcplx e = alm[i], b = alm[K + i];
                    xcplx cp = -(e + I * b) * pref[l], cm = -(e - I * b) * pref[l];
                    xreal par = (l % 2) ? -1.0L : 1.0L;
                    for (int t = 0; t < T; ++t) {
                        acc[t] += cp * lam1[t];
                        acc[T + t] += par * cp * lam2[t];
                        acc[2 * T + t] += cm * lam2[t];
                        acc[3 * T + t] += par * cm * lam1[t];
                    }
                }
                for (int c = 0; c < 4; ++c)
                    for (int t = 0; t < T; ++t) out[c * MT + (long)m * T + t] = (cplx)acc[c * T + t];
            }
        }
        free(acc);
        free(buf);
        free(A);
    }
}

/* oracle_adjoint in long double; same arguments and output layout. */
void oracle_adjoint_ld(int spin, int lmax, int T, const double *x, const cplx *in, cplx *out, int m_lo,
                       int m_hi) {
    long K = (long)(lmax + 1) * (lmax + 2) / 2;
    long MT = (long)(lmax + 1) * T;
#pragma omp parallel
    {
        int L1 = lmax + 1;
        xreal *A = malloc(sizeof(xreal) * L1 * 8), *B = A + L1, *C = B + L1, *pref = C + L1;
        xreal *A2 = pref + L1, *B2 = A2 + L1, *C2 = B2 + L1, *pref2 = C2 + L1;
        xreal *buf = malloc(sizeof(xreal) * T * 10);
        xstate_t s1 = {buf, buf + T, buf + 2 * T}, s2 = {buf + 3 * T, buf + 4 * T, buf + 5 * T};
        xreal *lam1 = buf + 6 * T, *lam2 = buf + 7 * T, *slog1 = buf + 8 * T, *slog2 = buf + 9 * T;
#pragma omp for schedule(dynamic, 1)
        for (int m = m_lo; m < m_hi; ++m) {
            int lmin = m > abs(spin) ? m : abs(spin);
            xreal sg1, sg2;
            long base = alm_base(m, lmax);
            if (spin == 0) {
                coeffs_ld(0, m, lmax, A, B, C, pref);
                seed_ld(0, m, T, x, &sg1, slog1);
                const cplx *Vn = in + (long)m * T, *Vs = in + MT + (long)m * T;
                for (int l = 0; l <= lmax; ++l) {
                    advance_ld(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    if (l < m) continue;
                    xcplx sn = 0, ss = 0;
                    for (int t = 0; t < T; ++t) { sn += lam1[t] * (xcplx)Vn[t]; ss += lam1[t] * (xcplx)Vs[t]; }
                    xreal par = (l % 2) ? -1.0L : 1.0L;
                    out[base + l - m] = (cplx)(pref[l] * (sn + par * ss));
                }
            } else {
                coeffs_ld(2, m, lmax, A, B, C, pref);
                coeffs_ld(-2, m, lmax, A2, B2, C2, pref2);
                seed_ld(2, m, T, x, &sg1, slog1);
                seed_ld(-2, m, T, x, &sg2, slog2);
                const cplx *Vpn = in + (long)m * T, *Sp = Vpn + MT, *Vmn = Sp + MT, *Sm = Vmn + MT;
                for (int l = 0; l <= lmax; ++l) {
                    advance_ld(l, lmin, A, B, C, T, x, sg1, slog1, s1, lam1);
                    advance_ld(l, lmin, A2, B2, C2, T, x, sg2, slog2, s2, lam2);
                    if (l < m) continue;
                    xcplx a1 = 0, a2 = 0, a3 = 0, a4 = 0;
                    for (int t = 0; t < T; ++t) {
                        a1 += lam1[t] * (xcplx)Vpn[t];
                        a2 += lam2[t] * (xcplx)Sp[t];
                        a3 += lam2[t] * (xcplx)Vmn[t];
                        a4 += lam1[t] * (xcplx)Sm[t];
                    }
                    xreal par = (l % 2) ? -1.0L : 1.0L;
                    out[base + l - m] = (cplx)(pref[l] * (a1 + par * a2));
                    out[K + base + l - m] = (cplx)(pref[l] * (a3 + par * a4));
                }
            }
        }
        free(buf);
        free(A);
    }
}
