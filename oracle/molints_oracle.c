/*
 * molints_oracle.c -- CPU oracle for the two-electron repulsion integral (ERI) path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file; only the
 * tests, __graft_entry__.smoke() (as the checker) and bench.py's CPU-baseline / reference
 * arm use it.  It is a plain-C, FP64 restatement of the reference Julia algorithms of
 * MolecularIntegrals.jl (paths below are relative to that project):
 *
 *   Boys function        Fm / farray / farray_recur / Fm_asymp     src/Boys.jl:9-36
 *   HGP VRR              vrr!                                      src/HGP.jl:135-242
 *   HGP HRR              hrr (primitive) / chrr (contracted)       src/HGP.jl:83-116, 392-424
 *   contraction          cvrr                                      src/HGP.jl:50-68
 *   driver               all_twoe_ints_chrr                        src/HGP.jl:22-34
 *   Huzinaga ERI         coulomb / Barray / Bterm / fB / B0        src/ERI.jl:15-94
 *   generic driver       all_twoe_ints                             src/ERI.jl:104-112
 *   normalisation        PGBF/CGBF normalize!, contract            src/Basis.jl:42-98
 *   AO tables            shell_indices, m2ao, shift_* tables       src/Basis.jl:269-395
 *   packed layout        triangle / iindex                         src/Utils.jl:14-19
 *
 * The reference HGP driver is not a correct integral producer for l>0; the restatement
 * fixes these defects (and only these), so that its output equals the normalised
 * all_twoe_ints layout:
 *   D1  packed order: results go to iindex(i,j,k,l), not to the fetcher's enumeration index
 *       (src/Basis.jl:203-209 versus src/ERI.jl:109).
 *   D2  sub-shell index: the chrr output is indexed by the cumulative AO index
 *       nao[L-1]+m, not by the within-shell m (src/HGP.jl:29-31 versus :87-115).
 *   D3  normalisation: primitive and contracted norms are applied (src/HGP.jl:57-63 uses raw
 *       coefficients; src/Basis.jl:86-98 applies both).
 *   D5  VRR prefactor: vrr! uses 2 pi^2.5 (zeta+eta)^-3/2 (src/HGP.jl:150); the HGP value
 *       [00|00]^(0) is 2 pi^2.5 / (zeta eta sqrt(zeta+eta)).  The two agree only when
 *       zeta*eta == zeta+eta, which holds for every VRR/HRR test in test/runtests.jl:152-235
 *       (all exponents 1.0).  prefactor_mode 1 reproduces the literal reference formula so
 *       that a test can show the difference; the drivers always use mode 0.
 *
 * Third-party arithmetic: the reference's Fm calls SpecialFunctions.jl v2.3.0 gamma and
 * gamma_inc (Manifest.toml).  It is not vendored; the same mathematical value
 * F_m(T) = Gamma(m+1/2) P(m+1/2,T) / (2 T^(m+1/2)) is computed here by the everywhere
 * convergent series F_m(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) in long double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_LTAB 8              /* cartesian AO tables up to l = 8 */
#define OR_MAXAO 165           /* nao_cum[8] */

static int g_ready = 0;
static int g_ncart[OR_LTAB + 1];
static int g_nao[OR_LTAB + 1];           /* cumulative count, src/Basis.jl:320-321 */
static int g_ao2m[OR_MAXAO][3];          /* src/Basis.jl:306-314 */
static int g_shell_number[OR_MAXAO];     /* src/Basis.jl:356-364 */
static int g_shift_index[OR_MAXAO][3];   /* a - 1_i, -1 if none; src/Basis.jl:326-344 */
static int g_shift_plus[OR_MAXAO][3];    /* a + 1_i, -1 at the top shell; :366-385 */
static int g_shift_dir[OR_MAXAO];        /* first argmax of ao2m[a]; :346-354 */

/* Component order within a shell: src/Basis.jl:269-279 for l <= 4 (note the l=3 order
 * xxx,xxy,xxz,xyy,xzz,xyz,...), canonical (x-power descending, then y) above. */
static void shell_components(int l, int comps[][3]) {
    int n = 0;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) {
            comps[n][0] = i; comps[n][1] = j; comps[n][2] = l - i - j; ++n;
        }
    if (l == 3) { /* swap positions 4 and 5: xzz before xyz */
        int t[3]; memcpy(t, comps[4], sizeof t); memcpy(comps[4], comps[5], sizeof t);
        memcpy(comps[5], t, sizeof t);
    }
}

int oracle_ao_index(int i, int j, int k) {
    int l = i + j + k;
    if (i < 0 || j < 0 || k < 0 || l > OR_LTAB) return -1;
    int base = l ? g_nao[l - 1] : 0;
    for (int a = base; a < g_nao[l]; ++a)
        if (g_ao2m[a][0] == i && g_ao2m[a][1] == j && g_ao2m[a][2] == k) return a;
    return -1;
}

void oracle_init(void) {
    if (g_ready) return;
    int a = 0;
    for (int l = 0; l <= OR_LTAB; ++l) {
        int comps[64][3];
        g_ncart[l] = (l + 1) * (l + 2) / 2;
        shell_components(l, comps);
        for (int m = 0; m < g_ncart[l]; ++m, ++a) {
            memcpy(g_ao2m[a], comps[m], sizeof comps[m]);
            g_shell_number[a] = l;
        }
        g_nao[l] = a;
    }
    g_ready = 1; /* ao_index below needs g_nao */
    for (a = 0; a < g_nao[OR_LTAB]; ++a) {
        int *m = g_ao2m[a];
        int best = 0;
        for (int i = 1; i < 3; ++i) if (m[i] > m[best]) best = i;
        g_shift_dir[a] = best;
        for (int i = 0; i < 3; ++i) {
            int mm[3] = {m[0], m[1], m[2]};
            if (m[i] == 0) g_shift_index[a][i] = -1;
            else { mm[i] -= 1; g_shift_index[a][i] = oracle_ao_index(mm[0], mm[1], mm[2]); }
            int mp[3] = {m[0], m[1], m[2]};
            if (g_shell_number[a] == OR_LTAB) g_shift_plus[a][i] = -1;
            else { mp[i] += 1; g_shift_plus[a][i] = oracle_ao_index(mp[0], mp[1], mp[2]); }
        }
    }
}

int oracle_nao(int l) { oracle_init(); return (l < 0) ? 0 : g_nao[l]; }
void oracle_ao2m(int a, int *out3) { oracle_init(); memcpy(out3, g_ao2m[a], 3 * sizeof(int)); }

/* ---------------------------------------------------------------- Boys function */

static double dfact2(int n) { /* factorial2, src/Utils.jl:5; (-1)!! = 1 */
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

/* Gamma(a, x) e^x x^-a for x > a + 1 by the Legendre continued fraction (DLMF 8.9.2),
 * evaluated with the modified Lentz method. */
static long double upper_gamma_cf(long double a, long double x) {
    const long double tiny = 1e-4000L;
    long double b = x + 1.0L - a, c = 1.0L / tiny, d = 1.0L / b, h = d;
    for (int i = 1; i < 10000; ++i) {
        long double an = -i * (i - a);
        b += 2.0L;
        d = an * d + b;
        if (fabsl(d) < tiny) d = tiny;
        c = b + an / c;
        if (fabsl(c) < tiny) c = tiny;
        d = 1.0L / d;
        long double del = d * c;
        h *= del;
        if (fabsl(del - 1.0L) < 1e-21L) break;
    }
    return h;
}

/* F_m(T) in long double: the everywhere convergent series below T = 50, the continued
 * fraction for the upper incomplete gamma function above. */
static long double boys_ld(int m, long double t) {
    if (t < 1e-18L) return 1.0L / (2 * m + 1);
    if (t > 50.0L && t > m + 1.5L) {
        /* F_m = (Gamma(m+1/2) - Gamma(m+1/2, T)) / (2 T^(m+1/2)) */
        long double a = m + 0.5L;
        long double g = sqrtl(3.14159265358979323846264338327950288L);
        for (int k = 1; k <= m; ++k) g *= (k - 0.5L);
        long double ta = powl(t, a);
        long double upper = expl(-t) * ta * upper_gamma_cf(a, t);
        return (g - upper) / (2.0L * ta);
    }
    long double sum = 0.0L, term = 1.0L / (2 * m + 1);
    for (int k = 0; k < 100000; ++k) {
        sum += term;
        if (k > t && term < sum * 1e-22L) break;
        term *= 2.0L * t / (2 * m + 2 * k + 3);
    }
    return expl(-t) * sum;
}

/* Fm(m,T), src/Boys.jl:29-34 (T < 1e-18 returns 1/(2m+1)). */
double oracle_boys(int m, double T) {
    if (T < 1e-18) return 1.0 / (2 * m + 1);
    return (double)boys_ld(m, T);
}

static long double boys_asymp_ld(int m, long double T) {
    long double f2 = 1.0L;
    for (int k = 2 * m - 1; k > 1; k -= 2) f2 *= k;
    return sqrtl(3.14159265358979323846264338327950288L / 2) * f2 / powl(2 * T, m + 0.5L);
}

/* Fm_asymp, src/Boys.jl:36. */
double oracle_boys_asymp(int m, double T) {
    return sqrt(M_PI / 2) * dfact2(2 * m - 1) / pow(2 * T, m + 0.5);
}

/* Tmax of farray (src/Boys.jl:19).  The reference value 30 is the default; tests may raise
 * it to make the oracle's Boys function exact at every T. */
static double g_boys_tmax = 30.0;
void oracle_set_boys_tmax(double tmax) { g_boys_tmax = tmax; }
double oracle_get_boys_tmax(void) { return g_boys_tmax; }

/* Orientation of each shell quartet handed to chrr.  0 (default): the reference's, chrr(I,J,K,L)
 * with I >= J, K >= L, pair(IJ) >= pair(KL) by shell index (src/HGP.jl:27-28).  1: the
 * engine's: in each pair the shell with the larger L is 'a' (ties keep the higher index
 * first), and the pair of higher class (la+lb, then la) is the bra.  The two are the same
 * mathematics; their rounding differs, and HRR accuracy depends strongly on which shell
 * receives the transferred angular momentum. */
static int g_orient = 0;
void oracle_set_orientation(int mode) { g_orient = mode; }
int oracle_get_orientation(void) { return g_orient; }

/* Orientation 2 (the engine's present rule): shell x goes first in the pair (x, y) if it has
 * the larger L, or, for equal L and for an f-d pair, the larger sqrt(min * max exponent).
 * Moving angular momentum away from the tighter shell keeps the HRR from cancelling. */
static double oracle_tightness(const double *expn, const int *nprim, const int *prim_off, int s) {
    double lo = expn[prim_off[s]], hi = lo;
    for (int i = 1; i < nprim[s]; ++i) {
        const double e = expn[prim_off[s] + i];
        if (e < lo) lo = e;
        if (e > hi) hi = e;
    }
    return sqrt(lo * hi);
}
#define oracle_a_first(bp, x, y)                                                                     \
    (((bp)->L[x] == (bp)->L[y] || ((bp)->L[x] >= 2 && (bp)->L[y] >= 2 && (bp)->L[x] + (bp)->L[y] == 5)) \
         ? oracle_tightness((bp)->expn_in, (bp)->nprim, (bp)->prim_off, x) >                            \
               oracle_tightness((bp)->expn_in, (bp)->nprim, (bp)->prim_off, y)                          \
         : (bp)->L[x] > (bp)->L[y])

/* ---------------------------------------------------------------- the HGP core, twice */

static inline int64_t tri64(int64_t i) { return i * (i + 1) / 2; }
int64_t oracle_iindex(int64_t i, int64_t j, int64_t k, int64_t l);
size_t oracle_hrr_size(int la, int lb, int lc, int ld);

#define REAL double
#define PFX(name) d_##name
#define R_EXP exp
#define R_SQRT sqrt
#define R_POW pow
#define R_PI M_PI
#define BOYS_EXACT(m, T) oracle_boys((m), (T))
#define BOYS_ASYMP(m, T) oracle_boys_asymp((m), (T))
#include "hgp_core.h"
#undef REAL
#undef PFX
#undef R_EXP
#undef R_SQRT
#undef R_POW
#undef R_PI
#undef BOYS_EXACT
#undef BOYS_ASYMP

#define REAL long double
#define PFX(name) ld_##name
#define R_EXP expl
#define R_SQRT sqrtl
#define R_POW powl
#define R_PI 3.14159265358979323846264338327950288L
#define BOYS_EXACT(m, T) boys_ld((m), (T))
#define BOYS_ASYMP(m, T) boys_asymp_ld((m), (T))
#include "hgp_core.h"
#undef REAL
#undef PFX
#undef R_EXP
#undef R_SQRT
#undef R_POW
#undef R_PI
#undef BOYS_EXACT
#undef BOYS_ASYMP

void oracle_farray(int mmax, double T, double *out) { d_farray(mmax, T, out); }

void oracle_vrr(int amax, int cmax, double aexpn, double bexpn, double cexpn, double dexpn,
                const double *A, const double *B, const double *C, const double *D,
                int prefactor_mode, double *vrrs) {
    d_vrr(amax, cmax, aexpn, bexpn, cexpn, dexpn, A, B, C, D, prefactor_mode, vrrs);
}

size_t oracle_hrr_size(int la, int lb, int lc, int ld) {
    oracle_init();
    return (size_t)g_nao[la + lb] * g_nao[lb] * g_nao[lc + ld] * g_nao[ld];
}

/* hrr(ashell,bshell,cshell,dshell, exps, centres), src/HGP.jl:392-424. */
void oracle_hrr(int la, int lb, int lc, int ld, double aexpn, double bexpn, double cexpn,
                double dexpn, const double *A, const double *B, const double *C,
                const double *D, int prefactor_mode, double *hrrs) {
    oracle_init();
    int amax = la + lb, cmax = lc + ld, mmax = amax + cmax + 1;
    size_t nv = (size_t)mmax * g_nao[amax] * g_nao[cmax];
    double *v = (double *)malloc(sizeof(double) * nv);
    d_vrr(amax, cmax, aexpn, bexpn, cexpn, dexpn, A, B, C, D, prefactor_mode, v);
    d_hrr_block(la, lb, lc, ld, A, B, C, D, v, hrrs); /* m = 0 slice is the first block */
    free(v);
}

static int64_t eri_packed_hgp_dispatch(int nshell, const double *xyz, const int *L, const int *nprim,
                                   const int *prim_off, const double *expn, const double *coef,
                                   double *out, int nthreads, int64_t stride);

int oracle_eri_packed_hgp(int nshell, const double *xyz, const int *L, const int *nprim,
                          const int *prim_off, const double *expn, const double *coef,
                          double *out, int nthreads) {
    int64_t r = eri_packed_hgp_dispatch(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads, 1);
    return r < 0 ? (int)r : 0;
}

/* The same driver over every stride-th shell quartet only (a bounded CPU-baseline sample);
 * returns the number of integrals written, or -1. */
int64_t oracle_eri_packed_hgp_sample(int nshell, const double *xyz, const int *L,
                                     const int *nprim, const int *prim_off, const double *expn,
                                     const double *coef, double *out, int nthreads,
                                     int64_t stride) {
    return eri_packed_hgp_dispatch(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads,
                               stride < 1 ? 1 : stride);
}


/* Dispatch of the HGP driver: FP64 (the oracle proper) or long double (near-exact). */
static int g_use_ld = 0;
static int64_t eri_packed_hgp_dispatch(int nshell, const double *xyz, const int *L, const int *nprim,
                                       const int *prim_off, const double *expn, const double *coef,
                                       double *out, int nthreads, int64_t stride) {
    if (!g_use_ld)
        return d_eri_packed_hgp_impl(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads, stride);
    return ld_eri_packed_hgp_impl(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads, stride);
}

/* all_twoe_ints_chrr restated as above, evaluated in long double (64-bit mantissa). */
int oracle_eri_packed_hgp_ld(int nshell, const double *xyz, const int *L, const int *nprim,
                             const int *prim_off, const double *expn, const double *coef,
                             double *out, int nthreads) {
    int64_t r = ld_eri_packed_hgp_impl(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads, 1);
    return r < 0 ? (int)r : 0;
}

/* One contracted, normalised shell quartet (ab|cd), out[ma][mb][mc][md]. */
int oracle_shell_quartet(int nshell, const double *xyz, const int *L, const int *nprim,
                         const int *prim_off, const double *expn, const double *coef,
                         int sa, int sb, int sc, int sd, double *out) {
    oracle_init();
    d_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0, 0, 0};
    d_basis_prepare(&b);
    d_shell_quartet(&b, sa, sb, sc, sd, out);
    d_basis_release(&b);
    return 0;
}

/* ---------------------------------------------------------------- normalisation */

/* PGBF norm after normalize!, src/Basis.jl:42-44: 1/sqrt(overlap(p,p)).  With the
 * self-overlap of src/OneInts.jl:41-52 at PA=PB=0 this is the closed form
 * (2a/pi)^(3/4) (4a)^(L/2) / sqrt((2I-1)!!(2J-1)!!(2K-1)!!). */
double oracle_pgbf_norm(double expn, int I, int J, int K) {
    int L = I + J + K;
    return pow(2 * expn / M_PI, 0.75) * pow(4 * expn, 0.5 * L) /
           sqrt(dfact2(2 * I - 1) * dfact2(2 * J - 1) * dfact2(2 * K - 1));
}

/* CGBF norm after the addbf! sequence, src/Basis.jl:73-83: 1/sqrt(<phi|phi>), where the
 * same-centre overlap of two normalised primitives with equal powers is
 * (2 sqrt(a b)/(a+b))^(L+3/2).  It depends on the shell only. */
double oracle_cgbf_norm(int L, int nprim, const double *expn, const double *coef) {
    double s = 0;
    for (int i = 0; i < nprim; ++i)
        for (int j = 0; j < nprim; ++j) {
            double a = expn[i], b = expn[j];
            s += coef[i] * coef[j] * pow(2 * sqrt(a * b) / (a + b), L + 1.5);
        }
    return 1.0 / sqrt(s);
}

/* ---------------------------------------------------------------- packed layout */

/* 0-based iindex (src/Utils.jl:14-19 minus one). */
int64_t oracle_iindex(int64_t i, int64_t j, int64_t k, int64_t l) {
    int64_t ij = i >= j ? tri64(i) + j : tri64(j) + i;
    int64_t kl = k >= l ? tri64(k) + l : tri64(l) + k;
    return ij >= kl ? tri64(ij) + kl : tri64(kl) + ij;
}
int64_t oracle_npacked(int64_t n) { return n * (n + 1) * (n * n + n + 2) / 8; }

/* ---------------------------------------------------------------- Huzinaga */

static double ipow(double x, int n) { double r = 1; for (int i = 0; i < n; ++i) r *= x; return r; }
static double factd(int n) { double r = 1; for (int i = 2; i <= n; ++i) r *= i; return r; }
static double binom(int n, int k) { return (k < 0 || k > n) ? 0 : factd(n) / (factd(k) * factd(n - k)); }

/* binomial_prefactor, src/OneInts.jl:93-94 */
static double binomial_prefactor(int s, int ia, int ib, double xpa, double xpb) {
    double sum = 0;
    for (int t = 0; t <= s; ++t)
        if (s - ia <= t && t <= ib)
            sum += binom(ia, s - t) * ipow(xpa, ia - s + t) * binom(ib, t) * ipow(xpb, ib - t);
    return sum;
}
/* fact_ratio2, B0, fB: src/ERI.jl:62-65 */
static double fact_ratio2(int a, int b) { return factd(a) / factd(b) / factd(a - 2 * b); }
static double B0(int i, int r, double g) { return fact_ratio2(i, r) * pow(4 * g, r - i); }
static double fB(int i, int l1, int l2, double p, double a, double b, int r, double g) {
    return binomial_prefactor(i, l1, l2, p - a, p - b) * B0(i, r, g);
}
/* Bterm (THO eq. 2.22), src/ERI.jl:67-75 */
static double Bterm(int i1, int i2, int r1, int r2, int u, int l1, int l2, int l3, int l4,
                    double Px, double Ax, double Bx, double Qx, double Cx, double Dx,
                    double g1, double g2, double delta) {
    int e = i1 + i2 - 2 * (r1 + r2);
    return fB(i1, l1, l2, Px, Ax, Bx, r1, g1) * ((i2 & 1) ? -1.0 : 1.0) *
           fB(i2, l3, l4, Qx, Cx, Dx, r2, g2) * ((u & 1) ? -1.0 : 1.0) * fact_ratio2(e, u) *
           ipow(Qx - Px, e - 2 * u) / pow(delta, e - u);
}
/* Barray, src/ERI.jl:77-94 */
static void Barray(int l1, int l2, int l3, int l4, double p, double a, double b, double q,
                   double c, double d, double g1, double g2, double delta, double *B) {
    int Imax = l1 + l2 + l3 + l4 + 1;
    for (int i = 0; i < Imax; ++i) B[i] = 0;
    for (int i1 = 0; i1 <= l1 + l2; ++i1)
        for (int i2 = 0; i2 <= l3 + l4; ++i2)
            for (int r1 = 0; r1 <= i1 / 2; ++r1)
                for (int r2 = 0; r2 <= i2 / 2; ++r2)
                    for (int u = 0; u <= (i1 + i2) / 2 - r1 - r2; ++u) {
                        int I = i1 + i2 - 2 * (r1 + r2) - u;
                        B[I] += Bterm(i1, i2, r1, r2, u, l1, l2, l3, l4, p, a, b, q, c, d, g1, g2, delta);
                    }
}

/* coulomb(aexpn,ax,ay,az,aI,aJ,aK, ...), src/ERI.jl:15-46 (raw primitives). */
double oracle_coulomb_prim(double aexpn, double ax, double ay, double az, int aI, int aJ, int aK,
                           double bexpn, double bx, double by, double bz, int bI, int bJ, int bK,
                           double cexpn, double cx, double cy, double cz, int cI, int cJ, int cK,
                           double dexpn, double dx, double dy, double dz, int dI, int dJ, int dK) {
    double rab2 = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
    double rcd2 = (cx - dx) * (cx - dx) + (cy - dy) * (cy - dy) + (cz - dz) * (cz - dz);
    double g1 = aexpn + bexpn, g2 = cexpn + dexpn;
    double px = (aexpn * ax + bexpn * bx) / g1, py = (aexpn * ay + bexpn * by) / g1,
           pz = (aexpn * az + bexpn * bz) / g1;
    double qx = (cexpn * cx + dexpn * dx) / g2, qy = (cexpn * cy + dexpn * dy) / g2,
           qz = (cexpn * cz + dexpn * dz) / g2;
    double rpq2 = (px - qx) * (px - qx) + (py - qy) * (py - qy) + (pz - qz) * (pz - qz);
    double delta = 0.25 * (1 / g1 + 1 / g2);
    double Bx[32], By[32], Bz[32];
    Barray(aI, bI, cI, dI, px, ax, bx, qx, cx, dx, g1, g2, delta, Bx);
    Barray(aJ, bJ, cJ, dJ, py, ay, by, qy, cy, dy, g1, g2, delta, By);
    Barray(aK, bK, cK, dK, pz, az, bz, qz, cz, dz, g1, g2, delta, Bz);
    double x = 0.25 * rpq2 / delta, s = 0;
    for (int I = 0; I <= aI + bI + cI + dI; ++I)
        for (int J = 0; J <= aJ + bJ + cJ + dJ; ++J)
            for (int K = 0; K <= aK + bK + cK + dK; ++K)
                s += Bx[I] * By[J] * Bz[K] * oracle_boys(I + J + K, x);
    return 2 * pow(M_PI, 2.5) / (g1 * g2 * sqrt(g1 + g2)) * exp(-aexpn * bexpn * rab2 / g1) *
           exp(-cexpn * dexpn * rcd2 / g2) * s;
}

/* all_twoe_ints(bfs, coulomb), src/ERI.jl:104-112 with contract (src/Basis.jl:86-98):
 * one normalised contracted Huzinaga integral per unique function quartet. */
int oracle_eri_packed_huzinaga(int nshell, const double *xyz, const int *L, const int *nprim,
                               const int *prim_off, const double *expn, const double *coef,
                               double *out, int nthreads) {
    oracle_init();
    d_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0, 0, 0};
    for (int s = 0; s < nshell; ++s)
        if (L[s] < 0 || L[s] > 6 || nprim[s] < 1) return -1;
    d_basis_prepare(&b);
    int n = b.nbf;
    int *fsh = (int *)malloc(sizeof(int) * n), *fao = (int *)malloc(sizeof(int) * n);
    for (int s = 0; s < nshell; ++s)
        for (int m = 0; m < g_ncart[L[s]]; ++m) {
            fsh[b.fn_off[s] + m] = s;
            fao[b.fn_off[s] + m] = (L[s] ? g_nao[L[s] - 1] : 0) + m;
        }
    int64_t npair = (int64_t)n * (n + 1) / 2;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t ij = 0; ij < npair; ++ij) {
        int64_t i = (int64_t)((sqrt(8.0 * (double)ij + 1.0) - 1.0) / 2.0);
        while (tri64(i) > ij) --i;
        while (tri64(i + 1) <= ij) ++i;
        int64_t j = ij - tri64(i);
        int f[4] = {(int)i, (int)j, 0, 0};
        for (int64_t kl = 0; kl <= ij; ++kl) {
            int64_t k = (int64_t)((sqrt(8.0 * (double)kl + 1.0) - 1.0) / 2.0);
            while (tri64(k) > kl) --k;
            while (tri64(k + 1) <= kl) ++k;
            f[2] = (int)k; f[3] = (int)(kl - tri64(k));
            double s = 0;
            int sh[4], pw[4][3];
            for (int t = 0; t < 4; ++t) {
                sh[t] = fsh[f[t]];
                memcpy(pw[t], g_ao2m[fao[f[t]]], sizeof pw[t]);
            }
            for (int pa = 0; pa < nprim[sh[0]]; ++pa)
                for (int pb = 0; pb < nprim[sh[1]]; ++pb)
                    for (int pc = 0; pc < nprim[sh[2]]; ++pc)
                        for (int pd = 0; pd < nprim[sh[3]]; ++pd) {
                            int ia = prim_off[sh[0]] + pa, ib = prim_off[sh[1]] + pb;
                            int ic = prim_off[sh[2]] + pc, id = prim_off[sh[3]] + pd;
                            const double *A = xyz + 3 * sh[0], *B = xyz + 3 * sh[1];
                            const double *C = xyz + 3 * sh[2], *D = xyz + 3 * sh[3];
                            double v = oracle_coulomb_prim(
                                expn[ia], A[0], A[1], A[2], pw[0][0], pw[0][1], pw[0][2],
                                expn[ib], B[0], B[1], B[2], pw[1][0], pw[1][1], pw[1][2],
                                expn[ic], C[0], C[1], C[2], pw[2][0], pw[2][1], pw[2][2],
                                expn[id], D[0], D[1], D[2], pw[3][0], pw[3][1], pw[3][2]);
                            s += b.ncoef[ia] * b.ncoef[ib] * b.ncoef[ic] * b.ncoef[id] * v;
                        }
            for (int t = 0; t < 4; ++t) s *= d_comp_factor(fao[f[t]]);
            out[tri64(ij) + kl] = s;
        }
    }
    free(fsh); free(fao);
    d_basis_release(&b);
    return 0;
}

/* ---------------------------------------------------------------- Rys quadrature */

/* Rys roots and weights in long double, independently of the reference's fitted polynomials
 * (Root1..Root5, src/Rys.jl:176-1478): the measure exp(-X t^2) dt on t in [0,1] is
 * discretised by Gauss-Legendre on [0, t_max] (t_max = min(1, sqrt(80/X)), beyond which the
 * measure is below e^-80), the Stieltjes procedure gives the recurrence of the polynomials
 * orthogonal in x = t^2 (discretised Stieltjes, Gautschi), the nodes are the zeros of the
 * degree-n polynomial found by Sturm bisection of the Jacobi matrix, and the weights are the
 * Christoffel numbers 1 / sum_k p_k(x_i)^2 of the orthonormal polynomials. */
#define RYS_NGL 240
static long double g_gl_t[RYS_NGL], g_gl_w[RYS_NGL];
static int g_gl_ready = 0;

static void gauss_legendre_ld(void) {
    if (g_gl_ready) return;
    const int n = RYS_NGL;
    const long double pi = 3.14159265358979323846264338327950288L;
    for (int i = 0; i < (n + 1) / 2; ++i) {
        long double z = cosl(pi * (i + 0.75L) / (n + 0.5L)), pp = 0;
        for (int it = 0; it < 100; ++it) {
            long double p1 = 1, p2 = 0;
            for (int j = 1; j <= n; ++j) {
                long double p3 = p2;
                p2 = p1;
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1);
            long double dz = p1 / pp;
            z -= dz;
            if (fabsl(dz) < 1e-21L) break;
        }
        /* nodes on [-1,1] -> [0,1] */
        g_gl_t[i] = (1 - z) / 2;
        g_gl_t[n - 1 - i] = (1 + z) / 2;
        g_gl_w[i] = g_gl_w[n - 1 - i] = 1.0L / ((1 - z * z) * pp * pp);
    }
    g_gl_ready = 1;
}

/* number of eigenvalues of the symmetric tridiagonal (a, sqrt(b)) below x (Sturm count) */
static int sturm_count(int n, const long double *a, const long double *b, long double x) {
    int c = 0;
    long double q = a[0] - x;
    if (q < 0) ++c;
    for (int k = 1; k < n; ++k) {
        if (q == 0) q = 1e-4000L;
        q = (a[k] - x) - b[k] / q;
        if (q < 0) ++c;
    }
    return c;
}

int oracle_rys_roots(int n, double X, double *roots, double *weights) {
    if (n < 1 || n > 12 || !(X >= 0)) return -1;
    gauss_legendre_ld();
    long double tmax = X > 80.0 ? sqrtl(80.0L / X) : 1.0L;
    long double x[RYS_NGL], lam[RYS_NGL], p0[RYS_NGL], p1[RYS_NGL];
    for (int k = 0; k < RYS_NGL; ++k) {
        long double t = tmax * g_gl_t[k];
        x[k] = t * t;
        lam[k] = tmax * g_gl_w[k] * expl(-(long double)X * t * t);
        p0[k] = 0;
        p1[k] = 1;
    }
    long double a[16], b[16], norm_prev = 0;
    for (int j = 0; j < n; ++j) {
        long double nrm = 0, xn = 0;
        for (int k = 0; k < RYS_NGL; ++k) {
            nrm += lam[k] * p1[k] * p1[k];
            xn += lam[k] * x[k] * p1[k] * p1[k];
        }
        a[j] = xn / nrm;
        b[j] = j == 0 ? nrm : nrm / norm_prev;
        norm_prev = nrm;
        for (int k = 0; k < RYS_NGL; ++k) {
            long double pn = (x[k] - a[j]) * p1[k] - (j ? b[j] : 0) * p0[k];
            p0[k] = p1[k];
            p1[k] = pn;
        }
    }
    for (int i = 0; i < n; ++i) {
        long double lo = 0, hi = 1;
        for (int it = 0; it < 200; ++it) {
            long double mid = (lo + hi) / 2;
            if (sturm_count(n, a, b, mid) > i) hi = mid; else lo = mid;
            if (hi - lo < 1e-22L * hi) break;
        }
        long double xi = (lo + hi) / 2;
        /* orthonormal polynomials at xi: p_{k+1} = ((x - a_k) p_k - sqrt(b_k) p_{k-1}) / sqrt(b_{k+1}) */
        long double s = 0, q0 = 0, q1 = 1 / sqrtl(b[0]);
        s += q1 * q1;
        for (int k = 0; k + 1 < n; ++k) {
            long double q2 = ((xi - a[k]) * q1 - (k ? sqrtl(b[k]) : 0) * q0) / sqrtl(b[k + 1]);
            q0 = q1;
            q1 = q2;
            s += q1 * q1;
        }
        roots[i] = (double)xi;
        weights[i] = (double)(1 / s);
    }
    return 0;
}

/* RecurFactors, Recur, Shift and Int1d of src/Rys.jl:86-156, with the root in x = t^2
 * (the reference passes u = t^2/(1-t^2): 1/(1+u) = 1-x, u/(1+u) = x). */
static double rys_int1d(double x, int i, int j, int k, int l, double xi, double xj, double xk,
                        double xl, double ai, double aj, double ak, double al, double G[8][8]) {
    const int n = i + j, m = k + l;
    const double A = ai + aj, B = ak + al;
    const double Px = (ai * xi + aj * xj) / A, Qx = (ak * xk + al * xl) / B;
    const double ooopt = 1 - x, fact = x / (A + B);
    const double B0 = 0.5 * fact, B1 = 0.5 * ooopt / A + 0.5 * fact, B1p = 0.5 * ooopt / B + 0.5 * fact;
    const double C = (Px - xi) * ooopt + (B * (Qx - xi) + A * (Px - xi)) * fact;
    const double Cp = (Qx - xk) * ooopt + (B * (Qx - xk) + A * (Px - xk)) * fact;
    G[0][0] = M_PI * exp(-ai * aj * (xi - xj) * (xi - xj) / (ai + aj) -
                         ak * al * (xk - xl) * (xk - xl) / (ak + al)) / sqrt(A * B);
    if (n > 0) G[1][0] = C * G[0][0];
    if (m > 0) G[0][1] = Cp * G[0][0];
    for (int a = 2; a <= n; ++a) G[a][0] = B1 * (a - 1) * G[a - 2][0] + C * G[a - 1][0];
    for (int bb = 2; bb <= m; ++bb) G[0][bb] = B1p * (bb - 1) * G[0][bb - 2] + Cp * G[0][bb - 1];
    if (m > 0 && n > 0)
        for (int a = 1; a <= n; ++a) {
            G[a][1] = a * B0 * G[a - 1][0] + Cp * G[a][0];
            for (int bb = 2; bb <= m; ++bb)
                G[a][bb] = B1p * (bb - 1) * G[a][bb - 2] + a * B0 * G[a - 1][bb - 1] + Cp * G[a][bb - 1];
        }
    /* Shift: I(i,j,k,l) from G(n,m) = I(n,0,m,0) */
    double ijkl = 0;
    for (int mm = 0; mm <= l; ++mm) {
        double ijm0 = 0;
        for (int nn = 0; nn <= j; ++nn) ijm0 += binom(j, nn) * ipow(xi - xj, j - nn) * G[nn + i][mm + k];
        ijkl += binom(l, mm) * ipow(xk - xl, l - mm) * ijm0;
    }
    return ijkl;
}

/* coulomb_rys(PGBF...) without norms, src/Rys.jl:59-83. */
double oracle_coulomb_rys_prim(double aexpn, const double *A, const int *ia, double bexpn,
                               const double *B, const int *ib, double cexpn, const double *C,
                               const int *ic, double dexpn, const double *D, const int *id) {
    int norder = (ia[0] + ia[1] + ia[2] + ib[0] + ib[1] + ib[2] + ic[0] + ic[1] + ic[2] + id[0] +
                  id[1] + id[2]) / 2 + 1;
    double zeta = aexpn + bexpn, eta = cexpn + dexpn, rho = zeta * eta / (zeta + eta);
    double P[3], Q[3], rpq2 = 0;
    for (int t = 0; t < 3; ++t) {
        P[t] = (aexpn * A[t] + bexpn * B[t]) / zeta;
        Q[t] = (cexpn * C[t] + dexpn * D[t]) / eta;
        rpq2 += (P[t] - Q[t]) * (P[t] - Q[t]);
    }
    double roots[16], weights[16], G[8][8], s = 0;
    if (oracle_rys_roots(norder, rpq2 * rho, roots, weights) != 0) return NAN;
    for (int r = 0; r < norder; ++r) {
        double v = weights[r];
        for (int t = 0; t < 3; ++t)
            v *= rys_int1d(roots[r], ia[t], ib[t], ic[t], id[t], A[t], B[t], C[t], D[t], aexpn, bexpn,
                           cexpn, dexpn, G);
        s += v;
    }
    return 2 * sqrt(rho / M_PI) * s;
}

/* all_twoe_ints_rys, src/Rys.jl:16-43, with the contracted-function norms applied (D4): one
 * normalised contracted Rys integral per unique function quartet, at iindex. */
int oracle_eri_packed_rys(int nshell, const double *xyz, const int *L, const int *nprim,
                          const int *prim_off, const double *expn, const double *coef,
                          double *out, int nthreads) {
    oracle_init();
    d_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0, 0, 0};
    for (int s = 0; s < nshell; ++s)
        if (L[s] < 0 || L[s] > 4 || nprim[s] < 1) return -1;
    d_basis_prepare(&b);
    int n = b.nbf;
    int *fsh = (int *)malloc(sizeof(int) * n), *fao = (int *)malloc(sizeof(int) * n);
    for (int s = 0; s < nshell; ++s)
        for (int m = 0; m < g_ncart[L[s]]; ++m) {
            fsh[b.fn_off[s] + m] = s;
            fao[b.fn_off[s] + m] = (L[s] ? g_nao[L[s] - 1] : 0) + m;
        }
    int64_t npair = (int64_t)n * (n + 1) / 2;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t ij = 0; ij < npair; ++ij) {
        int64_t i = (int64_t)((sqrt(8.0 * (double)ij + 1.0) - 1.0) / 2.0);
        while (tri64(i) > ij) --i;
        while (tri64(i + 1) <= ij) ++i;
        int f[4] = {(int)i, (int)(ij - tri64(i)), 0, 0};
        for (int64_t kl = 0; kl <= ij; ++kl) {
            int64_t k = (int64_t)((sqrt(8.0 * (double)kl + 1.0) - 1.0) / 2.0);
            while (tri64(k) > kl) --k;
            while (tri64(k + 1) <= kl) ++k;
            f[2] = (int)k;
            f[3] = (int)(kl - tri64(k));
            int sh[4];
            for (int t = 0; t < 4; ++t) sh[t] = fsh[f[t]];
            double s = 0;
            for (int pa = 0; pa < nprim[sh[0]]; ++pa)
                for (int pb = 0; pb < nprim[sh[1]]; ++pb)
                    for (int pc = 0; pc < nprim[sh[2]]; ++pc)
                        for (int pd = 0; pd < nprim[sh[3]]; ++pd) {
                            int ii[4] = {prim_off[sh[0]] + pa, prim_off[sh[1]] + pb,
                                         prim_off[sh[2]] + pc, prim_off[sh[3]] + pd};
                            double v = oracle_coulomb_rys_prim(
                                expn[ii[0]], xyz + 3 * sh[0], g_ao2m[fao[f[0]]], expn[ii[1]],
                                xyz + 3 * sh[1], g_ao2m[fao[f[1]]], expn[ii[2]], xyz + 3 * sh[2],
                                g_ao2m[fao[f[2]]], expn[ii[3]], xyz + 3 * sh[3], g_ao2m[fao[f[3]]]);
                            s += b.ncoef[ii[0]] * b.ncoef[ii[1]] * b.ncoef[ii[2]] * b.ncoef[ii[3]] * v;
                        }
            for (int t = 0; t < 4; ++t) s *= d_comp_factor(fao[f[t]]);
            out[tri64(ij) + kl] = s;
        }
    }
    free(fsh); free(fao);
    d_basis_release(&b);
    return 0;
}
