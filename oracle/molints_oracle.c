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

/* Fm(m,T), src/Boys.jl:29-34 (T < 1e-18 returns 1/(2m+1)). */
double oracle_boys(int m, double T) {
    if (T < 1e-18) return 1.0 / (2 * m + 1);
    if (T > 50.0 && T > m + 1.5) {
        /* F_m = (Gamma(m+1/2) - Gamma(m+1/2, T)) / (2 T^(m+1/2)) */
        long double a = m + 0.5L, t = T;
        long double g = sqrtl(3.14159265358979323846264338327950288L);
        for (int k = 1; k <= m; ++k) g *= (k - 0.5L);
        long double ta = powl(t, a);
        long double upper = expl(-t) * ta * upper_gamma_cf(a, t);
        return (double)((g - upper) / (2.0L * ta));
    }
    long double t = T, sum = 0.0L, term = 1.0L / (2 * m + 1);
    for (int k = 0; k < 100000; ++k) {
        sum += term;
        if (k > T && term < sum * 1e-22L) break;
        term *= 2.0L * t / (2 * m + 2 * k + 3);
    }
    return (double)(expl(-t) * sum);
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

/* farray(mmax,T), src/Boys.jl:19-27 with farray_recur :9-17; out[0..mmax-1] = F_0..F_mmax-1. */
void oracle_farray(int mmax, double T, double *out) {
    if (T < g_boys_tmax) {
        out[mmax - 1] = oracle_boys(mmax - 1, T);
        double emt = exp(-T);
        for (int m = mmax - 2; m >= 0; --m) out[m] = (2 * T * out[m + 1] + emt) / (2 * m + 1);
        return;
    }
    out[mmax - 1] = oracle_boys_asymp(mmax - 1, T);
    for (int m = mmax - 2; m >= 0; --m) out[m] = T * out[m + 1] / (m + 0.5);
}

/* ---------------------------------------------------------------- HGP VRR / HRR */

static inline double dist2(const double *a, const double *b) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

/* vrr!(vrrs, amax, cmax, ...), src/HGP.jl:135-242.  vrrs is [mmax][nao(amax)][nao(cmax)]
 * (m fastest in the reference; slowest here -- the layout is internal).
 * prefactor_mode 0: HGP prefactor 2 pi^2.5/(zeta eta sqrt(zeta+eta)) (D5 fixed);
 * prefactor_mode 1: the literal src/HGP.jl:150 expression 2 pi^2.5 (zeta+eta)^-3/2. */
void oracle_vrr(int amax, int cmax, double aexpn, double bexpn, double cexpn, double dexpn,
                const double *A, const double *B, const double *C, const double *D,
                int prefactor_mode, double *vrrs) {
    oracle_init();
    const int mmax = amax + cmax + 1;
    const int nA = g_nao[amax], nC = g_nao[cmax];
#define V(m, a, c) vrrs[((size_t)(m) * nA + (a)) * nC + (c)]
    memset(vrrs, 0, sizeof(double) * (size_t)mmax * nA * nC);
    double zeta = aexpn + bexpn, eta = cexpn + dexpn, ze = zeta + eta;
    double ooz = 1 / zeta, ooe = 1 / eta, ooze = 1 / ze, oortze = sqrt(ooze);
    double P[3], Q[3], W[3], PA[3], WP[3], QC[3], WQ[3];
    for (int i = 0; i < 3; ++i) {
        P[i] = (aexpn * A[i] + bexpn * B[i]) * ooz;
        Q[i] = (cexpn * C[i] + dexpn * D[i]) * ooe;
        W[i] = (zeta * P[i] + eta * Q[i]) * ooze;
        PA[i] = P[i] - A[i]; WP[i] = W[i] - P[i]; QC[i] = Q[i] - C[i]; WQ[i] = W[i] - Q[i];
    }
    double rab2 = dist2(A, B), rcd2 = dist2(C, D), rpq2 = dist2(P, Q);
    double T = zeta * eta * rpq2 * ooze;
    double ex = exp(-aexpn * bexpn * rab2 * ooz - cexpn * dexpn * rcd2 * ooe);
    double pref = (prefactor_mode == 1) ? 2 * M_PI * M_PI * sqrt(M_PI) * ooze * oortze * ex
                                        : 2 * M_PI * M_PI * sqrt(M_PI) * ooz * ooe * oortze * ex;
    double Fms[64];
    oracle_farray(mmax, T, Fms);
    for (int m = 0; m < mmax; ++m) V(m, 0, 0) = pref * Fms[m];
    if (mmax == 1) return;
    /* a-build, eq. 6a with c = 0: src/HGP.jl:180-197 */
    for (int aplus = 1; aplus < nA; ++aplus) {
        int ashell = g_shell_number[aplus];
        int i = g_shift_dir[aplus];
        int a = g_shift_index[aplus][i];
        int lim = mmax - ashell;
        int aminus = g_shift_index[a][i];
        if (aminus >= 0) {
            double a_i = 0.5 * ooz * g_ao2m[a][i];
            for (int m = 0; m < lim; ++m)
                V(m, aplus, 0) = PA[i] * V(m, a, 0) + WP[i] * V(m + 1, a, 0) +
                                 a_i * (V(m, aminus, 0) - eta * ooze * V(m + 1, aminus, 0));
        } else {
            for (int m = 0; m < lim; ++m)
                V(m, aplus, 0) = PA[i] * V(m, a, 0) + WP[i] * V(m + 1, a, 0);
        }
    }
    /* c-build, eq. 6d: src/HGP.jl:204-240 */
    for (int cplus = 1; cplus < nC; ++cplus) {
        int cshell = g_shell_number[cplus];
        int i = g_shift_dir[cplus];
        int c = g_shift_index[cplus][i];
        int cminus = g_shift_index[c][i];
        for (int a = 0; a < nA; ++a) {
            int ashell = g_shell_number[a];
            int lim = mmax - cshell - ashell;
            int aminus = g_shift_index[a][i];
            double c_i = (cminus >= 0) ? 0.5 * ooe * g_ao2m[c][i] : 0.0;
            double a_i = (aminus >= 0) ? 0.5 * ooze * g_ao2m[a][i] : 0.0;
            for (int m = 0; m < lim; ++m) {
                double v = QC[i] * V(m, a, c) + WQ[i] * V(m + 1, a, c);
                if (aminus >= 0) v += a_i * V(m + 1, aminus, c);
                if (cminus >= 0) v += c_i * (V(m, a, cminus) - zeta * ooze * V(m + 1, a, cminus));
                V(m, a, cplus) = v;
            }
        }
    }
#undef V
}

/* HRR on a contracted or primitive [a0|c0] block (the loops of chrr, src/HGP.jl:87-114,
 * identical to hrr, :395-422).  vrr0 is [nao(la+lb)][nao(lc+ld)]; hrrs is
 * [nao(la+lb)][nao(lb)][nao(lc+ld)][nao(ld)] in cumulative AO indices. */
static void hrr_block(int la, int lb, int lc, int ld, const double *A, const double *B,
                      const double *C, const double *D, const double *vrr0, double *hrrs) {
    const int n1 = g_nao[la + lb], n2 = g_nao[lb], n3 = g_nao[lc + ld], n4 = g_nao[ld];
#define H(a, b, c, d) hrrs[(((size_t)(a) * n2 + (b)) * n3 + (c)) * n4 + (d)]
    memset(hrrs, 0, sizeof(double) * (size_t)n1 * n2 * n3 * n4);
    for (int c = 0; c < n3; ++c)
        for (int a = 0; a < n1; ++a) H(a, 0, c, 0) = vrr0[(size_t)a * n3 + c];
    for (int c = 0; c < n3; ++c)
        for (int bplus = 1; bplus < n2; ++bplus) {
            int j = g_shift_dir[bplus];
            int b = g_shift_index[bplus][j];
            int bs = g_shell_number[b];
            int alim = g_nao[la + lb - bs - 1];
            for (int a = 0; a < alim; ++a) {
                int aplus = g_shift_plus[a][j];
                H(a, bplus, c, 0) = H(aplus, b, c, 0) + (A[j] - B[j]) * H(a, b, c, 0);
            }
        }
    for (int dplus = 1; dplus < n4; ++dplus) {
        int j = g_shift_dir[dplus];
        int d = g_shift_index[dplus][j];
        int ds = g_shell_number[d];
        int clim = g_nao[lc + ld - ds - 1];
        for (int c = 0; c < clim; ++c) {
            int cplus = g_shift_plus[c][j];
            for (int b = 0; b < n2; ++b)
                for (int a = 0; a < g_nao[la]; ++a)
                    H(a, b, c, dplus) = H(a, b, cplus, d) + (C[j] - D[j]) * H(a, b, c, d);
        }
    }
#undef H
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
    oracle_vrr(amax, cmax, aexpn, bexpn, cexpn, dexpn, A, B, C, D, prefactor_mode, v);
    hrr_block(la, lb, lc, ld, A, B, C, D, v, hrrs); /* m = 0 slice is the first block */
    free(v);
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

static inline int64_t tri64(int64_t i) { return i * (i + 1) / 2; }
/* 0-based iindex (src/Utils.jl:14-19 minus one). */
int64_t oracle_iindex(int64_t i, int64_t j, int64_t k, int64_t l) {
    int64_t ij = i >= j ? tri64(i) + j : tri64(j) + i;
    int64_t kl = k >= l ? tri64(k) + l : tri64(l) + k;
    return ij >= kl ? tri64(ij) + kl : tri64(kl) + ij;
}
int64_t oracle_npacked(int64_t n) { return n * (n + 1) * (n * n + n + 2) / 8; }

/* ---------------------------------------------------------------- contracted HGP */

typedef struct {
    int nshell;
    const double *xyz; const int *L; const int *nprim; const int *prim_off;
    const double *expn; const double *coef;
    /* derived */
    double *ncoef;  /* coef * radial primitive norm * CGBF norm */
    int *fn_off;    /* first function index of each shell */
    int nbf;
} oracle_basis;

static void basis_prepare(oracle_basis *b) {
    int nprim_tot = 0;
    for (int s = 0; s < b->nshell; ++s)
        if (b->prim_off[s] + b->nprim[s] > nprim_tot) nprim_tot = b->prim_off[s] + b->nprim[s];
    b->ncoef = (double *)malloc(sizeof(double) * (nprim_tot > 0 ? nprim_tot : 1));
    b->fn_off = (int *)malloc(sizeof(int) * (b->nshell + 1));
    int off = 0;
    for (int s = 0; s < b->nshell; ++s) {
        int L = b->L[s], p0 = b->prim_off[s];
        double cn = oracle_cgbf_norm(L, b->nprim[s], b->expn + p0, b->coef + p0);
        for (int p = 0; p < b->nprim[s]; ++p) {
            double a = b->expn[p0 + p];
            b->ncoef[p0 + p] = b->coef[p0 + p] * cn * pow(2 * a / M_PI, 0.75) * pow(4 * a, 0.5 * L);
        }
        b->fn_off[s] = off;
        off += g_ncart[L];
    }
    b->fn_off[b->nshell] = off;
    b->nbf = off;
}
static void basis_release(oracle_basis *b) { free(b->ncoef); free(b->fn_off); }

static double comp_factor(int a) { /* 1/sqrt((2I-1)!!(2J-1)!!(2K-1)!!) */
    return 1.0 / sqrt(dfact2(2 * g_ao2m[a][0] - 1) * dfact2(2 * g_ao2m[a][1] - 1) *
                      dfact2(2 * g_ao2m[a][2] - 1));
}

/* chrr(ash,bsh,csh,dsh) with cvrr, src/HGP.jl:50-116, on normalised coefficients (D3),
 * returning (ab|cd) for the shells' own components, out[ma][mb][mc][md] (D2). */
static void shell_quartet(const oracle_basis *b, int sa, int sb, int sc, int sd, double *out) {
    int la = b->L[sa], lb = b->L[sb], lc = b->L[sc], ld = b->L[sd];
    int amax = la + lb, cmax = lc + ld, mmax = amax + cmax + 1;
    int nA = g_nao[amax], nC = g_nao[cmax];
    const double *A = b->xyz + 3 * sa, *B = b->xyz + 3 * sb, *C = b->xyz + 3 * sc,
                 *D = b->xyz + 3 * sd;
    double *vrrs = (double *)malloc(sizeof(double) * (size_t)mmax * nA * nC);
    double *cvrrs = (double *)calloc((size_t)nA * nC, sizeof(double));
    for (int pd = 0; pd < b->nprim[sd]; ++pd)
        for (int pc = 0; pc < b->nprim[sc]; ++pc)
            for (int pb = 0; pb < b->nprim[sb]; ++pb)
                for (int pa = 0; pa < b->nprim[sa]; ++pa) {
                    int ia = b->prim_off[sa] + pa, ib = b->prim_off[sb] + pb;
                    int ic = b->prim_off[sc] + pc, id = b->prim_off[sd] + pd;
                    oracle_vrr(amax, cmax, b->expn[ia], b->expn[ib], b->expn[ic], b->expn[id],
                               A, B, C, D, 0, vrrs);
                    double cf = b->ncoef[ia] * b->ncoef[ib] * b->ncoef[ic] * b->ncoef[id];
                    for (size_t x = 0; x < (size_t)nA * nC; ++x) cvrrs[x] += cf * vrrs[x];
                }
    size_t nh = oracle_hrr_size(la, lb, lc, ld);
    double *hrrs = (double *)malloc(sizeof(double) * nh);
    hrr_block(la, lb, lc, ld, A, B, C, D, cvrrs, hrrs);
    const int n2 = g_nao[lb], n3 = g_nao[lc + ld], n4 = g_nao[ld];
    int oa = la ? g_nao[la - 1] : 0, ob = lb ? g_nao[lb - 1] : 0;
    int oc = lc ? g_nao[lc - 1] : 0, od = ld ? g_nao[ld - 1] : 0;
    int x = 0;
    for (int ma = 0; ma < g_ncart[la]; ++ma)
        for (int mb = 0; mb < g_ncart[lb]; ++mb)
            for (int mc = 0; mc < g_ncart[lc]; ++mc)
                for (int md = 0; md < g_ncart[ld]; ++md, ++x) {
                    int a = oa + ma, bb = ob + mb, c = oc + mc, d = od + md;
                    out[x] = hrrs[(((size_t)a * n2 + bb) * n3 + c) * n4 + d] * comp_factor(a) *
                             comp_factor(bb) * comp_factor(c) * comp_factor(d);
                }
    free(vrrs); free(cvrrs); free(hrrs);
}

/* Orientation of each shell quartet handed to chrr.  0 (default): the reference's, chrr(I,J,K,L)
 * with I >= J, K >= L, pair(IJ) >= pair(KL) by shell index (src/HGP.jl:27-28).  1: the
 * engine's: in each pair the shell with the larger L is 'a' (ties keep the higher index
 * first), and the pair of higher class (la+lb, then la) is the bra.  The two are the same
 * mathematics; their rounding differs, and HRR accuracy depends strongly on which shell
 * receives the transferred angular momentum. */
static int g_orient = 0;
void oracle_set_orientation(int mode) { g_orient = mode; }
int oracle_get_orientation(void) { return g_orient; }

/* all_twoe_ints_chrr, src/HGP.jl:22-34, with D1-D3 and D5 fixed: every unique shell
 * quartet (I>=J, K>=L, pair(IJ)>=pair(KL)) is computed once and scattered to the 0-based
 * iindex positions.  nthreads > 1 uses OpenMP with a dynamic schedule, the analogue of
 * the reference's Threads.@threads over shell quartets. */
static int64_t eri_packed_hgp_impl(int nshell, const double *xyz, const int *L, const int *nprim,
                                   const int *prim_off, const double *expn, const double *coef,
                                   double *out, int nthreads, int64_t stride);

int oracle_eri_packed_hgp(int nshell, const double *xyz, const int *L, const int *nprim,
                          const int *prim_off, const double *expn, const double *coef,
                          double *out, int nthreads) {
    int64_t r = eri_packed_hgp_impl(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads, 1);
    return r < 0 ? (int)r : 0;
}

/* The same driver over every stride-th shell quartet only (a bounded CPU-baseline sample);
 * returns the number of integrals written, or -1. */
int64_t oracle_eri_packed_hgp_sample(int nshell, const double *xyz, const int *L,
                                     const int *nprim, const int *prim_off, const double *expn,
                                     const double *coef, double *out, int nthreads,
                                     int64_t stride) {
    return eri_packed_hgp_impl(nshell, xyz, L, nprim, prim_off, expn, coef, out, nthreads,
                               stride < 1 ? 1 : stride);
}

static int64_t eri_packed_hgp_impl(int nshell, const double *xyz, const int *L, const int *nprim,
                                   const int *prim_off, const double *expn, const double *coef,
                                   double *out, int nthreads, int64_t stride) {
    oracle_init();
    oracle_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0};
    for (int s = 0; s < nshell; ++s)
        if (L[s] < 0 || L[s] > 3 || nprim[s] < 1) return -1;
    basis_prepare(&b);
    int64_t npair = (int64_t)nshell * (nshell + 1) / 2;
    int64_t nquart = npair * (npair + 1) / 2;
    int *pi = (int *)malloc(sizeof(int) * npair), *pj = (int *)malloc(sizeof(int) * npair);
    for (int i = 0, p = 0; i < nshell; ++i)
        for (int j = 0; j <= i; ++j, ++p) { pi[p] = i; pj[p] = j; }
    int64_t written = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : written)
    {
    double *buf = (double *)malloc(sizeof(double) * 15 * 15 * 15 * 15);
#pragma omp for schedule(dynamic, 64)
    for (int64_t q = 0; q < nquart; q += stride) {
        int64_t p1 = (int64_t)((sqrt(8.0 * (double)q + 1.0) - 1.0) / 2.0);
        while (tri64(p1) > q) --p1;
        while (tri64(p1 + 1) <= q) ++p1;
        int64_t p2 = q - tri64(p1);
        int I = pi[p1], J = pj[p1], K = pi[p2], Lsh = pj[p2];
        if (g_orient == 1) {
            int t;
            if (L[I] < L[J]) { t = I; I = J; J = t; }
            if (L[K] < L[Lsh]) { t = K; K = Lsh; Lsh = t; }
            int sb = L[I] + L[J], sk = L[K] + L[Lsh];
            if (sk > sb || (sk == sb && L[K] > L[I])) {
                t = I; I = K; K = t; t = J; J = Lsh; Lsh = t;
            }
        }
        int na = g_ncart[L[I]], nb = g_ncart[L[J]], nc = g_ncart[L[K]], nd = g_ncart[L[Lsh]];
        shell_quartet(&b, I, J, K, Lsh, buf);
        int x = 0;
        for (int ma = 0; ma < na; ++ma)
            for (int mb = 0; mb < nb; ++mb)
                for (int mc = 0; mc < nc; ++mc)
                    for (int md = 0; md < nd; ++md, ++x) {
                        int64_t i = b.fn_off[I] + ma, j = b.fn_off[J] + mb;
                        int64_t k = b.fn_off[K] + mc, l = b.fn_off[Lsh] + md;
                        if (I == J && i < j) continue;
                        if (K == Lsh && k < l) continue;
                        int64_t ij = i >= j ? tri64(i) + j : tri64(j) + i;
                        int64_t kl = k >= l ? tri64(k) + l : tri64(l) + k;
                        if (p1 == p2 && ij < kl) continue;
                        out[oracle_iindex(i, j, k, l)] = buf[x];
                        ++written;
                    }
    }
    free(buf);
    }
    free(pi); free(pj);
    basis_release(&b);
    return written;
}

/* One contracted, normalised shell quartet (ab|cd), out[ma][mb][mc][md]. */
int oracle_shell_quartet(int nshell, const double *xyz, const int *L, const int *nprim,
                         const int *prim_off, const double *expn, const double *coef,
                         int sa, int sb, int sc, int sd, double *out) {
    oracle_init();
    oracle_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0};
    basis_prepare(&b);
    shell_quartet(&b, sa, sb, sc, sd, out);
    basis_release(&b);
    return 0;
}

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
    oracle_basis b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0};
    for (int s = 0; s < nshell; ++s)
        if (L[s] < 0 || L[s] > 6 || nprim[s] < 1) return -1;
    basis_prepare(&b);
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
            for (int t = 0; t < 4; ++t) s *= comp_factor(fao[f[t]]);
            out[tri64(ij) + kl] = s;
        }
    }
    free(fsh); free(fao);
    basis_release(&b);
    return 0;
}
