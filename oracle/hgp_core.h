/* hgp_core.h -- the HGP restatement of the oracle, generic over the arithmetic type.
 *
 * TEST INFRASTRUCTURE ONLY.  Included by molints_oracle.c twice: with REAL = double (the
 * oracle proper, names d_*) and with REAL = long double (names ld_*), so that the same
 * restated algorithm can be run with a 64-bit mantissa as a near-exact reference for the
 * FP64 parity tests.  Citations refer to MolecularIntegrals.jl as in molints_oracle.c.
 * Expects: REAL, PFX(name), R_EXP, R_SQRT, R_POW, R_PI, BOYS_EXACT(m,T), BOYS_ASYMP(m,T).
 */
/* farray(mmax,T), src/Boys.jl:19-27 with farray_recur :9-17; out[0..mmax-1] = F_0..F_mmax-1. */
static void PFX(farray)(int mmax, REAL T, REAL *out) {
    if (T < g_boys_tmax) {
        out[mmax - 1] = BOYS_EXACT(mmax - 1, T);
        REAL emt = R_EXP(-T);
        for (int m = mmax - 2; m >= 0; --m) out[m] = (2 * T * out[m + 1] + emt) / (2 * m + 1);
        return;
    }
    out[mmax - 1] = BOYS_ASYMP(mmax - 1, T);
    for (int m = mmax - 2; m >= 0; --m) out[m] = T * out[m + 1] / ((REAL)m + (REAL)0.5);
}

/* ---------------------------------------------------------------- HGP VRR / HRR */

static inline REAL PFX(dist2)(const REAL *a, const REAL *b) {
    REAL dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}

/* vrr!(vrrs, amax, cmax, ...), src/HGP.jl:135-242.  vrrs is [mmax][nao(amax)][nao(cmax)]
 * (m fastest in the reference; slowest here -- the layout is internal).
 * prefactor_mode 0: HGP prefactor 2 pi^2.5/(zeta eta R_SQRT(zeta+eta)) (D5 fixed);
 * prefactor_mode 1: the literal src/HGP.jl:150 expression 2 pi^2.5 (zeta+eta)^-3/2. */
static void PFX(vrr)(int amax, int cmax, REAL aexpn, REAL bexpn, REAL cexpn, REAL dexpn,
                const REAL *A, const REAL *B, const REAL *C, const REAL *D,
                int prefactor_mode, REAL *vrrs) {
    oracle_init();
    const int mmax = amax + cmax + 1;
    const int nA = g_nao[amax], nC = g_nao[cmax];
#define V(m, a, c) vrrs[((size_t)(m) * nA + (a)) * nC + (c)]
    memset(vrrs, 0, sizeof(REAL) * (size_t)mmax * nA * nC);
    REAL zeta = aexpn + bexpn, eta = cexpn + dexpn, ze = zeta + eta;
    REAL ooz = 1 / zeta, ooe = 1 / eta, ooze = 1 / ze, oortze = R_SQRT(ooze);
    REAL P[3], Q[3], W[3], PA[3], WP[3], QC[3], WQ[3];
    for (int i = 0; i < 3; ++i) {
        P[i] = (aexpn * A[i] + bexpn * B[i]) * ooz;
        Q[i] = (cexpn * C[i] + dexpn * D[i]) * ooe;
        W[i] = (zeta * P[i] + eta * Q[i]) * ooze;
        PA[i] = P[i] - A[i]; WP[i] = W[i] - P[i]; QC[i] = Q[i] - C[i]; WQ[i] = W[i] - Q[i];
    }
    REAL rab2 = PFX(dist2)(A, B), rcd2 = PFX(dist2)(C, D), rpq2 = PFX(dist2)(P, Q);
    REAL T = zeta * eta * rpq2 * ooze;
    REAL ex = R_EXP(-aexpn * bexpn * rab2 * ooz - cexpn * dexpn * rcd2 * ooe);
    REAL pref = (prefactor_mode == 1) ? 2 * R_PI * R_PI * R_SQRT(R_PI) * ooze * oortze * ex
                                        : 2 * R_PI * R_PI * R_SQRT(R_PI) * ooz * ooe * oortze * ex;
    REAL Fms[64];
    PFX(farray)(mmax, T, Fms);
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
            REAL a_i = 0.5 * ooz * g_ao2m[a][i];
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
            REAL c_i = (cminus >= 0) ? 0.5 * ooe * g_ao2m[c][i] : 0.0;
            REAL a_i = (aminus >= 0) ? 0.5 * ooze * g_ao2m[a][i] : 0.0;
            for (int m = 0; m < lim; ++m) {
                REAL v = QC[i] * V(m, a, c) + WQ[i] * V(m + 1, a, c);
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
static void PFX(hrr_block)(int la, int lb, int lc, int ld, const REAL *A, const REAL *B,
                      const REAL *C, const REAL *D, const REAL *vrr0, REAL *hrrs) {
    const int n1 = g_nao[la + lb], n2 = g_nao[lb], n3 = g_nao[lc + ld], n4 = g_nao[ld];
#define H(a, b, c, d) hrrs[(((size_t)(a) * n2 + (b)) * n3 + (c)) * n4 + (d)]
    memset(hrrs, 0, sizeof(REAL) * (size_t)n1 * n2 * n3 * n4);
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



/* ---------------------------------------------------------------- contracted HGP */

typedef struct {
    int nshell;
    const double *xyz_in; const int *L; const int *nprim; const int *prim_off;
    const double *expn_in; const double *coef;
    /* derived, in REAL */
    REAL *xyz, *expn;
    REAL *ncoef;  /* coef * radial primitive norm * CGBF norm */
    int *fn_off;  /* first function index of each shell */
    int nbf;
} PFX(basis);

/* CGBF norm after the addbf! sequence, src/Basis.jl:73-83 (see oracle_cgbf_norm). */
static REAL PFX(cgbf_norm)(int L, int nprim, const REAL *expn, const double *coef) {
    REAL s = 0;
    for (int i = 0; i < nprim; ++i)
        for (int j = 0; j < nprim; ++j) {
            REAL a = expn[i], b = expn[j];
            s += (REAL)coef[i] * (REAL)coef[j] * R_POW(2 * R_SQRT(a * b) / (a + b), (REAL)L + 1.5);
        }
    return 1 / R_SQRT(s);
}

static void PFX(basis_prepare)(PFX(basis) *b) {
    int nprim_tot = 0;
    for (int s = 0; s < b->nshell; ++s)
        if (b->prim_off[s] + b->nprim[s] > nprim_tot) nprim_tot = b->prim_off[s] + b->nprim[s];
    const size_t np = nprim_tot > 0 ? (size_t)nprim_tot : 1;
    b->ncoef = (REAL *)malloc(sizeof(REAL) * np);
    b->expn = (REAL *)malloc(sizeof(REAL) * np);
    b->xyz = (REAL *)malloc(sizeof(REAL) * (3 * (size_t)b->nshell + 1));
    b->fn_off = (int *)malloc(sizeof(int) * (b->nshell + 1));
    for (int k = 0; k < nprim_tot; ++k) b->expn[k] = b->expn_in[k];
    for (int k = 0; k < 3 * b->nshell; ++k) b->xyz[k] = b->xyz_in[k];
    int off = 0;
    for (int s = 0; s < b->nshell; ++s) {
        int L = b->L[s], p0 = b->prim_off[s];
        REAL cn = PFX(cgbf_norm)(L, b->nprim[s], b->expn + p0, b->coef + p0);
        for (int p = 0; p < b->nprim[s]; ++p) {
            REAL a = b->expn[p0 + p];
            b->ncoef[p0 + p] = (REAL)b->coef[p0 + p] * cn * R_POW(2 * a / R_PI, (REAL)0.75) *
                               R_POW(4 * a, (REAL)0.5 * L);
        }
        b->fn_off[s] = off;
        off += g_ncart[L];
    }
    b->fn_off[b->nshell] = off;
    b->nbf = off;
}
static void PFX(basis_release)(PFX(basis) *b) {
    free(b->ncoef); free(b->fn_off); free(b->expn); free(b->xyz);
}

static REAL PFX(comp_factor)(int a) { /* 1/sqrt((2I-1)!!(2J-1)!!(2K-1)!!) */
    return 1 / R_SQRT((REAL)(dfact2(2 * g_ao2m[a][0] - 1) * dfact2(2 * g_ao2m[a][1] - 1) *
                             dfact2(2 * g_ao2m[a][2] - 1)));
}

/* chrr(ash,bsh,csh,dsh) with cvrr, src/HGP.jl:50-116, on normalised coefficients (D3),
 * returning (ab|cd) for the shells' own components, out[ma][mb][mc][md] (D2). */
static void PFX(shell_quartet)(const PFX(basis) *b, int sa, int sb, int sc, int sd, REAL *out) {
    int la = b->L[sa], lb = b->L[sb], lc = b->L[sc], ld = b->L[sd];
    int amax = la + lb, cmax = lc + ld, mmax = amax + cmax + 1;
    int nA = g_nao[amax], nC = g_nao[cmax];
    const REAL *A = b->xyz + 3 * sa, *B = b->xyz + 3 * sb, *C = b->xyz + 3 * sc,
                 *D = b->xyz + 3 * sd;
    REAL *vrrs = (REAL *)malloc(sizeof(REAL) * (size_t)mmax * nA * nC);
    REAL *cvrrs = (REAL *)calloc((size_t)nA * nC, sizeof(REAL));
    for (int pd = 0; pd < b->nprim[sd]; ++pd)
        for (int pc = 0; pc < b->nprim[sc]; ++pc)
            for (int pb = 0; pb < b->nprim[sb]; ++pb)
                for (int pa = 0; pa < b->nprim[sa]; ++pa) {
                    int ia = b->prim_off[sa] + pa, ib = b->prim_off[sb] + pb;
                    int ic = b->prim_off[sc] + pc, id = b->prim_off[sd] + pd;
                    PFX(vrr)(amax, cmax, b->expn[ia], b->expn[ib], b->expn[ic], b->expn[id],
                               A, B, C, D, 0, vrrs);
                    REAL cf = b->ncoef[ia] * b->ncoef[ib] * b->ncoef[ic] * b->ncoef[id];
                    for (size_t x = 0; x < (size_t)nA * nC; ++x) cvrrs[x] += cf * vrrs[x];
                }
    size_t nh = oracle_hrr_size(la, lb, lc, ld);
    REAL *hrrs = (REAL *)malloc(sizeof(REAL) * nh);
    PFX(hrr_block)(la, lb, lc, ld, A, B, C, D, cvrrs, hrrs);
    const int n2 = g_nao[lb], n3 = g_nao[lc + ld], n4 = g_nao[ld];
    int oa = la ? g_nao[la - 1] : 0, ob = lb ? g_nao[lb - 1] : 0;
    int oc = lc ? g_nao[lc - 1] : 0, od = ld ? g_nao[ld - 1] : 0;
    int x = 0;
    for (int ma = 0; ma < g_ncart[la]; ++ma)
        for (int mb = 0; mb < g_ncart[lb]; ++mb)
            for (int mc = 0; mc < g_ncart[lc]; ++mc)
                for (int md = 0; md < g_ncart[ld]; ++md, ++x) {
                    int a = oa + ma, bb = ob + mb, c = oc + mc, d = od + md;
                    out[x] = hrrs[(((size_t)a * n2 + bb) * n3 + c) * n4 + d] * PFX(comp_factor)(a) *
                             PFX(comp_factor)(bb) * PFX(comp_factor)(c) * PFX(comp_factor)(d);
                }
    free(vrrs); free(cvrrs); free(hrrs);
}

/* all_twoe_ints_chrr, src/HGP.jl:22-34, with D1-D3 and D5 fixed: every unique shell
 * quartet (I>=J, K>=L, pair(IJ)>=pair(KL)) is computed once and scattered to the 0-based
 * iindex positions.  nthreads > 1 uses OpenMP with a dynamic schedule, the analogue of
 * the reference's Threads.@threads over shell quartets. */
static int64_t PFX(eri_packed_hgp_impl)(int nshell, const double *xyz, const int *L,
                                        const int *nprim, const int *prim_off,
                                        const double *expn, const double *coef, double *out,
                                        int nthreads, int64_t stride) {
    oracle_init();
    PFX(basis) b = {nshell, xyz, L, nprim, prim_off, expn, coef, 0, 0, 0, 0, 0};
    for (int s = 0; s < nshell; ++s)
        if (L[s] < 0 || L[s] > 4 || nprim[s] < 1) return -1;  /* shell_indices reach l = 4 */
    PFX(basis_prepare)(&b);
    int64_t npair = (int64_t)nshell * (nshell + 1) / 2;
    int64_t nquart = npair * (npair + 1) / 2;
    int *pi = (int *)malloc(sizeof(int) * npair), *pj = (int *)malloc(sizeof(int) * npair);
    for (int i = 0, p = 0; i < nshell; ++i)
        for (int j = 0; j <= i; ++j, ++p) { pi[p] = i; pj[p] = j; }
    int64_t written = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : written)
    {
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 15 * 15 * 15 * 15);
#pragma omp for schedule(dynamic, 64)
    for (int64_t q = 0; q < nquart; q += stride) {
        int64_t p1 = (int64_t)((sqrt(8.0 * (double)q + 1.0) - 1.0) / 2.0);
        while (tri64(p1) > q) --p1;
        while (tri64(p1 + 1) <= q) ++p1;
        int64_t p2 = q - tri64(p1);
        int I = pi[p1], J = pj[p1], K = pi[p2], Lsh = pj[p2];
        if (g_orient == 1 || g_orient == 2) {
            int t;
            if (g_orient == 2) {
                /* larger L first; equal L, and an f-d pair, put the tighter shell first */
                if (oracle_a_first(&b, J, I)) { t = I; I = J; J = t; }
                if (oracle_a_first(&b, Lsh, K)) { t = K; K = Lsh; Lsh = t; }
            } else {
                if (L[I] < L[J]) { t = I; I = J; J = t; }
                if (L[K] < L[Lsh]) { t = K; K = Lsh; Lsh = t; }
            }
            int sb = L[I] + L[J], sk = L[K] + L[Lsh];
            if (sk > sb || (sk == sb && L[K] > L[I])) {
                t = I; I = K; K = t; t = J; J = Lsh; Lsh = t;
            }
        }
        int na = g_ncart[L[I]], nb = g_ncart[L[J]], nc = g_ncart[L[K]], nd = g_ncart[L[Lsh]];
        PFX(shell_quartet)(&b, I, J, K, Lsh, buf);
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
                        out[oracle_iindex(i, j, k, l)] = (double)buf[x];
                        ++written;
                    }
    }
    free(buf);
    }
    free(pi); free(pj);
    PFX(basis_release)(&b);
    return written;
}

