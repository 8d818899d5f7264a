/*
 * CPU oracle for the pconf hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference's algorithm for the
 * determinant-pair Hamiltonian build and the sparse products of the Davidson
 * loop.  It exists to check the CUDA product path and to time a CPU baseline;
 * nothing in the product library links or calls it.
 *
 * Parity status: the reference is Fortran 2008 + MPI and no Fortran compiler
 * is available, and the reference ships no tests, fixtures or golden outputs.
 * The restatement is therefore checked against independent known answers
 * (exact 3j values, a second-quantisation build of H, dense eigensolves,
 * J^2 eigenvalues) rather than against the reference's own outputs:
 * parity with the reference itself is unpinned.
 *
 * Each function cites the reference routine it follows (paths relative to the
 * pCI source tree).  Index conventions follow the Fortran: m-state indices,
 * orbital indices and determinant indices are 1-based values stored in
 * 0-based C arrays.  Floating-point expressions keep the Fortran evaluation
 * order; build with -ffp-contract=off so no multiply-add is fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int ne, nst, ns, nso, nx, mj, nlx, kbrt;
    int64_t nd;
    int nc;
    const int32_t *iarr;          /* [nd*ne] 1-based m-states, det-major (Iarr(Ne,Nd)) */
    const int32_t *nh, *jz;       /* [nst] */
    const int32_t *nn, *kk, *ll, *jj; /* [ns] */
    const int32_t *ndc;           /* [nc] */
    const double *hint_lut;       /* [nx*nx], entry ind-1 = HintLUT(ind) */
    const double *gaunt_lut;      /* [n_gaunt_lut] = GauntLUT(0:max) */
    int64_t n_gaunt_lut;
    int64_t ngint;
    int r2_is_f64;
    const void *rint2;            /* [ngint*(kbrt?2:1)] */
    const int32_t *iint2, *iint3; /* [ngint] */
    double gj;
    /* FindGint hash, built by orc_build_hash (BuildGintHash) */
    int64_t cap;
    int32_t *hiac, *hibd;
    int64_t *hpos;
    int err;                      /* 1 = missing integral, 2 = m not conserved */
} orc_sys;

/* ---------------------------------------------------------------- hash --- */

/* BuildGintHash, src/integrals.f90:604-632: open addressing, key
 * iac*104729+ibd, capacity the smallest power of two >= 2*Ngint (min 4). */
int orc_build_hash(orc_sys *s)
{
    int64_t cap = 4;
    while (cap < 2 * (s->ngint > 1 ? s->ngint : 1)) cap *= 2;
    s->cap = cap;
    s->hiac = (int32_t *)malloc(sizeof(int32_t) * cap);
    s->hibd = (int32_t *)malloc(sizeof(int32_t) * cap);
    s->hpos = (int64_t *)calloc(cap, sizeof(int64_t));
    if (!s->hiac || !s->hibd || !s->hpos) return -1;
    for (int64_t i = 0; i < s->ngint; i++) {
        int64_t h = (int64_t)s->iint2[i] * 104729LL + (int64_t)s->iint3[i];
        int64_t slot = h % cap;
        if (slot < 0) slot += cap;
        while (s->hpos[slot] != 0) slot = (slot + 1) % cap;
        s->hiac[slot] = s->iint2[i];
        s->hibd[slot] = s->iint3[i];
        s->hpos[slot] = i + 1;
    }
    return 0;
}

void orc_free_hash(orc_sys *s)
{
    free(s->hiac); free(s->hibd); free(s->hpos);
    s->hiac = s->hibd = NULL; s->hpos = NULL;
}

/* FindGint, src/integrals.f90:563-581.  1-based position or 0. */
static int64_t find_gint(const orc_sys *s, int iac, int ibd)
{
    int64_t h = (int64_t)iac * 104729LL + (int64_t)ibd;
    int64_t slot = h % s->cap;
    if (slot < 0) slot += s->cap;
    while (s->hpos[slot] != 0) {
        if (s->hiac[slot] == iac && s->hibd[slot] == ibd) return s->hpos[slot];
        slot = (slot + 1) % s->cap;
    }
    return 0;
}

static double rint2_at(const orc_sys *s, int64_t pos1, int comp)
{
    int64_t stride = s->kbrt ? 2 : 1;
    int64_t i = (pos1 - 1) * stride + comp;
    if (s->r2_is_f64) return ((const double *)s->rint2)[i];
    return (double)((const float *)s->rint2)[i];
}

/* ------------------------------------------------------------ integrals --- */

/* Hint, src/integrals.f90:122-151 (Ksig = 0, C_is = 0). */
double orc_hint(const orc_sys *s, int ia, int ib)
{
    double e = 0.0;
    if (s->jz[ia - 1] == s->jz[ib - 1]) {
        int na = s->nh[ia - 1], nb = s->nh[ib - 1];
        if (s->kk[na - 1] == s->kk[nb - 1]) {
            if (na > nb) { int n = na; na = nb; nb = n; }
            int ind = s->nx * (na - s->nso - 1) + (nb - s->nso);
            e = s->hint_lut[ind - 1];
        }
    }
    return e;
}

/* Gaunt, src/integrals.f90:509-561 (K_gnt /= 1: absent entries give 0). */
double orc_gaunt(const orc_sys *s, int k, double xj1, double xm1, double xj2, double xm2)
{
    double j1 = xj1, j2 = xj2, m1 = xm1, m2 = xm2, x, g = 0.0;
    int is = 1;
    int im = (int)fabs(m2 - m1);
    if (k >= im) {
        if (k == 0) {
            if (j1 == j2) return 1.0 * is;
        } else {
            if (j2 < j1) {
                x = j2; j2 = j1; j1 = x;
                x = m2; m2 = m1; m1 = x;
                if (im != 2 * (im / 2)) is = -is;
            }
            if (m1 <= 0.0) {
                m1 = -m1; m2 = -m2;
                int ij = (int)(k + j1 - j2);
                if (ij != 2 * (ij / 2)) is = -is;
            }
            int ib1 = 2 * s->nlx + 1;
            int ib2 = ib1 * ib1;
            int64_t ind = (int64_t)(ib2 * (ib2 * k + 2 * (ib1 * j1 + j2)) + ib1 * (j1 + m1) + (j2 + m2));
            if (ind >= 0 && ind <= s->n_gaunt_lut - 1) {
                g = s->gaunt_lut[ind];
                return g * is;
            }
        }
    }
    return g * is;
}

/* Gint, src/integrals.f90:153-293 (Ksig < 2, no SMS).  <i1 i2|V|i3 i4>
 * antisymmetrised: the direct term, then the exchange term (i3<->i4) with the
 * opposite sign; each sums Gaunt*Gaunt*R^k over the allowed k. */
double orc_gint(orc_sys *s, int i1, int i2, int i3, int i4)
{
    int l_br = s->kbrt != 0;
    double e = 0.0;
    int is = 1;
    int ia = i1, ib = i2, ic = i3, id = i4;
    for (int ii = 1; ii <= 2; ii++) {
        int ma = s->jz[ia - 1], mb = s->jz[ib - 1], mc = s->jz[ic - 1], md = s->jz[id - 1];
        if (ma + mb != mc + md) { s->err = 2; return 0.0; }
        int na = s->nh[ia - 1], nb = s->nh[ib - 1], nc = s->nh[ic - 1], nd = s->nh[id - 1];
        int la = s->ll[na - 1], lb = s->ll[nb - 1], lc = s->ll[nc - 1], ld = s->ll[nd - 1];
        int i = la + lb + lc + ld;
        int ibr = 0, k;
        if (i == 2 * (i / 2)) {
            int ja = s->jj[na - 1], jb = s->jj[nb - 1], jc = s->jj[nc - 1], jd = s->jj[nd - 1];
            if (na > nc) { k = na; na = nc; nc = k; ibr++; }
            if (nb > nd) { k = nb; nb = nd; nd = k; ibr++; }
            if (na > nb) { k = na; na = nb; nb = k; k = nc; nc = nd; nd = k; }
            if (na == nb && nc > nd) { k = nc; nc = nd; nd = k; }
            ibr = (ibr == 1) ? -1 : 1;
            int iac0 = s->nx * (na - s->nso - 1) + (nc - s->nso);
            int ibd0 = s->nx * (nb - s->nso - 1) + (nd - s->nso);
            int kmin = abs(ja - jc) / 2 + 1;
            k = abs(jb - jd) / 2 + 1;
            if (kmin < k) kmin = k;
            int kmax = (ja + jc) / 2 + 1;
            k = (jb + jd) / 2 + 1;
            if (kmax > k) kmax = k;
            int i_br = la + lc + kmin - 1;
            int is_br = (i_br != 2 * (i_br / 2)) ? ibr : 1;
            for (int k1 = kmin; k1 <= kmax; k1++) {
                k = k1 - 1;
                i = k + la + lc;
                int l_pr = (i == 2 * (i / 2));
                if (l_pr || l_br) {
                    is_br = is_br * ibr;
                    int iac = s->nx * s->nx * k + iac0;
                    int ibd = ibd0;
                    int64_t mi8 = find_gint(s, iac, ibd);
                    if (mi8 == 0) { s->err = 1; return 0.0; }
                    double rabcd = rint2_at(s, mi8, 0);
                    if (l_br) rabcd = rabcd + is_br * rint2_at(s, mi8, 1);
                    double g1 = orc_gaunt(s, k, ja * 0.5, ma * 0.5, jc * 0.5, mc * 0.5);
                    double g2 = orc_gaunt(s, k, jd * 0.5, md * 0.5, jb * 0.5, mb * 0.5);
                    e = e + ((is * g1) * g2) * rabcd;
                }
            }
        }
        k = ic; ic = id; id = k;
        is = -is;
    }
    return e;
}

/* ------------------------------------------------------------------ J^2 --- */

/* Plj, src/formj2.f90:48-67. */
double orc_plj(const orc_sys *s, int ia, int ib)
{
    double t = 0.0;
    int na = s->nh[ia - 1], nb = s->nh[ib - 1];
    if (na == nb) {
        int ma = s->jz[ia - 1], mb = s->jz[ib - 1];
        if (ma == mb + 2) {
            int ja = s->jj[na - 1];
            t = sqrt((double)(ja * (ja + 2) - ma * mb));
        }
    }
    return t;
}

/* F_J2, src/formj2.f90:13-46: J^2 element in units of (2j)^2. */
double orc_f_j2(const orc_sys *s, const int32_t *idet, int is, int nf, int ia, int ic, int ib, int id)
{
    double t = 0.0;
    if (nf == 0) {
        t = (double)(s->mj * s->mj);
        for (int iq = 0; iq < s->ne; iq++) {
            int a = idet[iq];
            int na = s->nh[a - 1], ja = s->jj[na - 1], ma = s->jz[a - 1];
            t = t + (double)(ja * (ja + 2) - ma * ma);
            for (int jq = iq + 1; jq < s->ne; jq++) {
                int b = idet[jq];
                double p1 = orc_plj(s, a, b), p2 = orc_plj(s, b, a);
                t = t - p1 * p1 - p2 * p2;
            }
        }
    } else if (nf == 2) {
        t = is * (orc_plj(s, ia, ic) * orc_plj(s, id, ib) + orc_plj(s, ic, ia) * orc_plj(s, ib, id)
                  - orc_plj(s, ia, id) * orc_plj(s, ic, ib) - orc_plj(s, id, ia) * orc_plj(s, ib, ic));
    }
    return t;
}

/* --------------------------------------------------------- determinants --- */

/* Rspq_phase1 + Rspq_phase2, src/determinants.f90:595-725.  On return nf is
 * the number of differing m-states (3 = "more than two"); for nf = 1, 2 the
 * arrays hold orbital ids: i[1] (det1) / j[1] (det2) the later difference,
 * i[2] / j[2] the earlier one; *is the fermion sign. */
void orc_rspq(const int32_t *id1, const int32_t *id2, int ne, int *is, int *nf, int i[3], int j[3])
{
    int ni = 0, nj = 0;
    *is = 1; *nf = 3;
    i[0] = 1; j[0] = 1; i[1] = j[1] = i[2] = j[2] = 0;
    while (i[0] <= ne && j[0] <= ne) {
        int l1 = id1[i[0] - 1], l2 = id2[j[0] - 1];
        if (l1 == l2) { i[0]++; j[0]++; }
        else if (l1 > l2) {
            if (++nj > 2) return;
            j[2] = j[1]; j[1] = j[0]; j[0]++;
        } else {
            if (++ni > 2) return;
            i[2] = i[1]; i[1] = i[0]; i[0]++;
        }
    }
    if (i[0] > j[0]) {
        *nf = ni;
        switch (ne - j[0]) {
        case 0: j[2] = j[1]; j[1] = ne; break;
        case 1: j[2] = ne - 1; j[1] = ne; break;
        }
    } else {
        *nf = nj;
        switch (ne - i[0]) {
        case 0: i[2] = i[1]; i[1] = ne; break;
        case 1: i[2] = ne - 1; i[1] = ne; break;
        }
    }
    /* phase 2 */
    if (*nf == 1) {
        if (abs(j[1] - i[1]) % 2 == 1) *is = -*is;
        i[1] = id1[i[1] - 1]; j[1] = id2[j[1] - 1];
    } else if (*nf == 2) {
        if (abs(j[1] - i[1]) % 2 == 1) *is = -*is;
        if (abs(j[2] - i[2]) % 2 == 1) *is = -*is;
        i[1] = id1[i[1] - 1]; j[1] = id2[j[1] - 1];
        i[2] = id1[i[2] - 1]; j[2] = id2[j[2] - 1];
    }
}

/* CompD, src/determinants.f90:748-779 on orbital lists. */
int orc_compd(const int32_t *c1, const int32_t *c2, int ne)
{
    int ni = 0, nj = 0, i = 0, j = 0;
    while (i < ne && j < ne) {
        int l1 = c1[i], l2 = c2[j];
        if (l1 == l2) { i++; j++; }
        else if (l1 > l2) { if (++nj > 2) return 3; j++; }
        else { if (++ni > 2) return 3; i++; }
    }
    return ni > nj ? ni : nj;
}

/* get_det_indexes + compare_bit_dets, src/determinants.f90:933-1034: the
 * bit-string path over 32-bit words, kept to compare its phases with Rspq's. */
void orc_bit_compare(const int32_t *b1, const int32_t *b2, int nints, int *ndiffs, int *is,
                     int d1[3], int d2[3])
{
    int nf = 0;
    *ndiffs = -1;
    for (int w = 0; w < nints; w++) {
        if (b1[w] != 0 || b2[w] != 0) {
            nf += __builtin_popcount((uint32_t)(b1[w] ^ b2[w]));
            if (nf >= 6) { *ndiffs = 3; break; }
        }
    }
    if (*ndiffs < 0) *ndiffs = (nf + 1) / 2;
    d1[0] = d1[1] = d1[2] = 0; d2[0] = d2[1] = d2[2] = 0;
    *is = 1;
    if (*ndiffs > 2) return;
    int i1 = 1, j1 = 1, nzb = 0, first = 0, l1[2] = {0, 0}, l2[2] = {0, 0};
    for (int w = 0; w < nints; w++) {
        if (b1[w] == 0 && b2[w] == 0) continue;
        for (int bit = 0; bit < 32; bit++) {
            int bt1 = (b1[w] >> bit) & 1, bt2 = (b2[w] >> bit) & 1;
            if (bt1 || bt2) first = 1;
            if (!bt1 && !bt2) { if (first) nzb++; }
            else if (bt1 != bt2) {
                int pos = 32 * w + bit + 1;
                if (bt1) { i1++; if (i1 <= 3) { d1[i1 - 1] = pos; l1[i1 - 2] = pos - nzb; } }
                if (bt2) { j1++; if (j1 <= 3) { d2[j1 - 1] = pos; l2[j1 - 2] = pos - nzb; } }
                if ((*ndiffs == 1 && i1 == 2 && j1 == 2) || (*ndiffs == 2 && i1 == 3 && j1 == 3)) break;
            }
        }
    }
    if (*ndiffs == 1) {
        if (nzb > 0) { int l = abs(l2[0] - l1[0] - 1); if (l % 2 == 1) *is = -*is; }
    } else if (*ndiffs == 2) {
        int l = abs(l2[0] - l1[0] - nzb % 2);
        if (l % 2 == 1) *is = -*is;
        l = abs(l2[1] - l1[1] - nzb % 2);
        if (l % 2 == 1) *is = -*is;
        int t = d2[1]; d2[1] = d2[2]; d2[2] = t;
        t = d1[1]; d1[1] = d1[2]; d1[2] = t;
    }
}

/* ------------------------------------------------------------- Hmltn --- */

/* Hmltn, src/pconf.F90:1653-1692.  Called with (i2,i1,j2,j1) =
 * (jIndexes(3), iIndexes(3), jIndexes(2), iIndexes(2)). */
double orc_hmltn(orc_sys *s, const int32_t *idet, int is, int nf, int i2, int i1, int j2, int j1)
{
    double t = 0.0;
    if (nf == 2) {
        t = t + orc_gint(s, i2, j2, i1, j1) * is;
        if (s->gj != 0.0) t = t + s->gj * orc_f_j2(s, idet, is, nf, i2, i1, j2, j1);
        else t = t + s->gj * 0.0;
    } else if (nf == 1) {
        for (int iq = 0; iq < s->ne; iq++) {
            int a = idet[iq];
            if (a != j1) t = t + orc_gint(s, j2, a, j1, a) * is;
        }
        t = t + orc_hint(s, j2, j1) * is;
    } else if (nf == 0) {
        for (int iq = 0; iq < s->ne; iq++) {
            int a = idet[iq];
            for (int jq = iq + 1; jq < s->ne; jq++) {
                int b = idet[jq];
                t = t + orc_gint(s, a, b, a, b) * is;
            }
            t = t + orc_hint(s, a, a) * is;
        }
        if (s->gj != 0.0) t = t + s->gj * orc_f_j2(s, idet, is, nf, i2, i1, j2, j1);
    }
    return t;
}

/* Element (n, k) of H, 1-based determinant indices, with its difference count. */
double orc_h_element(orc_sys *s, int64_t n, int64_t k, int *nf_out)
{
    const int32_t *d1 = s->iarr + (n - 1) * s->ne, *d2 = s->iarr + (k - 1) * s->ne;
    int is, nf, ii[3], jj[3];
    orc_rspq(d1, d2, s->ne, &is, &nf, ii, jj);
    *nf_out = nf;
    if (nf > 2) return 0.0;
    return orc_hmltn(s, d1, is, nf, jj[2], ii[2], jj[1], ii[1]);
}

/* ------------------------------------------------------------- FormH --- */

typedef struct { int64_t n, cap; int32_t *col; double *val; } rowbuf;

static void rb_push(rowbuf *b, int32_t c, double v)
{
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 4096;
        b->col = (int32_t *)realloc(b->col, sizeof(int32_t) * b->cap);
        b->val = (double *)realloc(b->val, sizeof(double) * b->cap);
    }
    b->col[b->n] = c; b->val[b->n] = v; b->n++;
}

/* FormH for rows [row_lo, row_hi] (1-based, inclusive), npes = 1 semantics
 * (src/pconf.F90:1227-1290): configuration-level screening with CompD against
 * the first determinant of each configuration block, then Rspq and Hmltn for
 * every k <= n; exact zeros are counted in numzero and not stored.
 *
 * If rowptr/col/val are NULL only the counts are returned: per-row nonzero
 * counts go to row_cnt (length row_hi-row_lo+1).  Otherwise rowptr[0..nrows]
 * (0-based prefix) must already hold the counts' prefix sum and col (1-based)
 * and val are filled.  Returns NumH for the range; *numzero, *hmin,
 * *pairs (candidate pairs with diff <= 2) are accumulated. */
int64_t orc_form_h(orc_sys *s, int64_t row_lo, int64_t row_hi, int64_t *row_cnt,
                   const int64_t *rowptr, int32_t *col, double *val,
                   int64_t *numzero, double *hmin, int64_t *pairs, int nthreads)
{
    int64_t nrows = row_hi - row_lo + 1;
    int64_t *cstart = (int64_t *)malloc(sizeof(int64_t) * (s->nc + 1));
    int32_t *conf = (int32_t *)malloc(sizeof(int32_t) * (size_t)s->nd * s->ne);
    cstart[0] = 0;
    for (int ic = 0; ic < s->nc; ic++) cstart[ic + 1] = cstart[ic] + s->ndc[ic];
    for (int64_t x = 0; x < s->nd * s->ne; x++) conf[x] = s->nh[s->iarr[x] - 1];
    int64_t numh = 0, nz = 0, npairs = 0;
    double hm = INFINITY;
    int err = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(+:numh,nz,npairs) reduction(min:hm) reduction(max:err)
    {
        orc_sys ls = *s;
        ls.err = 0;
#pragma omp for schedule(dynamic, 16)
        for (int64_t r = 0; r < nrows; r++) {
            int64_t n = row_lo + r;
            const int32_t *d1 = s->iarr + (n - 1) * s->ne;
            const int32_t *c1 = conf + (n - 1) * s->ne;
            int64_t cnt = 0, pos = rowptr ? rowptr[r] : 0;
            int64_t k = 0;
            for (int ic = 0; ic < s->nc; ic++) {
                int64_t kx = s->ndc[ic];
                if (k + kx > n) kx = n - k;
                if (kx != 0) {
                    if (orc_compd(c1, conf + k * s->ne, s->ne) > 2) { k += kx; continue; }
                    for (int64_t k1 = 0; k1 < kx; k1++) {
                        k++;
                        const int32_t *d2 = s->iarr + (k - 1) * s->ne;
                        int is, nf, ii[3], jj[3];
                        orc_rspq(d1, d2, s->ne, &is, &nf, ii, jj);
                        if (nf <= 2) {
                            npairs++;
                            double tt = orc_hmltn(&ls, d1, is, nf, jj[2], ii[2], jj[1], ii[1]);
                            if (tt != 0.0) {
                                if (col) { col[pos] = (int32_t)k; val[pos] = tt; pos++; }
                                cnt++;
                                if (tt < hm) hm = tt;
                            } else {
                                nz++;
                            }
                        }
                    }
                }
                if (k >= n) break;
            }
            if (row_cnt) row_cnt[r] = cnt;
            numh += cnt;
        }
        if (ls.err > err) err = ls.err;
    }
    free(cstart); free(conf);
    *numzero += nz;
    if (hm < *hmin) *hmin = hm;
    if (pairs) *pairs += npairs;
    s->err = err;
    return numh;
}

/* FormJ for all rows (npes = 1, src/formj2.f90:120-172): pairs inside each
 * configuration block with diff 0 or 2 and F_J2 /= 0, k <= n.  Same
 * count/fill protocol as orc_form_h over all Nd rows. */
int64_t orc_form_j(orc_sys *s, int64_t *row_cnt, const int64_t *rowptr, int32_t *col, double *val)
{
    int64_t numj = 0, n = 0;
    for (int ic = 0; ic < s->nc; ic++) {
        int64_t ndn = s->ndc[ic];
        for (int64_t n1 = 1; n1 <= ndn; n1++) {
            n++;
            const int32_t *d1 = s->iarr + (n - 1) * s->ne;
            int64_t k = n - n1, cnt = 0, pos = rowptr ? rowptr[n - 1] : 0;
            for (int64_t k1 = 1; k1 <= n1; k1++) {
                k++;
                const int32_t *d2 = s->iarr + (k - 1) * s->ne;
                int is, nf, ii[3], jj[3];
                orc_rspq(d1, d2, s->ne, &is, &nf, ii, jj);
                if (nf == 0 || nf == 2) {
                    double tt = orc_f_j2(s, d1, is, nf, jj[2], ii[2], jj[1], ii[1]);
                    if (tt != 0.0) {
                        if (col) { col[pos] = (int32_t)k; val[pos] = tt; pos++; }
                        cnt++;
                    }
                }
            }
            if (row_cnt) row_cnt[n - 1] = cnt;
            numj += cnt;
        }
    }
    return numj;
}

/* ------------------------------------------------- sparse products --- */

/* Mxmpy, src/davidson.f90:572-647 (npes = 1): y = (H - Hmin I) x for one
 * vector from the lower-triangle CSR, scattering the transpose part.  diag,
 * if non-NULL, receives H_nn - Hmin. */
void orc_mxmpy(int64_t nd, const int64_t *rowptr, const int32_t *col, const double *val,
               double hmin, const double *x, double *y, double *diag)
{
    for (int64_t n = 0; n < nd; n++) y[n] = 0.0;
    for (int64_t n = 1; n <= nd; n++) {
        for (int64_t l = rowptr[n - 1]; l < rowptr[n]; l++) {
            int64_t k = col[l];
            double t = val[l];
            if (n == k) {
                t = t - hmin;
                if (diag) diag[n - 1] = t;
            }
            y[n - 1] = y[n - 1] + t * x[k - 1];
            if (n != k) y[k - 1] = y[k - 1] + t * x[n - 1];
        }
    }
}

/* Mxmpy over a block of nv vectors, x/y column-major [nd, nv]; row-parallel
 * with OpenMP when threads > 1 (the transpose part goes to per-thread
 * buffers that are summed afterwards).  Used by the timed CPU baseline. */
void orc_mxmpy_block(int64_t nd, const int64_t *rowptr, const int32_t *col, const double *val,
                     double hmin, int nv, const double *x, double *y, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    int nt = 1;
#endif
    double *buf = (double *)calloc((size_t)nt * nd * nv, sizeof(double));
#pragma omp parallel
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        double *yb = buf + (size_t)tid * nd * nv;
#pragma omp for schedule(dynamic, 256)
        for (int64_t n = 1; n <= nd; n++) {
            for (int64_t l = rowptr[n - 1]; l < rowptr[n]; l++) {
                int64_t k = col[l];
                double t = val[l];
                if (n == k) t = t - hmin;
                for (int v = 0; v < nv; v++) {
                    yb[(size_t)v * nd + n - 1] += t * x[(size_t)v * nd + k - 1];
                    if (n != k) yb[(size_t)v * nd + k - 1] += t * x[(size_t)v * nd + n - 1];
                }
            }
        }
    }
    for (size_t i = 0; i < (size_t)nd * nv; i++) {
        double a = 0.0;
        for (int t = 0; t < nt; t++) a += buf[(size_t)t * nd * nv + i];
        y[i] = a;
    }
    free(buf);
}

/* Mxmpy (src/davidson.f90:572-647) over a subset of rows, for the timed CPU
 * baseline: rows[0..nrows) (1-based) with their CSR slices rp[nrows+1] into
 * col (1-based) / val, nv vectors column-major [nd, nv].  OpenMP over the
 * rows; the row part goes to the row's own entry, the transpose part is added
 * atomically into the full-length vectors. */
void orc_mxmpy_rows(int64_t nd, int64_t nrows, const int64_t *rows, const int64_t *rp, const int32_t *col,
                    const double *val, int nv, const double *x, double *y, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < nrows; i++) {
        const int64_t n = rows[i];
        for (int64_t l = rp[i]; l < rp[i + 1]; l++) {
            const int64_t k = col[l];
            const double t = val[l];
            for (int v = 0; v < nv; v++) {
                const double a = t * x[(size_t)v * nd + k - 1];
#pragma omp atomic
                y[(size_t)v * nd + n - 1] += a;
                if (n != k) {
                    const double b = t * x[(size_t)v * nd + n - 1];
#pragma omp atomic
                    y[(size_t)v * nd + k - 1] += b;
                }
            }
        }
    }
}

/* J_av, src/formj2.f90:355-387: <x|J^2|x> over rows/cols <= nx, returned as J. */
double orc_j_av(int64_t nd, const int64_t *rowptr, const int32_t *col, const double *val,
                const double *x, int64_t nx)
{
    double xj = 0.0;
    for (int64_t n = 1; n <= nd; n++) {
        if (n > nx) continue;
        for (int64_t l = rowptr[n - 1]; l < rowptr[n]; l++) {
            int64_t k = col[l];
            double t = val[l];
            if (k <= nx) {
                double r = t * x[k - 1] * x[n - 1];
                if (n != k) r = r + r;
                xj = xj + r;
            }
        }
    }
    return 0.5 * (sqrt(1.0 + xj) - 1.0);
}

/* ---------------------------------------------------------------- LSJ --- */

/* Plus_j, src/pconf.F90:3129-3140 (Plj). */
static double orc_plus_j(const orc_sys *s, int ia, int ib)
{
    double t = 0.0;
    int na = s->nh[ia - 1], nb = s->nh[ib - 1];
    if (na == nb) {
        int ma = s->jz[ia - 1], mb = s->jz[ib - 1];
        if (ma == mb + 2) {
            int ja = s->jj[na - 1];
            t = sqrt(ja * (ja + 2) - ma * mb + 0.0);
        }
    }
    return t;
}

/* plus_s, src/pconf.F90:2964-2997. */
static double orc_plus_s(const orc_sys *s, int ia, int ib)
{
    double t = 0.0, ta, tb;
    if (s->jz[ia - 1] != s->jz[ib - 1] + 2) return t;
    int na = s->nh[ia - 1], nb = s->nh[ib - 1];
    if (s->nn[na - 1] != s->nn[nb - 1]) return t;
    if (s->ll[na - 1] != s->ll[nb - 1]) return t;
    int ja = s->jj[na - 1], jb = s->jj[nb - 1], la = s->ll[na - 1], lb = s->ll[nb - 1];
    int msa = 1, mja = s->jz[ia - 1], mjb = s->jz[ib - 1];
    int mla = (mja - msa) / 2;
    if (abs(mla) > la) return t;
    ta = 0.0;
    if (ja == 2 * la + 1) ta = sqrt((ja + mja) / (2.0 * ja));
    if (ja == 2 * la - 1) ta = -sqrt((ja - mja + 2.0) / (2.0 * ja + 4.0));
    tb = 0.0;
    if (jb == 2 * lb + 1) tb = sqrt((jb - mjb) / (2.0 * jb));
    if (jb == 2 * lb - 1) tb = sqrt((jb + mjb + 2.0) / (2.0 * jb + 4.0));
    t = -sqrt(0.5) * ta * tb;
    return t;
}

/* ta / tb factors of plus_l, p0_s, p0_l for spin projection msa. */
static void orc_lsj_tatb(int ja, int la, int mja, int jb, int lb, int mjb, int msa, double *ta, double *tb)
{
    *ta = 0.0;
    *tb = 0.0;
    if (msa == 1) {
        if (ja == 2 * la + 1) *ta = sqrt((ja + mja) / (2.0 * ja));
        if (ja == 2 * la - 1) *ta = -sqrt((ja - mja + 2.0) / (2.0 * ja + 4.0));
        if (jb == 2 * lb + 1) *tb = sqrt((jb + mjb) / (2.0 * jb));
        if (jb == 2 * lb - 1) *tb = -sqrt((jb - mjb + 2.0) / (2.0 * jb + 4.0));
    }
    if (msa == -1) {
        if (ja == 2 * la + 1) *ta = sqrt((ja - mja) / (2.0 * ja));
        if (ja == 2 * la - 1) *ta = sqrt((ja + mja + 2.0) / (2.0 * ja + 4.0));
        if (jb == 2 * lb + 1) *tb = sqrt((jb - mjb) / (2.0 * jb));
        if (jb == 2 * lb - 1) *tb = sqrt((jb + mjb + 2.0) / (2.0 * jb + 4.0));
    }
}

/* plus_l (src/pconf.F90:2999-3042, kind 0), p0_s (3044-3086, kind 1),
 * p0_l (3088-3127, kind 2). */
static double orc_lsj_one(const orc_sys *s, int ia, int ib, int kind)
{
    double t = 0.0, ta, tb;
    int mja = s->jz[ia - 1], mjb = s->jz[ib - 1];
    if (kind == 0 ? (mja != mjb + 2) : (mja != mjb)) return t;
    int na = s->nh[ia - 1], nb = s->nh[ib - 1];
    if (s->nn[na - 1] != s->nn[nb - 1]) return t;
    if (s->ll[na - 1] != s->ll[nb - 1]) return t;
    int ja = s->jj[na - 1], jb = s->jj[nb - 1], la = s->ll[na - 1], lb = s->ll[nb - 1];
    for (int msa = -1; msa <= 1; msa += 2) {
        int mla = (mja - msa) / 2;
        int mlb = kind == 0 ? (mjb - msa) / 2 : mla;
        if (abs(mla) > la) continue;
        if (kind == 0 && abs(mlb) > lb) continue;
        orc_lsj_tatb(ja, la, mja, jb, lb, mjb, msa, &ta, &tb);
        if (kind == 0) t = t - sqrt(0.5 * (lb * (lb + 1.0) - mlb * (mlb + 1.0))) * ta * tb;
        else if (kind == 1) t = t + 0.5 * msa * (ta * tb);
        else t = t + mla * (ta * tb);
    }
    return t;
}

#define PLJ(a, b) orc_plus_j(s, a, b)
#define PLS(a, b) orc_plus_s(s, a, b)
#define PLL(a, b) orc_lsj_one(s, a, b, 0)
#define P0S(a, b) orc_lsj_one(s, a, b, 1)
#define P0L(a, b) orc_lsj_one(s, a, b, 2)

/* lsj_det, src/pconf.F90:2865-2962. */
void orc_lsj_det(const orc_sys *s, const int32_t *d1, const int32_t *d2, double *tj_, double *tl_, double *ts_)
{
    double tj = 0.0, tl = 0.0, ts = 0.0;
    int is, nf, ii[3], jj[3];
    orc_rspq(d1, d2, s->ne, &is, &nf, ii, jj);
    /* Rspq(idet1,idet2,is,nf,i1,j1,i2,j2): i2/j2 the later difference */
    int i1 = ii[2], j1 = jj[2], i2 = ii[1], j2 = jj[1];
    if (nf == 0) {
        tj = s->mj * s->mj;
        for (int iq = 0; iq < s->ne; iq++) {
            int ia = d1[iq], na = s->nh[ia - 1], ja = s->jj[na - 1], la = s->ll[na - 1], ma = s->jz[ia - 1];
            tj = tj + (ja * (ja + 2) - ma * ma);
            ts = ts + 0.75;
            tl = tl + la * (la + 1);
            for (int jq = iq + 1; jq < s->ne; jq++) {
                int ib = d1[jq];
                tj = tj - pow(PLJ(ia, ib), 2) - pow(PLJ(ib, ia), 2);
                ts = ts + 2 * (P0S(ia, ia) * P0S(ib, ib) - pow(P0S(ia, ib), 2));
                ts = ts - 2 * (pow(PLS(ia, ib), 2) + pow(PLS(ib, ia), 2));
                tl = tl + 2 * (P0L(ia, ia) * P0L(ib, ib) - pow(P0L(ia, ib), 2));
                tl = tl - 2 * (pow(PLL(ia, ib), 2) + pow(PLL(ib, ia), 2));
            }
        }
    }
    if (nf == 1) {
        int ia = i2, ib = j2;
        int ka = s->nh[ia - 1], kb = s->nh[ib - 1];
        if (s->nn[ka - 1] == s->nn[kb - 1]) {
            for (int iq = 0; iq < s->ne; iq++) {
                int ic = d1[iq];
                if (ic == i2) continue;
                ts = ts + 2 * (P0S(ia, ib) * P0S(ic, ic) - P0S(ia, ic) * P0S(ib, ic));
                ts = ts - 2 * (PLS(ia, ic) * PLS(ib, ic) + PLS(ic, ia) * PLS(ic, ib));
                tl = tl + 2 * (P0L(ia, ib) * P0L(ic, ic) - P0L(ia, ic) * P0L(ib, ic));
                tl = tl - 2 * (PLL(ia, ic) * PLL(ib, ic) + PLL(ic, ia) * PLL(ic, ib));
            }
            ts = ts * is;
            tl = tl * is;
        }
    }
    if (nf == 2) {
        int ia = i1, ic = j1, ib = i2, id = j2;
        int na = s->nn[s->nh[ia - 1] - 1], nc = s->nn[s->nh[ic - 1] - 1];
        int nb = s->nn[s->nh[ib - 1] - 1], nd = s->nn[s->nh[id - 1] - 1];
        if ((na == nc && nb == nd) || (na == nd && nb == nc)) {
            tj = PLJ(ia, ic) * PLJ(id, ib) + PLJ(ic, ia) * PLJ(ib, id) - PLJ(ia, id) * PLJ(ic, ib) - PLJ(id, ia) * PLJ(ib, ic);
            ts = ts + 2 * (P0S(ia, ic) * P0S(id, ib) - P0S(ia, id) * P0S(ic, ib));
            ts = ts + 2 * (PLS(ia, ic) * PLS(id, ib) + PLS(ic, ia) * PLS(ib, id) - PLS(ia, id) * PLS(ic, ib) -
                           PLS(id, ia) * PLS(ib, ic));
            tl = tl + 2 * (P0L(ia, ic) * P0L(id, ib) - P0L(ia, id) * P0L(ic, ib));
            tl = tl + 2 * (PLL(ia, ic) * PLL(id, ib) + PLL(ic, ia) * PLL(ib, id) - PLL(ia, id) * PLL(ic, ib) -
                           PLL(id, ia) * PLL(ib, ic));
            tj = tj * is;
            ts = ts * is;
            tl = tl * is;
        }
    }
    *tj_ = tj;
    *tl_ = tl * 4;
    *ts_ = ts * 4;
}

/* calcLSJ, src/pconf.F90:2805-2863, for configurations ic_lo..ic_hi
 * (1-based): the sums sum[q*nv + m] (q = J, L, S) of c_n c_k t over the
 * pairs n <= k (doubled for n /= k); X is Nd x nv column-major.  CompNRC
 * compares the non-relativistic orbitals Nh0 (src/determinants.f90:62-82)
 * and CompC the relativistic ones. */
void orc_lsj(const orc_sys *s, const double *X, int nv, int ic_lo, int ic_hi, double *sum)
{
    int ne = s->ne;
    int *nh0 = (int *)malloc(sizeof(int) * (size_t)s->nst);
    for (int i = 0; i < s->nst; i++) {
        int ni = s->nh[i];
        int nrorb = ni > 1 && s->nn[ni - 2] == s->nn[ni - 1] && s->ll[ni - 2] == s->ll[ni - 1];
        nh0[i] = nrorb ? ni - 1 : ni;
    }
    int64_t *start = (int64_t *)malloc(sizeof(int64_t) * ((size_t)s->nc + 1));
    start[0] = 0;
    for (int c = 0; c < s->nc; c++) start[c + 1] = start[c] + s->ndc[c];
    for (int q = 0; q < 3 * nv; q++) sum[q] = 0.0;
    int32_t c1[8], c2[8];
    for (int ic1 = ic_lo; ic1 <= ic_hi; ic1++) {
        int64_t ndn = s->ndc[ic1 - 1], n = start[ic1 - 1];
        for (int64_t n1 = 1; n1 <= ndn; n1++) {
            n++;
            const int32_t *d1 = s->iarr + (n - 1) * ne;
            int64_t k = n - 1;
            for (int ic2 = ic1; ic2 <= s->nc; ic2++) {
                int64_t ndk = s->ndc[ic2 - 1], k1n = ic2 == ic1 ? n1 : 1;
                const int32_t *d2 = s->iarr + k * ne;   /* determinant k + 1 */
                for (int e = 0; e < ne; e++) { c1[e] = nh0[d1[e] - 1]; c2[e] = nh0[d2[e] - 1]; }
                if (orc_compd(c1, c2, ne) > 0) { k += ndk; continue; }
                for (int e = 0; e < ne; e++) { c1[e] = s->nh[d1[e] - 1]; c2[e] = s->nh[d2[e] - 1]; }
                if (orc_compd(c1, c2, ne) > 2) { k += ndk; continue; }
                for (int64_t k1 = k1n; k1 <= ndk; k1++) {
                    k++;
                    double tj, tl, ts;
                    orc_lsj_det(s, d1, s->iarr + (k - 1) * ne, &tj, &tl, &ts);
                    if (tj == 0.0 && tl == 0.0 && ts == 0.0) continue;
                    for (int m = 0; m < nv; m++) {
                        double ckn = X[(int64_t)m * s->nd + n - 1] * X[(int64_t)m * s->nd + k - 1];
                        if (n != k) ckn = 2 * ckn;
                        sum[m] = sum[m] + ckn * tj;
                        sum[nv + m] = sum[nv + m] + ckn * tl;
                        sum[2 * nv + m] = sum[2 * nv + m] + ckn * ts;
                    }
                }
            }
        }
    }
    free(start);
    free(nh0);
}

/* ------------------------------------------------------ density matrix --- */

/* FormDM's density pass, src/pdtm.f90:1254-1310, one vector b (length nd):
 * ro[(j-1)*nst + i-1] = Ro(i, j) over 1-based m-states (Npo = 0). */
void orc_density(const orc_sys *s, const double *b, double trd, double *ro)
{
    int ne = s->ne, nst = s->nst;
    int32_t c1[8], c2[8];
    for (int64_t q = 0; q < (int64_t)nst * nst; q++) ro[q] = 0.0;
    int64_t n = 0;
    for (int ic1 = 1; ic1 <= s->nc; ic1++) {
        int64_t n2 = s->ndc[ic1 - 1];
        for (int64_t n1 = 1; n1 <= n2; n1++) {
            n++;
            double bn = b[n - 1];
            if (!(fabs(bn) > trd)) continue;
            const int32_t *d1 = s->iarr + (n - 1) * ne;
            int64_t k = 0;
            for (int ic2 = 1; ic2 <= ic1; ic2++) {
                int64_t kx = s->ndc[ic2 - 1];
                if (ic1 == ic2) kx = n1;
                const int32_t *d2 = s->iarr + k * ne;
                for (int e = 0; e < ne; e++) { c1[e] = s->nh[d1[e] - 1]; c2[e] = s->nh[d2[e] - 1]; }
                if (orc_compd(c1, c2, ne) > 1) { k += kx; continue; }
                for (int64_t k1 = 1; k1 <= kx; k1++) {
                    k++;
                    double bk = b[k - 1];
                    if (!(fabs(bn * bk) > trd)) continue;
                    int is, nf, ii[3], jj[3];
                    orc_rspq(d1, s->iarr + (k - 1) * ne, ne, &is, &nf, ii, jj);
                    if (nf == 0) {
                        int nn = n == k ? 1 : 2;
                        for (int iq = 0; iq < ne; iq++) {
                            int i1 = d1[iq];
                            ro[(int64_t)(i1 - 1) * nst + i1 - 1] += bn * bk * is * nn;
                        }
                    }
                    if (nf == 1) {
                        int j1 = ii[1], j2 = jj[1];
                        ro[(int64_t)(j2 - 1) * nst + j1 - 1] += bn * bk * is;
                        ro[(int64_t)(j1 - 1) * nst + j2 - 1] = ro[(int64_t)(j2 - 1) * nst + j1 - 1];
                    }
                }
            }
        }
    }
}

/* FormTM's transition density, src/pdtm.f90:1538-1605: final-state vector
 * bf over system f, initial-state bi over system si (same m-states);
 * ro[(j-1)*nst + i-1] = Ro(i, j), i the initial determinant's m-state. */
void orc_transition_density(const orc_sys *si, const orc_sys *f, const double *bi, const double *bf, double trd,
                            double *ro)
{
    int ne = f->ne, nst = f->nst;
    int32_t c1[8], c2[8];
    for (int64_t q = 0; q < (int64_t)nst * nst; q++) ro[q] = 0.0;
    for (int64_t n = 1; n <= f->nd; n++) {                 /* final state */
        double bn = bf[n - 1];
        if (!(fabs(bn) > trd)) continue;
        const int32_t *d2 = f->iarr + (n - 1) * ne;
        int64_t k = 0;
        for (int ic = 1; ic <= si->nc; ic++) {
            int64_t kx = si->ndc[ic - 1];
            const int32_t *d1 = si->iarr + k * ne;
            for (int e = 0; e < ne; e++) { c1[e] = f->nh[d2[e] - 1]; c2[e] = si->nh[d1[e] - 1]; }
            if (orc_compd(c1, c2, ne) > 1) { k += kx; continue; }
            for (int64_t k1 = 1; k1 <= kx; k1++) {
                k++;                                        /* initial state */
                double bk = bi[k - 1];
                if (!(fabs(bk * bn) > trd)) continue;
                const int32_t *dk = si->iarr + (k - 1) * ne;
                int is, nf, ii[3], jj[3];
                orc_rspq(d2, dk, ne, &is, &nf, ii, jj);
                if (nf == 0)
                    for (int iq = 0; iq < ne; iq++) {
                        int i1 = dk[iq];
                        ro[(int64_t)(i1 - 1) * nst + i1 - 1] += bn * bk * is;
                    }
                if (nf == 1) {
                    int j1 = jj[1], j2 = ii[1];                 /* initial, final */
                    ro[(int64_t)(j2 - 1) * nst + j1 - 1] += bn * bk * is;
                }
            }
        }
    }
}
