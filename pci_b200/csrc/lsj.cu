// LSJ and one-particle density matrices of CI vectors.
//
// LSJ: per-level <J^2>, <L^2>, <S^2> of CI vectors in the determinant basis,
// as pconf's lsj / calcLSJ / lsj_det compute them (src/pconf.F90:2672-2962)
// for kLSJ = 1, returned as J, L, S (x = (sqrt(<X^2> + 1) - 1) / 2).
//
// The reference loops over every determinant n and every later determinant k
// whose non-relativistic configuration equals n's (CompNRC = 0) and whose
// relativistic configuration differs by at most two orbitals (CompC <= 2).
// Here the host groups the configurations by their non-relativistic orbital
// multiset once per call, lists the configuration pairs (c1 <= c2) of each
// group with CompD <= 2, and one warp evaluates the determinant pairs of one
// configuration pair: the difference of the two occupation lists (Rspq), the
// one-electron elements of J+, S+, Sz, L+, Lz between m-states, and the
// contributions c_n c_k t (doubled off the diagonal) to every level, summed
// in registers and added to the result once per warp.  Compiled with
// -fmad=false so each pair's terms follow the reference's operation order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "pci_internal.h"

namespace {

constexpr int LSJ_NVC = 8;   // levels per launch

// Device memory released when the scope ends.
struct LsjBuf {
    void *p = nullptr;
    ~LsjBuf() { dev_free(p); }
};

// What lsj_det needs of one m-state.
struct LMs {
    int orb, n, l, j2, m2;
};

__device__ __forceinline__ LMs lms(const uint32_t *msd, const int8_t *orb_n, int a)
{
    const uint32_t w = __ldg(&msd[a]);
    LMs r;
    r.orb = (int)(w & 1023u);
    r.m2 = (int)((w >> 16) & 255u) - 128;
    r.l = (int)((w >> 24) & 15u);
    r.j2 = 2 * (int)((w >> 28) & 15u) + 1;
    r.n = orb_n[r.orb];
    return r;
}

// Plus_j (src/pconf.F90:3129-3140)
__device__ double d_plus_j(const LMs &a, const LMs &b)
{
    double t = 0.0;
    if (a.orb == b.orb && a.m2 == b.m2 + 2) t = sqrt((double)(a.j2 * (a.j2 + 2) - a.m2 * b.m2) + 0.0);
    return t;
}

// The jj -> ls coefficients shared by plus_s, plus_l, p0_s, p0_l for spin
// projection msa (+-1) of m-state a, with the sign convention of the
// reference's "ta" (first) and "tb" (second) factors.
__device__ __forceinline__ double d_ta(int j, int l, int mj, int msa)
{
    double t = 0.0;
    if (msa == 1) {
        if (j == 2 * l + 1) t = sqrt((j + mj) / (2.0 * j));
        if (j == 2 * l - 1) t = -sqrt((j - mj + 2.0) / (2.0 * j + 4.0));
    } else {
        if (j == 2 * l + 1) t = sqrt((j - mj) / (2.0 * j));
        if (j == 2 * l - 1) t = sqrt((j + mj + 2.0) / (2.0 * j + 4.0));
    }
    return t;
}

// plus_s (src/pconf.F90:2964-2997)
__device__ double d_plus_s(const LMs &a, const LMs &b)
{
    if (a.m2 != b.m2 + 2 || a.n != b.n || a.l != b.l) return 0.0;
    const int mla = (a.m2 - 1) / 2;
    if (abs(mla) > a.l) return 0.0;
    const double ta = d_ta(a.j2, a.l, a.m2, 1);
    double tb = 0.0;   // spin down of b
    if (b.j2 == 2 * b.l + 1) tb = sqrt((b.j2 - b.m2) / (2.0 * b.j2));
    if (b.j2 == 2 * b.l - 1) tb = sqrt((b.j2 + b.m2 + 2.0) / (2.0 * b.j2 + 4.0));
    return -sqrt(0.5) * ta * tb;
}

// plus_l (src/pconf.F90:2999-3042)
__device__ double d_plus_l(const LMs &a, const LMs &b)
{
    if (a.m2 != b.m2 + 2 || a.n != b.n || a.l != b.l) return 0.0;
    double t = 0.0;
    for (int msa = -1; msa <= 1; msa += 2) {
        const int mla = (a.m2 - msa) / 2, mlb = (b.m2 - msa) / 2;
        if (abs(mla) > a.l || abs(mlb) > b.l) continue;
        const double ta = d_ta(a.j2, a.l, a.m2, msa), tb = d_ta(b.j2, b.l, b.m2, msa);
        t = t - sqrt(0.5 * (b.l * (b.l + 1.0) - mlb * (mlb + 1.0))) * ta * tb;
    }
    return t;
}

// p0_s (src/pconf.F90:3044-3086) and p0_l (3088-3127): Sz and Lz
template <bool SPIN>
__device__ double d_p0(const LMs &a, const LMs &b)
{
    if (a.m2 != b.m2 || a.n != b.n || a.l != b.l) return 0.0;
    double t = 0.0;
    for (int msa = -1; msa <= 1; msa += 2) {
        const int mla = (a.m2 - msa) / 2;
        if (abs(mla) > a.l) continue;
        const double ta = d_ta(a.j2, a.l, a.m2, msa), tb = d_ta(b.j2, b.l, b.m2, msa);
        if (SPIN) t = t + 0.5 * msa * (ta * tb);
        else t = t + mla * (ta * tb);
    }
    return t;
}

// Difference of two sorted occupation lists as Rspq (src/determinants.f90:
// 499-590) reports it: nf (3 = more than two), the differing m-states
// (i1, i2 of det1 and j1, j2 of det2, earlier then later) and the sign.
template <int NE>
struct LDiff {
    int nf, is, i1, i2, j1, j2;
};

template <int NE>
__device__ __forceinline__ LDiff<NE> l_diff(const uint16_t *d1, const uint16_t *d2)
{
    unsigned ma = 0, mb = 0;
#pragma unroll
    for (int i = 0; i < NE; i++)
#pragma unroll
        for (int j = 0; j < NE; j++)
            if (d1[i] == d2[j]) { ma |= 1u << i; mb |= 1u << j; }
    LDiff<NE> r;
    r.nf = NE - __popc(ma);
    r.is = 1;
    r.i1 = r.i2 = r.j1 = r.j2 = -1;
    if (r.nf == 1 || r.nf == 2) {
        const unsigned ua = (~ma) & ((1u << NE) - 1), ub = (~mb) & ((1u << NE) - 1);
        const int ip1 = __ffs(ua) - 1, jp1 = __ffs(ub) - 1;
        const int ip2 = 31 - __clz(ua), jp2 = 31 - __clz(ub);
        if (r.nf == 1) {
            r.i2 = d1[ip1];
            r.j2 = d2[jp1];
            r.is = ((ip1 + jp1) & 1) ? -1 : 1;
        } else {
            r.i1 = d1[ip1];
            r.j1 = d2[jp1];
            r.i2 = d1[ip2];
            r.j2 = d2[jp2];
            r.is = ((ip1 + jp1 + ip2 + jp2) & 1) ? -1 : 1;
        }
    }
    return r;
}

// lsj_det (src/pconf.F90:2865-2962) for one determinant pair: tj, tl, ts.
template <int NE>
__device__ void d_lsj_det(const uint32_t *msd, const int8_t *orb_n, int mj, const uint16_t *d1, const uint16_t *d2,
                          double &tj, double &tl, double &ts)
{
    tj = 0.0;
    tl = 0.0;
    ts = 0.0;
    const LDiff<NE> df = l_diff<NE>(d1, d2);
    if (df.nf == 0) {
        tj = (double)(mj * mj);
#pragma unroll
        for (int iq = 0; iq < NE; iq++) {
            const LMs a = lms(msd, orb_n, d1[iq]);
            tj = tj + (double)(a.j2 * (a.j2 + 2) - a.m2 * a.m2);
            ts = ts + 0.75;
            tl = tl + (double)(a.l * (a.l + 1));
#pragma unroll
            for (int jq = iq + 1; jq < NE; jq++) {
                const LMs b = lms(msd, orb_n, d1[jq]);
                const double pj1 = d_plus_j(a, b), pj2 = d_plus_j(b, a);
                tj = tj - pj1 * pj1 - pj2 * pj2;
                const double sab = d_p0<true>(a, b);
                ts = ts + 2 * (d_p0<true>(a, a) * d_p0<true>(b, b) - sab * sab);
                const double s1 = d_plus_s(a, b), s2 = d_plus_s(b, a);
                ts = ts - 2 * (s1 * s1 + s2 * s2);
                const double lab = d_p0<false>(a, b);
                tl = tl + 2 * (d_p0<false>(a, a) * d_p0<false>(b, b) - lab * lab);
                const double l1 = d_plus_l(a, b), l2 = d_plus_l(b, a);
                tl = tl - 2 * (l1 * l1 + l2 * l2);
            }
        }
    } else if (df.nf == 1) {
        const LMs a = lms(msd, orb_n, df.i2), b = lms(msd, orb_n, df.j2);
        if (a.n == b.n) {
#pragma unroll
            for (int iq = 0; iq < NE; iq++) {
                if (d1[iq] == df.i2) continue;
                const LMs c = lms(msd, orb_n, d1[iq]);
                ts = ts + 2 * (d_p0<true>(a, b) * d_p0<true>(c, c) - d_p0<true>(a, c) * d_p0<true>(b, c));
                ts = ts - 2 * (d_plus_s(a, c) * d_plus_s(b, c) + d_plus_s(c, a) * d_plus_s(c, b));
                tl = tl + 2 * (d_p0<false>(a, b) * d_p0<false>(c, c) - d_p0<false>(a, c) * d_p0<false>(b, c));
                tl = tl - 2 * (d_plus_l(a, c) * d_plus_l(b, c) + d_plus_l(c, a) * d_plus_l(c, b));
            }
            ts = ts * df.is;
            tl = tl * df.is;
        }
    } else if (df.nf == 2) {
        // ia = i1, ic = j1, ib = i2, id = j2
        const LMs a = lms(msd, orb_n, df.i1), c = lms(msd, orb_n, df.j1);
        const LMs b = lms(msd, orb_n, df.i2), d = lms(msd, orb_n, df.j2);
        if ((a.n == c.n && b.n == d.n) || (a.n == d.n && b.n == c.n)) {
            tj = d_plus_j(a, c) * d_plus_j(d, b) + d_plus_j(c, a) * d_plus_j(b, d) - d_plus_j(a, d) * d_plus_j(c, b) -
                 d_plus_j(d, a) * d_plus_j(b, c);
            ts = ts + 2 * (d_p0<true>(a, c) * d_p0<true>(d, b) - d_p0<true>(a, d) * d_p0<true>(c, b));
            ts = ts + 2 * (d_plus_s(a, c) * d_plus_s(d, b) + d_plus_s(c, a) * d_plus_s(b, d) -
                           d_plus_s(a, d) * d_plus_s(c, b) - d_plus_s(d, a) * d_plus_s(b, c));
            tl = tl + 2 * (d_p0<false>(a, c) * d_p0<false>(d, b) - d_p0<false>(a, d) * d_p0<false>(c, b));
            tl = tl + 2 * (d_plus_l(a, c) * d_plus_l(d, b) + d_plus_l(c, a) * d_plus_l(b, d) -
                           d_plus_l(a, d) * d_plus_l(c, b) - d_plus_l(d, a) * d_plus_l(b, c));
            tj = tj * df.is;
            ts = ts * df.is;
            tl = tl * df.is;
        }
    }
    ts = ts * 4;
    tl = tl * 4;
}

// One warp per configuration pair (c1 <= c2 of one non-relativistic group):
// every determinant pair n <= k, summed into out[q * nv + v] (q = J, L, S)
// for levels v0 .. v0 + LSJ_NVC - 1 (X column-major, leading dimension nd).
template <int NE>
__global__ void __launch_bounds__(128) k_lsj(const uint16_t *__restrict__ occ, const int64_t *__restrict__ conf_start,
                                             const uint32_t *__restrict__ msd, const int8_t *__restrict__ orb_n,
                                             int mj, const int2 *__restrict__ items, int64_t nitems,
                                             const double *__restrict__ X, int64_t nd, int nv, int v0, double *out)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int nvc = min(LSJ_NVC, nv - v0);
    for (int64_t w = warp; w < nitems; w += nwarps) {
        const int2 it = items[w];
        const int64_t n0 = conf_start[it.x], nr = conf_start[it.x + 1] - n0;
        const int64_t k0 = conf_start[it.y], nk = conf_start[it.y + 1] - k0;
        const bool same = it.x == it.y;
        double acc[3][LSJ_NVC];
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int v = 0; v < LSJ_NVC; v++) acc[q][v] = 0.0;
        for (int64_t p = lane; p < nr * nk; p += 32) {
            const int64_t a = p / nk, b = p - a * nk;
            if (same && b < a) continue;
            const int64_t n = n0 + a, k = k0 + b;
            uint16_t d1[NE], d2[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) { d1[e] = occ[n * NE + e]; d2[e] = occ[k * NE + e]; }
            double tj, tl, ts;
            d_lsj_det<NE>(msd, orb_n, mj, d1, d2, tj, tl, ts);
            if (tj == 0.0 && tl == 0.0 && ts == 0.0) continue;
#pragma unroll
            for (int v = 0; v < LSJ_NVC; v++) {
                if (v < nvc) {
                    double ckn = X[(int64_t)(v0 + v) * nd + n] * X[(int64_t)(v0 + v) * nd + k];
                    if (n != k) ckn = 2 * ckn;
                    acc[0][v] = acc[0][v] + ckn * tj;
                    acc[1][v] = acc[1][v] + ckn * tl;
                    acc[2][v] = acc[2][v] + ckn * ts;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 3; q++)
#pragma unroll
            for (int v = 0; v < LSJ_NVC; v++) {
                double s = acc[q][v];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
                if (lane == 0 && v < nvc && s != 0.0) atomicAdd(&out[q * nv + v0 + v], s);
            }
    }
}

// FormDM (src/pdtm.f90:1134-1336): the one-particle density matrix of each
// level over the determinant pairs n >= k whose relativistic configurations
// differ by at most one orbital, both coefficients and their product above
// trd.  One warp per FormH adjacency entry (c1, c2 <= c1, skipped unless
// CompD <= 1); ro[(v * nst + j) * nst + i] = Ro(i, j) (0-based m-states,
// column-major per level).  The reference adds b_n b_k is to Ro(a, b) and
// then sets Ro(b, a) = Ro(a, b), which leaves the running total in both:
// adding the term to both entries gives the same matrix.
template <int NE>
__global__ void __launch_bounds__(128) k_dm(const uint16_t *__restrict__ occ, const int64_t *__restrict__ conf_start,
                                            const uint16_t *__restrict__ conf_orb, const int64_t *__restrict__ adj_ptr,
                                            const int32_t *__restrict__ adj, int nc, const double *__restrict__ X,
                                            int64_t nd, int nv, int nst, double trd, double *ro)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nitems = adj_ptr[nc];
    for (int64_t w = warp; w < nitems; w += nwarps) {
        // row configuration of adjacency entry w (adj_ptr is ascending)
        int lo = 0, hi = nc - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (adj_ptr[mid] <= w) lo = mid; else hi = mid - 1;
        }
        const int c1 = lo, c2 = adj[w];
        uint16_t o1[NE], o2[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) { o1[e] = conf_orb[(int64_t)c1 * NE + e]; o2[e] = conf_orb[(int64_t)c2 * NE + e]; }
        int i = 0, j = 0, ni = 0, nj = 0;
        while (i < NE && j < NE) {
            if (o1[i] == o2[j]) { i++; j++; }
            else if (o1[i] > o2[j]) { nj++; j++; }
            else { ni++; i++; }
        }
        if (max(ni + NE - i, nj + NE - j) > 1) continue;   // CompC > 1
        const int64_t n0 = conf_start[c1], nr = conf_start[c1 + 1] - n0;
        const int64_t k0 = conf_start[c2], nk = conf_start[c2 + 1] - k0;
        for (int64_t p = lane; p < nr * nk; p += 32) {
            const int64_t a = p / nk, b = p - a * nk;
            const int64_t n = n0 + a, k = k0 + b;
            if (k > n) continue;
            uint16_t d1[NE], d2[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) { d1[e] = occ[n * NE + e]; d2[e] = occ[k * NE + e]; }
            const LDiff<NE> df = l_diff<NE>(d1, d2);
            if (df.nf > 1) continue;
            for (int v = 0; v < nv; v++) {
                const double bn = X[(int64_t)v * nd + n], bk = X[(int64_t)v * nd + k];
                if (!(fabs(bn) > trd) || !(fabs(bn * bk) > trd)) continue;
                double *r = ro + (int64_t)v * nst * nst;
                if (df.nf == 0) {
#pragma unroll
                    for (int e = 0; e < NE; e++) atomicAdd(&r[(int64_t)d1[e] * nst + d1[e]], bn * bk);
                } else {
                    const double t = bn * bk * df.is;
                    atomicAdd(&r[(int64_t)df.j2 * nst + df.i2], t);
                    atomicAdd(&r[(int64_t)df.i2 * nst + df.j2], t);
                }
            }
        }
    }
}

// FormTM's transition density (src/pdtm.f90:1538-1605): final-state
// determinants n (basis F) against initial-state determinants k (basis I)
// whose relativistic configurations differ by at most one orbital,
// |b_n| > trd and |b_n b_k| > trd; Rspq takes the final determinant first.
// Equal determinants add b_n b_k to Ro(i, i) for each occupied m-state, one
// differing m-state adds b_n b_k is to Ro(initial's, final's).  One warp per
// final configuration finds the initial configurations within one orbital
// (32 at a time, a ballot of the lanes' CompD), then its lanes take the
// determinant pairs of each.
template <int NE>
__global__ void __launch_bounds__(128) k_tdm(const uint16_t *__restrict__ occ_f, const int64_t *__restrict__ cs_f,
                                             const uint16_t *__restrict__ orb_f, int nc_f,
                                             const uint16_t *__restrict__ occ_i, const int64_t *__restrict__ cs_i,
                                             const uint16_t *__restrict__ orb_i, int nc_i,
                                             const double *__restrict__ bf, const double *__restrict__ bi, int nst,
                                             double trd, double *ro)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t cf = warp; cf < nc_f; cf += nwarps) {
        uint16_t of[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) of[e] = orb_f[cf * NE + e];
        const int64_t n0 = cs_f[cf], nr = cs_f[cf + 1] - n0;
        for (int c0 = 0; c0 < nc_i; c0 += 32) {
            const int ci = c0 + lane;
            bool near = false;
            if (ci < nc_i) {
                int i = 0, j = 0, ni = 0, nj = 0;
                while (i < NE && j < NE) {
                    const uint16_t a = of[i], b = orb_i[(int64_t)ci * NE + j];
                    if (a == b) { i++; j++; }
                    else if (a > b) { nj++; j++; }
                    else { ni++; i++; }
                }
                near = max(ni + NE - i, nj + NE - j) <= 1;
            }
            unsigned m = __ballot_sync(0xffffffffu, near);
            while (m) {
                const int c = c0 + __ffs(m) - 1;
                m &= m - 1;
                const int64_t k0 = cs_i[c], nk = cs_i[c + 1] - k0;
                for (int64_t p = lane; p < nr * nk; p += 32) {
                    const int64_t a = p / nk, b = p - a * nk;
                    const int64_t n = n0 + a, k = k0 + b;
                    const double bn = bf[n], bk = bi[k];
                    if (!(fabs(bn) > trd) || !(fabs(bk * bn) > trd)) continue;
                    uint16_t d2[NE], d1[NE];
#pragma unroll
                    for (int e = 0; e < NE; e++) { d2[e] = occ_f[n * NE + e]; d1[e] = occ_i[k * NE + e]; }
                    const LDiff<NE> df = l_diff<NE>(d2, d1);
                    if (df.nf == 0) {
#pragma unroll
                        for (int e = 0; e < NE; e++) atomicAdd(&ro[(int64_t)d1[e] * nst + d1[e]], bn * bk * df.is);
                    } else if (df.nf == 1) {
                        // Ro(j1, j2): j1 the initial determinant's m-state, j2 the final's
                        atomicAdd(&ro[(int64_t)df.i2 * nst + df.j2], bn * bk * df.is);
                    }
                }
            }
        }
    }
}

template <int NE>
void launch_tdm(int blocks, cudaStream_t st, const pci_gpu *f, const pci_gpu *i, const double *bf, const double *bi,
                double trd, double *ro)
{
    k_tdm<NE><<<blocks, 128, 0, st>>>(f->d_occ, f->d_conf_start, f->d_conf_orb, f->nc, i->d_occ, i->d_conf_start,
                                      i->d_conf_orb, i->nc, bf, bi, f->nst, trd, ro);
}

template <int NE>
void launch_dm(int blocks, cudaStream_t st, const DevSys &S, const int64_t *adj_ptr, const int32_t *adj,
               const double *X, int nv, double trd, double *ro)
{
    k_dm<NE><<<blocks, 128, 0, st>>>(S.occ, S.conf_start, S.conf_orb, adj_ptr, adj, S.nc, X, S.nd, nv, S.nst, trd, ro);
}

template <int NE>
void launch_lsj(int blocks, cudaStream_t st, const DevSys &S, const int8_t *orb_n, const int2 *items, int64_t nitems,
                const double *X, int nv, int v0, double *out)
{
    k_lsj<NE><<<blocks, 128, 0, st>>>(S.occ, S.conf_start, S.msd, orb_n, S.mj, items, nitems, X, S.nd, nv, v0, out);
}

}  // namespace

// Configuration pairs (c1 <= c2) of equal non-relativistic configuration and
// relativistic CompD <= 2, the pairs calcLSJ visits (src/pconf.F90:2805-2863).
// A relativistic orbital that follows one of the same n and l maps to it
// (Nh0, src/determinants.f90:62-82).
static std::vector<int2> lsj_items(const pci_gpu *h, const std::vector<uint16_t> &conf_orb)
{
    const int ne = h->ne, nc = h->nc, nsu = h->nsu;
    std::vector<int> nr(nsu);
    for (int o = 0; o < nsu; o++)
        nr[o] = (o > 0 && h->h_orb_n[o - 1] == h->h_orb_n[o] && h->h_orb_l[o - 1] == h->h_orb_l[o]) ? o - 1 : o;
    std::map<std::vector<int>, std::vector<int>> groups;
    for (int c = 0; c < nc; c++) {
        if (h->h_ndc[c] == 0) continue;
        std::vector<int> key(ne);
        for (int e = 0; e < ne; e++) key[e] = nr[conf_orb[(size_t)c * ne + e]];
        std::sort(key.begin(), key.end());
        groups[key].push_back(c);
    }
    std::vector<int2> items;
    for (const auto &g : groups) {
        const std::vector<int> &cs = g.second;
        for (size_t x = 0; x < cs.size(); x++)
            for (size_t y = x; y < cs.size(); y++) {
                const uint16_t *a = &conf_orb[(size_t)cs[x] * ne], *b = &conf_orb[(size_t)cs[y] * ne];
                int i = 0, j = 0, ni = 0, nj = 0;
                while (i < ne && j < ne) {
                    if (a[i] == b[j]) { i++; j++; }
                    else if (a[i] > b[j]) { nj++; j++; }
                    else { ni++; i++; }
                }
                ni += ne - i;
                nj += ne - j;
                if (std::max(ni, nj) <= 2) items.push_back(make_int2(cs[x], cs[y]));
            }
    }
    return items;
}

extern "C" {

int pci_gpu_lsj(pci_gpu_t *h, const double *X, int32_t nv, double *xj, double *xl, double *xs)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!X || !xj || !xl || !xs) return set_err(h, PCI_E_INPUT, "null array");
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "LSJ before set_basis");
    if ((int)h->h_orb_n.size() != h->nsu) return set_err(h, PCI_E_STATE, "LSJ needs the principal numbers Nn");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "LSJ: nv must be 1..64");
    const int64_t nd = h->nd;
    int rc = 0;
    if (h->lsj_nitems < 0) {
        // the configuration pairs depend on the basis only: built once
        std::vector<uint16_t> conf_orb((size_t)h->nc * h->ne);
        PCI_CUDA(h, cudaMemcpy(conf_orb.data(), h->d_conf_orb, conf_orb.size() * 2, cudaMemcpyDeviceToHost));
        const std::vector<int2> items = lsj_items(h, conf_orb);
        h->d_lsj_items = (int2 *)dev_alloc(h, std::max<size_t>(items.size(), 1) * sizeof(int2), &rc);
        if (rc) return rc;
        PCI_CUDA(h, cudaMemcpy(h->d_lsj_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
        h->lsj_nitems = (int64_t)items.size();
    }
    LsjBuf d_x, d_out;
    d_x.p = dev_alloc(h, (size_t)nd * nv * 8, &rc);
    if (rc) return rc;
    d_out.p = dev_alloc(h, (size_t)3 * nv * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_x.p, X, (size_t)nd * nv * 8, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_out.p, 0, (size_t)3 * nv * 8, h->st));
    const DevSys S = make_devsys(h);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int blocks = nsm * 8;
    const int64_t nit = h->lsj_nitems;
    for (int v0 = 0; v0 < nv && nit > 0; v0 += LSJ_NVC) {
        const int2 *it = h->d_lsj_items;
        const double *x = (const double *)d_x.p;
        double *o = (double *)d_out.p;
        switch (h->ne) {
        case 1: launch_lsj<1>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 2: launch_lsj<2>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 3: launch_lsj<3>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 4: launch_lsj<4>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 5: launch_lsj<5>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 6: launch_lsj<6>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        case 7: launch_lsj<7>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        default: launch_lsj<8>(blocks, h->st, S, h->d_orb_n, it, nit, x, nv, v0, o); break;
        }
        PCI_CUDA(h, cudaGetLastError());
    }
    std::vector<double> sums((size_t)3 * nv);
    PCI_CUDA(h, cudaMemcpyAsync(sums.data(), d_out.p, sums.size() * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    for (int v = 0; v < nv; v++) {
        xj[v] = 0.5 * (sqrt(sums[v] + 1) - 1);
        xl[v] = 0.5 * (sqrt(sums[nv + v] + 1) - 1);
        xs[v] = 0.5 * (sqrt(sums[2 * nv + v] + 1) - 1);
    }
    return PCI_OK;
}

int pci_gpu_transition_density(pci_gpu_t *hi, pci_gpu_t *hf, const double *bi, const double *bf, double trd,
                               double *Ro)
{
    if (!hi || !hf) return PCI_E_INPUT;
    cudaSetDevice(hf->device);
    if (!bi || !bf || !Ro) return set_err(hf, PCI_E_INPUT, "null array");
    if (!hi->have_basis || !hf->have_basis) return set_err(hf, PCI_E_STATE, "transition density before set_basis");
    if (hi->device != hf->device) return set_err(hf, PCI_E_INPUT, "the two bases are on different devices");
    if (hi->ne != hf->ne || hi->nst != hf->nst || hi->h_nh != hf->h_nh || hi->h_jz != hf->h_jz)
        return set_err(hf, PCI_E_INPUT, "the two bases must share Ne and the m-states");
    int rc = 0;
    const int64_t nst = hf->nst;
    LsjBuf d_bi, d_bf, d_ro;
    d_bi.p = dev_alloc(hf, (size_t)hi->nd * 8, &rc);
    if (rc) return rc;
    d_bf.p = dev_alloc(hf, (size_t)hf->nd * 8, &rc);
    if (rc) return rc;
    d_ro.p = dev_alloc(hf, (size_t)nst * nst * 8, &rc);
    if (rc) return rc;
    cudaStream_t st = hf->st;
    PCI_CUDA(hf, cudaStreamSynchronize(hi->st));
    PCI_CUDA(hf, cudaMemcpyAsync(d_bi.p, bi, (size_t)hi->nd * 8, cudaMemcpyHostToDevice, st));
    PCI_CUDA(hf, cudaMemcpyAsync(d_bf.p, bf, (size_t)hf->nd * 8, cudaMemcpyHostToDevice, st));
    PCI_CUDA(hf, cudaMemsetAsync(d_ro.p, 0, (size_t)nst * nst * 8, st));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, hf->device);
    const int blocks = nsm * 8;
    const double *xb = (const double *)d_bf.p, *xa = (const double *)d_bi.p;
    double *r = (double *)d_ro.p;
    switch (hf->ne) {
    case 1: launch_tdm<1>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 2: launch_tdm<2>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 3: launch_tdm<3>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 4: launch_tdm<4>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 5: launch_tdm<5>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 6: launch_tdm<6>(blocks, st, hf, hi, xb, xa, trd, r); break;
    case 7: launch_tdm<7>(blocks, st, hf, hi, xb, xa, trd, r); break;
    default: launch_tdm<8>(blocks, st, hf, hi, xb, xa, trd, r); break;
    }
    PCI_CUDA(hf, cudaGetLastError());
    PCI_CUDA(hf, cudaMemcpyAsync(Ro, d_ro.p, (size_t)nst * nst * 8, cudaMemcpyDeviceToHost, st));
    PCI_CUDA(hf, cudaStreamSynchronize(st));
    return PCI_OK;
}

int pci_gpu_density(pci_gpu_t *h, const double *X, int32_t nv, double trd, double *Ro)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!X || !Ro) return set_err(h, PCI_E_INPUT, "null array");
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "density before set_basis");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "density: nv must be 1..64");
    int rc = 0;
    // FormH's configuration adjacency, in full (a PT block's window lists too few pairs)
    if ((!h->d_adj || h->adj_win_c1 >= 0) && (rc = hb_build_adjacency(h))) return rc;
    const int64_t nd = h->nd, nst = h->nst;
    LsjBuf d_x, d_ro;
    d_x.p = dev_alloc(h, (size_t)nd * nv * 8, &rc);
    if (rc) return rc;
    d_ro.p = dev_alloc(h, (size_t)nst * nst * nv * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_x.p, X, (size_t)nd * nv * 8, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_ro.p, 0, (size_t)nst * nst * nv * 8, h->st));
    const DevSys S = make_devsys(h);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int blocks = nsm * 8;
    const double *x = (const double *)d_x.p;
    double *r = (double *)d_ro.p;
    switch (h->ne) {
    case 1: launch_dm<1>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 2: launch_dm<2>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 3: launch_dm<3>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 4: launch_dm<4>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 5: launch_dm<5>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 6: launch_dm<6>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    case 7: launch_dm<7>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    default: launch_dm<8>(blocks, h->st, S, h->d_adj_ptr, h->d_adj, x, nv, trd, r); break;
    }
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaMemcpyAsync(Ro, d_ro.p, (size_t)nst * nst * nv * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    return PCI_OK;
}

}  // extern "C"
