// Device code of the Hamiltonian / J^2 build, shared by the per-Ne
// translation units (hbuild_ne.cu compiled once per electron count) and the
// host entry points in hbuild.cu.  Compiled with -fmad=false (see hbuild.cu).
#pragma once
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pci_internal.h"

#define FULL_MASK 0xffffffffu

// ------------------------------------------------------------- hashing ---

__host__ __device__ __forceinline__ unsigned long long hmix(unsigned long long x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

__host__ __device__ __forceinline__ unsigned long long hkey(int iac, int ibd)
{
    return ((unsigned long long)(unsigned)iac << 32) | (unsigned long long)(unsigned)ibd;
}

// ------------------------------------------------------- device physics ---

// One hash slot: key and value(s) with one 16-byte load (two with Breit).
__device__ __forceinline__ unsigned long long hslot(const DevSys &S, unsigned long long s, double &v0, double &v1)
{
    const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(S.htab) + s * (S.hw >> 1);
    const ulonglong2 a = __ldg(p);
    v0 = __longlong_as_double((long long)a.y);
    v1 = S.hw == 4 ? __longlong_as_double((long long)__ldg(p + 1).x) : 0.0;
    return a.x;
}

__device__ __forceinline__ double d_lookup(const DevSys &S, int iac, int ibd, int comp)
{
    unsigned long long key = hkey(iac, ibd);
    unsigned long long s = hmix(key) & S.hmask;
    for (int p = 0; p < PCI_MAX_PROBE; p++) {
        double v0, v1;
        const unsigned long long k = hslot(S, s, v0, v1);
        if (k == key) return comp ? v1 : v0;
        if (k == 0ULL) break;
        s = (s + 1) & S.hmask;
    }
    atomicOr(S.err, DERR_MISSING_INTEGRAL);
    return 0.0;
}

// Per-warp cache of the radial integrals one generic configuration tile
// needs, direct-mapped by the key hash; cleared and filled warp-synchronously
// at tile start (one writer per slot), read-only while the tile's pairs are
// evaluated.  A key that lost its slot is looked up in the global table, so
// a collision costs time, never correctness.
constexpr int CACHE_SLOTS_LOG2 = 6;
constexpr int CACHE_SLOTS = 1 << CACHE_SLOTS_LOG2;
struct TileCache {
    unsigned long long key[CACHE_SLOTS];
    double val[CACHE_SLOTS * 2];
};

__device__ __forceinline__ int cache_slot(unsigned long long key)
{
    const unsigned a = (unsigned)(key >> 32), b = (unsigned)key;
    return (int)((a * 0x9E3779B1u + b * 0x85EBCA77u) >> (32 - CACHE_SLOTS_LOG2)) & (CACHE_SLOTS - 1);
}

__device__ __forceinline__ double d_lookup_c(const DevSys &S, const TileCache *tc, int iac, int ibd, int comp)
{
    if (tc) {
        unsigned long long key = hkey(iac, ibd);
        int s = cache_slot(key);
        if (tc->key[s] == key) return tc->val[2 * s + comp];
    }
    return d_lookup(S, iac, ibd, comp);
}

// Term lists of one Gint(a,b,c,d) orbital quadruple: the k values of its
// direct (a,b,c,d) and exchange (a,b,d,c) sums that pass the parity rules, in
// ascending k, with the Gaunt-table block offset k * ntype^2 of each term and
// its radial integral.  Everything Gint sums except the two Gaunt factors
// depends only on the four orbitals, so a tile evaluates every element of a
// quadruple from these lists.
constexpr int KTERMS = 8;
struct QuadTerms {
    int nd, nx;
    int god[KTERMS], gox[KTERMS];
    double rd[KTERMS], rx[KTERMS];
};

// Tile kinds.  TILE_TWO: the configurations differ by two orbitals
// (A0,A1 -> B0,B1), every candidate is an nf = 2 element with orbitals
// (B0,B1,A0,A1), t[0].  TILE_ONE: they differ by one orbital (A0 -> B0); for
// each distinct spectator orbital s (spec[i]) t[2i] serves the nf = 1 terms
// Gint(q,x,p,x) with orbitals (B0,s,A0,s) and t[2i+1] the nf = 2 elements
// with orbitals (sorted(B0,s), sorted(A0,s)).  TILE_GENERIC: per-element
// Gint through the tile cache.
constexpr int TILE_GENERIC = -1, TILE_ONE = 1, TILE_TWO = 2;
constexpr int MAXSPEC = 3;
struct TilePlan {
    int nspec, a0, b0;
    int spec[MAXSPEC];
    QuadTerms t[2 * MAXSPEC];
};

// Packed per-m-state descriptor (built by pci_gpu_set_basis): orbital
// (bits 0-9), (j,m) type of the Gaunt table (10-15), 2m + 128 (16-23),
// l (24-27), (2j-1)/2 (28-31).
struct Ms {
    int orb, type, jz, l, j2;
};

__device__ __forceinline__ Ms ms_get(const DevSys &S, int i)
{
    uint32_t w = __ldg(&S.msd[i]);
    Ms m;
    m.orb = (int)(w & 1023u);
    m.type = (int)((w >> 10) & 63u);
    m.jz = (int)((w >> 16) & 255u) - 128;
    m.l = (int)((w >> 24) & 15u);
    m.j2 = 2 * (int)(w >> 28) + 1;
    return m;
}

// Hint (src/integrals.f90:122-151); m-states are 0-based.
__device__ __forceinline__ double d_hint(const DevSys &S, const Ms &a, const Ms &b)
{
    if (a.jz != b.jz) return 0.0;
    return __ldg(&S.h1[a.orb * S.nsu + b.orb]);
}

__device__ __forceinline__ double d_gaunt(const DevSys &S, int k, int t1, int t2)
{
    return __ldg(&S.gaunt[((size_t)k * S.ntype + t1) * S.ntype + t2]);
}

// Gint (src/integrals.f90:153-293) with Ksig < 2 and no SMS term.  Orbital
// indices are 0-based here, so the 1-based na-Nso-1 of the key becomes oa-Nso.
static __device__ double d_gint(const DevSys &S, const TileCache *cache, const Ms &m1, const Ms &m2, const Ms &m3,
                         const Ms &m4)
{
    const bool l_br = S.kbrt != 0;
    double e = 0.0;
    int is = 1;
#pragma unroll
    for (int ii = 0; ii < 2; ii++) {
        const Ms &A = m1, &B = m2, &Cc = ii ? m4 : m3, &D = ii ? m3 : m4;
        if (A.jz + B.jz != Cc.jz + D.jz) { atomicOr(S.err, DERR_M_NOT_CONSERVED); return 0.0; }
        int na = A.orb, nb = B.orb, nc = Cc.orb, nd = D.orb;
        int la = A.l, lc = Cc.l;
        if (((la + B.l + lc + D.l) & 1) == 0) {
            int ja = A.j2, jb = B.j2, jc = Cc.j2, jd = D.j2;
            int ibr = 0, k;
            if (na > nc) { k = na; na = nc; nc = k; ibr++; }
            if (nb > nd) { k = nb; nb = nd; nd = k; ibr++; }
            if (na > nb) { k = na; na = nb; nb = k; k = nc; nc = nd; nd = k; }
            if (na == nb && nc > nd) { k = nc; nc = nd; nd = k; }
            ibr = (ibr == 1) ? -1 : 1;
            int iac0 = S.nx * (na - S.nso) + (nc + 1 - S.nso);
            int ibd0 = S.nx * (nb - S.nso) + (nd + 1 - S.nso);
            int kmin = max(abs(ja - jc) / 2, abs(jb - jd) / 2);
            int kmax = min((ja + jc) / 2, (jb + jd) / 2);
            int is_br = ((la + lc + kmin) & 1) ? ibr : 1;
            for (k = kmin; k <= kmax; k++) {
                bool l_pr = ((k + la + lc) & 1) == 0;
                if (l_pr || l_br) {
                    is_br = is_br * ibr;
                    int iac = S.nx * S.nx * k + iac0;
                    double rabcd = d_lookup_c(S, cache, iac, ibd0, 0);
                    if (l_br) rabcd = rabcd + is_br * d_lookup_c(S, cache, iac, ibd0, 1);
                    double g1 = d_gaunt(S, k, A.type, Cc.type);
                    double g2 = d_gaunt(S, k, D.type, B.type);
                    e = e + ((is * g1) * g2) * rabcd;
                }
            }
        }
        is = -is;
    }
    return e;
}

// Plj (src/formj2.f90:48-67)
__device__ __forceinline__ double d_plj(const Ms &a, const Ms &b)
{
    if (a.orb == b.orb && a.jz == b.jz + 2) return sqrt((double)(a.j2 * (a.j2 + 2) - a.jz * b.jz));
    return 0.0;
}

// F_J2, nf = 0 (src/formj2.f90:23-38)
template <int NE>
__device__ double d_fj2_diag(const DevSys &S, const uint16_t *d)
{
    double t = (double)(S.mj * S.mj);
#pragma unroll
    for (int iq = 0; iq < NE; iq++) {
        Ms a = ms_get(S, d[iq]);
        t = t + (double)(a.j2 * (a.j2 + 2) - a.jz * a.jz);
#pragma unroll
        for (int jq = iq + 1; jq < NE; jq++) {
            Ms b = ms_get(S, d[jq]);
            double p1 = d_plj(a, b), p2 = d_plj(b, a);
            t = t - p1 * p1 - p2 * p2;
        }
    }
    return t;
}

// F_J2, nf = 2 (src/formj2.f90:39-41), arguments (ia, ic, ib, id)
__device__ __forceinline__ double d_fj2_two(const DevSys &S, int is, int ia, int ic, int ib, int id)
{
    Ms A = ms_get(S, ia), Cc = ms_get(S, ic), B = ms_get(S, ib), D = ms_get(S, id);
    return is * (d_plj(A, Cc) * d_plj(D, B) + d_plj(Cc, A) * d_plj(B, D)
                 - d_plj(A, D) * d_plj(Cc, B) - d_plj(D, A) * d_plj(B, Cc));
}

// Difference of two sorted occupation lists.  Positions of the differing
// m-states are list positions, so the fermion sign of Rspq_phase2
// (src/determinants.f90:709-724), (-1)^(|j2-i2| + |j3-i3|), is the parity of
// the sum of the four positions.
template <int NE>
struct Diff {
    int nf;
    int p1, p2, q1, q2;  // m-states: det1 (row) earlier/later, det2 (column) earlier/later
    int ip1, ip2, jp1, jp2;  // their positions in the two occupation lists
    int is;
};

template <int NE>
__device__ __forceinline__ Diff<NE> d_diff(const uint16_t *d1, const uint16_t *d2)
{
    unsigned ma = 0, mb = 0;
#pragma unroll
    for (int i = 0; i < NE; i++)
#pragma unroll
        for (int j = 0; j < NE; j++)
            if (d1[i] == d2[j]) { ma |= 1u << i; mb |= 1u << j; }
    Diff<NE> r;
    r.nf = NE - __popc(ma);
    r.p1 = r.p2 = r.q1 = r.q2 = -1;
    r.ip1 = r.ip2 = r.jp1 = r.jp2 = 0;
    r.is = 1;
    if (r.nf == 1 || r.nf == 2) {
        unsigned ua = (~ma) & ((1u << NE) - 1), ub = (~mb) & ((1u << NE) - 1);
        int ip1 = __ffs(ua) - 1, jp1 = __ffs(ub) - 1;
        int par = ip1 + jp1;
        r.p1 = d1[ip1];
        r.q1 = d2[jp1];
        r.ip1 = ip1;
        r.jp1 = jp1;
        if (r.nf == 2) {
            int ip2 = 31 - __clz(ua), jp2 = 31 - __clz(ub);
            par += ip2 + jp2;
            r.p2 = d1[ip2];
            r.q2 = d2[jp2];
            r.ip2 = ip2;
            r.jp2 = jp2;
        }
        r.is = (par & 1) ? -1 : 1;
    }
    return r;
}

// Hmltn (src/pconf.F90:1653-1692) as called from FormH with
// (i2, i1, j2, j1) = (jIndexes(3), iIndexes(3), jIndexes(2), iIndexes(2)).
template <int NE>
__device__ double d_hmltn(const DevSys &S, const TileCache *tc, const uint16_t *d1, const Diff<NE> &df)
{
    double t = 0.0;
    if (df.nf == 2) {
        // Gint(i2, j2, i1, j1) = Gint(q1, q2, p1, p2)
        Ms q1 = ms_get(S, df.q1), q2 = ms_get(S, df.q2), p1 = ms_get(S, df.p1), p2 = ms_get(S, df.p2);
        t = t + d_gint(S, tc, q1, q2, p1, p2) * df.is;
        if (S.gj != 0.0) t = t + S.gj * d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
    } else if (df.nf == 1) {
        // j2 = q (det2), j1 = p (det1)
        Ms q = ms_get(S, df.q1), p = ms_get(S, df.p1);
#pragma unroll
        for (int iq = 0; iq < NE; iq++) {
            int a = d1[iq];
            if (a != df.p1) {
                Ms x = ms_get(S, a);
                t = t + d_gint(S, tc, q, x, p, x) * df.is;
            }
        }
        t = t + d_hint(S, q, p) * df.is;
    } else {
        Ms m[NE];
#pragma unroll
        for (int iq = 0; iq < NE; iq++) m[iq] = ms_get(S, d1[iq]);
#pragma unroll
        for (int iq = 0; iq < NE; iq++) {
#pragma unroll
            for (int jq = iq + 1; jq < NE; jq++) t = t + d_gint(S, tc, m[iq], m[jq], m[iq], m[jq]) * 1;
            t = t + d_hint(S, m[iq], m[iq]) * 1;
        }
        if (S.gj != 0.0) t = t + S.gj * d_fj2_diag<NE>(S, d1);
    }
    return t;
}

// ---------------------------------------------------------- adjacency ---

// CompD (src/determinants.f90:748-779) on sorted orbital lists.
template <int NE>
__device__ __forceinline__ int d_compd(const uint16_t *a, const uint16_t *b)
{
    int ni = 0, nj = 0, i = 0, j = 0;
    while (i < NE && j < NE) {
        int l1 = a[i], l2 = b[j];
        if (l1 == l2) { i++; j++; }
        else if (l1 > l2) { if (++nj > 2) return 3; j++; }
        else { if (++ni > 2) return 3; i++; }
    }
    return ni > nj ? ni : nj;
}

// One warp per configuration c1: list c2 <= c1 (non-empty) with CompD <= 2.
// The count pass also records the work of c1 (pairs its rows will visit).
// With a window (w_c1 >= 0) only the rows of configurations w_c1 <= c1 <
// w_c2 get entries, and only c2 < w_c0 and c2 = c1 (conf_pt's rows of the PT
// space against the zero-order space, plus each PT configuration's own
// diagonal block for H_ii); c1 stays the last entry of its list either way.
template <int NE, int FILL>
__global__ void __launch_bounds__(256) k_adjacency(DevSys S, const int32_t *ndc, int64_t *cnt, int32_t *adj,
                                                   unsigned long long *work, int w_c1, int w_c0, int w_c2)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool win = w_c1 >= 0;
    for (int64_t c1 = warp; c1 < S.nc; c1 += nwarps) {
        if (ndc[c1] == 0 || (win && (c1 < w_c1 || c1 >= w_c2))) {
            if (!FILL && lane == 0) { cnt[c1] = 0; work[c1] = 0; }
            continue;
        }
        uint16_t a[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) a[e] = S.conf_orb[c1 * NE + e];
        int64_t base = FILL ? cnt[c1] : 0, c = 0;
        unsigned long long wsum = 0;
        // candidates t < nlo are c2 = t; one more (t = nlo) is c1 itself when the window cuts it off
        const int64_t nlo = (win && w_c0 < c1 + 1) ? (int64_t)w_c0 : c1 + 1;
        const int64_t ncand = nlo + ((win && c1 >= w_c0) ? 1 : 0);
        for (int64_t tb = 0; tb < ncand; tb += 32) {
            const int64_t t = tb + lane;
            const int64_t c2 = t < nlo ? t : c1;
            bool ok = false;
            if (t < ncand && ndc[c2] > 0) {
                uint16_t b[NE];
#pragma unroll
                for (int e = 0; e < NE; e++) b[e] = S.conf_orb[c2 * NE + e];
                ok = d_compd<NE>(a, b) <= 2;
                if (ok) wsum += ndc[c2];
            }
            unsigned m = __ballot_sync(FULL_MASK, ok);
            if (FILL && ok) adj[base + c + __popc(m & ((1u << lane) - 1))] = (int32_t)c2;
            c += __popc(m);
        }
        if (!FILL) {
            for (int o = 16; o > 0; o >>= 1) wsum += __shfl_down_sync(FULL_MASK, wsum, o);
            if (lane == 0) {
                cnt[c1] = c;
                work[c1] = wsum;   // determinant pairs per row of c1
            }
        }
    }
}

template <int NE>
static int adjacency_impl(pci_gpu *h, DevSys S, const int32_t *d_ndc)
{
    int rc = 0;
    int64_t nc = h->nc;
    int64_t *cnt = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) return rc;
    unsigned long long *work = (unsigned long long *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) { dev_free(cnt); return rc; }
    k_adjacency<NE, 0><<<148 * 8, 256, 0, h->st>>>(S, d_ndc, cnt, nullptr, work, h->adj_win_c1, h->adj_win_c0,
                                                   h->adj_win_c2);
    PCI_CUDA(h, cudaGetLastError());
    dev_free(h->d_adj_ptr);
    h->d_adj_ptr = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) { dev_free(cnt); dev_free(work); return rc; }
    PCI_CUDA(h, cudaMemsetAsync(h->d_adj_ptr, 0, 8, h->st));
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, h->d_adj_ptr + 1, nc, h->st);
    if ((rc = ensure_tmp(h, tb))) { dev_free(cnt); dev_free(work); return rc; }
    cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, h->d_adj_ptr + 1, nc, h->st);
    int64_t nadj = 0;
    h->h_rowwork.resize(nc);
    PCI_CUDA(h, cudaMemcpyAsync(h->h_rowwork.data(), work, nc * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(&nadj, h->d_adj_ptr + nc, 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    dev_free(h->d_adj);
    h->d_adj = (int32_t *)dev_alloc(h, std::max<int64_t>(nadj, 1) * 4, &rc);
    if (rc) { dev_free(cnt); dev_free(work); return rc; }
    S.adj_ptr = h->d_adj_ptr;
    k_adjacency<NE, 1><<<148 * 8, 256, 0, h->st>>>(S, d_ndc, h->d_adj_ptr, h->d_adj, nullptr, h->adj_win_c1,
                                                   h->adj_win_c0, h->adj_win_c2);
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    dev_free(cnt);
    dev_free(work);
    h->n_adj = nadj;
    return PCI_OK;
}

// ---------------------------------------------------------- tile cache ---

// Radial keys Gint visits for the argument orbitals (na, nb, nc, nd), both
// terms (direct, then c<->d exchange), exactly as d_gint computes them.
static __device__ int quad_keys(const DevSys &S, int na, int nb, int nc, int nd, unsigned long long *out, int cap)
{
    int n = 0;
    for (int ii = 0; ii < 2; ii++) {
        int a = na, b = nb, c = ii ? nd : nc, d = ii ? nc : nd;
        int la = S.orb_l[a], lb = S.orb_l[b], lc = S.orb_l[c], ld = S.orb_l[d];
        if (((la + lb + lc + ld) & 1) == 0) {
            int ja = S.orb_j[a], jb = S.orb_j[b], jc = S.orb_j[c], jd = S.orb_j[d];
            int k;
            if (a > c) { k = a; a = c; c = k; }
            if (b > d) { k = b; b = d; d = k; }
            if (a > b) { k = a; a = b; b = k; k = c; c = d; d = k; }
            if (a == b && c > d) { k = c; c = d; d = k; }
            int iac0 = S.nx * (a - S.nso) + (c + 1 - S.nso);
            int ibd0 = S.nx * (b - S.nso) + (d + 1 - S.nso);
            int kmin = max(abs(ja - jc) / 2, abs(jb - jd) / 2);
            int kmax = min((ja + jc) / 2, (jb + jd) / 2);
            for (k = kmin; k <= kmax; k++) {
                bool l_pr = ((k + la + lc) & 1) == 0;
                if ((l_pr || S.kbrt) && n < cap) out[n++] = hkey(S.nx * S.nx * k + iac0, ibd0);
            }
        }
    }
    return n;
}

constexpr int TILE_KEYS = 96;

// Warp-synchronous fill of the tile cache for configurations with sorted
// orbital lists o1 (rows) and o2 (columns), CompD(o1, o2) <= 2.  The keys are
// those of every Gint call an element of the tile can make:
//   CompD 2: Gint(q1,q2,p1,p2) with orbitals (b1,b2,a1,a2);
//   CompD 1: Gint(q,x,p,x) and the two-m-state case with a spectator s:
//            orbitals (c,s,a,s) for every spectator orbital s;
//   CompD 0: Gint(x,y,x,y) and same-configuration doubles: (s,t,s,t) for every
//            orbital pair of the configuration.
// Keys that miss the cache fall back to the global table, so a dropped or
// evicted key costs time, never correctness.
// Lane-parallel term lists of one orbital quadruple (a,b,c,d), built by the
// 16 lanes [base, base+16): lanes base..base+7 take the direct sum's k values
// kmin', kmin'+2, ... (kmin' the first k with the parity of la+lc), lanes
// base+8..base+15 the exchange sum's.  Returns (warp-uniformly) false if a
// needed integral is absent or a sum has more than KTERMS terms.
static __device__ bool plan_quad(const DevSys &S, QuadTerms *P, int qa, int qb, int qc, int qd, int base, int lane)
{
    const bool mine = lane >= base && lane < base + 16;
    const int ii = (lane >> 3) & 1, kk = lane & 7;
    int a = qa, b = qb, c = ii ? qd : qc, d = ii ? qc : qd;
    const int la = S.orb_l[a], lb = S.orb_l[b], lc = S.orb_l[c], ld = S.orb_l[d];
    const int ja = S.orb_j[a], jb = S.orb_j[b], jc = S.orb_j[c], jd = S.orb_j[d];
    int t;
    if (a > c) { t = a; a = c; c = t; }
    if (b > d) { t = b; b = d; d = t; }
    if (a > b) { t = a; a = b; b = t; t = c; c = d; d = t; }
    if (a == b && c > d) { t = c; c = d; d = t; }
    const int kmin = max(abs(ja - jc) / 2, abs(jb - jd) / 2);
    const int kmax = min((ja + jc) / 2, (jb + jd) / 2);
    const int k0 = kmin + ((kmin + la + lc) & 1);
    const int k = k0 + 2 * kk;
    const bool par = ((la + lb + lc + ld) & 1) == 0;
    const bool valid = mine && par && k <= kmax;
    bool found = true;
    double r = 0.0;
    if (valid) {
        const unsigned long long key = hkey(S.nx * S.nx * k + S.nx * (a - S.nso) + (c + 1 - S.nso),
                                            S.nx * (b - S.nso) + (d + 1 - S.nso));
        unsigned long long s = hmix(key) & S.hmask;
        found = false;
        for (int p = 0; p < PCI_MAX_PROBE; p++) {
            double v0, v1;
            const unsigned long long kq = hslot(S, s, v0, v1);
            if (kq == key) { r = v0; found = true; break; }
            if (kq == 0ULL) break;
            s = (s + 1) & S.hmask;
        }
    }
    const unsigned vm = __ballot_sync(FULL_MASK, valid);
    const unsigned bad = __ballot_sync(FULL_MASK, (valid && !found) ||
                                                  (mine && par && kk == KTERMS - 1 && k + 2 <= kmax));
    const unsigned grp = 0xffu << (lane & ~7);
    const int pos = __popc(vm & grp & ((1u << lane) - 1));
    if (valid) {
        if (ii == 0) { P->god[pos] = k * S.ntype * S.ntype; P->rd[pos] = r; }
        else { P->gox[pos] = k * S.ntype * S.ntype; P->rx[pos] = r; }
    }
    if (lane == base) {
        P->nd = __popc(vm & (0xffu << base));
        P->nx = __popc(vm & (0xffu << (base + 8)));
    }
    __syncwarp();
    return bad == 0;
}

// Gint(a,b,c,d) of m-states with Gaunt types (ta,tb,tc,td) from the term
// lists of their orbital quadruple, in d_gint's operation order: direct terms
// e + ((1*G(k,ta,tc))*G(k,td,tb))*R, then exchange terms
// e + ((-1*G(k,ta,td))*G(k,tc,tb))*R.  The Gaunt factors of the first four
// terms of both sums are loaded before any is used.
__device__ __forceinline__ double plan_gint(const DevSys &S, const QuadTerms &P, int ta, int tb, int tc, int td)
{
    const int nt = S.ntype;
    const int oac = ta * nt + tc, odb = td * nt + tb, oad = ta * nt + td, ocb = tc * nt + tb;
    const double *G = S.gaunt;
    double a1[4], a2[4], b1[4], b2[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        a1[u] = a2[u] = b1[u] = b2[u] = 0.0;
        if (u < P.nd) { a1[u] = __ldg(G + P.god[u] + oac); a2[u] = __ldg(G + P.god[u] + odb); }
        if (u < P.nx) { b1[u] = __ldg(G + P.gox[u] + oad); b2[u] = __ldg(G + P.gox[u] + ocb); }
    }
    double e = 0.0;
#pragma unroll
    for (int u = 0; u < 4; u++)
        if (u < P.nd) e = e + ((1 * a1[u]) * a2[u]) * P.rd[u];
    for (int i = 4; i < P.nd; i++) {
        const double g1 = __ldg(G + P.god[i] + oac), g2 = __ldg(G + P.god[i] + odb);
        e = e + ((1 * g1) * g2) * P.rd[i];
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
        if (u < P.nx) e = e + ((-1 * b1[u]) * b2[u]) * P.rx[u];
    for (int i = 4; i < P.nx; i++) {
        const double g1 = __ldg(G + P.gox[i] + oad), g2 = __ldg(G + P.gox[i] + ocb);
        e = e + ((-1 * g1) * g2) * P.rx[i];
    }
    return e;
}

// Prepare a tile for configurations with sorted orbital lists o1 (rows) and
// o2 (columns), CompD(o1, o2) <= 2: term lists for two- and one-orbital
// tiles (without the Breit term), otherwise the tile cache holding the keys
// of every Gint call an element of the tile can make:
//   CompD 2: Gint(q1,q2,p1,p2) with orbitals (b1,b2,a1,a2);
//   CompD 1: Gint(q,x,p,x) and the two-m-state case with a spectator s:
//            orbitals (c,s,a,s) for every spectator orbital s;
//   CompD 0: Gint(x,y,x,y) and same-configuration doubles: (s,t,s,t) for every
//            orbital pair of the configuration.
// Returns the tile kind (warp-uniform).
template <int NE>
__device__ int prepare_tile(const DevSys &S, TileCache *tc, TilePlan *plan, unsigned long long *keys,
                            const uint16_t *o1, const uint16_t *o2, int lane)
{
    // multiset differences of the two orbital lists (every lane; NE <= 8)
    int A[NE], B[NE], common[NE], na = 0, nb = 0, ncommon = 0;
    {
        int i = 0, j = 0;
        while (i < NE && j < NE) {
            if (o1[i] == o2[j]) { common[ncommon++] = o1[i]; i++; j++; }
            else if (o1[i] < o2[j]) A[na++] = o1[i++];
            else B[nb++] = o2[j++];
        }
        while (i < NE) A[na++] = o1[i++];
        while (j < NE) B[nb++] = o2[j++];
    }
    if (S.plans && na == 2) {
        if (plan_quad(S, &plan->t[0], B[0], B[1], A[0], A[1], 0, lane)) return TILE_TWO;
    } else if (S.plans && na == 1) {
        int spec[MAXSPEC], ns = 0;
        bool fits = true;
        for (int x = 0; x < ncommon; x++) {
            if (ns > 0 && spec[ns - 1] == common[x]) continue;   // common is sorted
            if (ns == MAXSPEC) { fits = false; break; }
            spec[ns++] = common[x];
        }
        if (fits) {
            const int a0 = A[0], b0 = B[0];
            bool ok = true;
            for (int x = 0; x < ns; x++) {
                // one pass per spectator: lanes 0-15 build the one-m-state lists
                // (B0,s,A0,s), lanes 16-31 the two-m-state lists
                const int sp = spec[x];
                const bool lo = lane < 16;
                const int qa = lo ? b0 : min(b0, sp), qb = lo ? sp : max(b0, sp);
                const int qc = lo ? a0 : min(a0, sp), qd = lo ? sp : max(a0, sp);
                ok = plan_quad(S, &plan->t[2 * x + (lo ? 0 : 1)], qa, qb, qc, qd, lo ? 0 : 16, lane) && ok;
            }
            if (ok) {
                if (lane == 0) {
                    plan->nspec = ns;
                    plan->a0 = a0;
                    plan->b0 = b0;
                    for (int x = 0; x < ns; x++) plan->spec[x] = spec[x];
                }
                __syncwarp();
                return TILE_ONE;
            }
        }
    }
    // generic tile: clear the cache (term lists may have overwritten it), list the keys, fill
    for (int t = lane; t < CACHE_SLOTS; t += 32) tc->key[t] = 0ULL;
    int nkeys = 0;
    if (lane == 0) {
        if (na == 2) {
            nkeys += quad_keys(S, B[0], B[1], A[0], A[1], keys + nkeys, TILE_KEYS - nkeys);
        } else if (na == 1) {
            int prev = -1;
            for (int s = 0; s < ncommon; s++) {
                if (common[s] == prev) continue;
                prev = common[s];
                nkeys += quad_keys(S, B[0], common[s], A[0], common[s], keys + nkeys, TILE_KEYS - nkeys);
            }
        } else if (na == 0) {
            for (int x = 0; x < NE; x++)
                for (int y = x + 1; y < NE; y++) {
                    bool seen = false;
                    for (int x2 = 0; x2 <= x && !seen; x2++)
                        for (int y2 = x2 + 1; y2 < NE && !seen; y2++)
                            if ((x2 < x || y2 < y) && o1[x2] == o1[x] && o1[y2] == o1[y]) seen = true;
                    if (!seen) nkeys += quad_keys(S, o1[x], o1[y], o1[x], o1[y], keys + nkeys, TILE_KEYS - nkeys);
                }
        }
    }
    nkeys = __shfl_sync(FULL_MASK, nkeys, 0);
    __syncwarp();
    for (int base = 0; base < nkeys; base += 32) {
        int idx = base + lane;
        unsigned long long key = idx < nkeys ? keys[idx] : 0ULL;
        int slot = idx < nkeys ? cache_slot(key) : -1 - lane;
        unsigned same = __match_any_sync(FULL_MASK, slot);
        bool writer = idx < nkeys && (__ffs(same) - 1) == lane;
        if (writer) {
            // prefetch only: a key absent from the table is left out of the
            // cache, so the element that needs it reports the missing integral
            unsigned long long s = hmix(key) & S.hmask;
            for (int p = 0; p < PCI_MAX_PROBE; p++) {
                double v0, v1;
                const unsigned long long kk = hslot(S, s, v0, v1);
                if (kk == key) {
                    tc->key[slot] = key;
                    tc->val[2 * slot] = v0;
                    tc->val[2 * slot + 1] = v1;
                    break;
                }
                if (kk == 0ULL) break;
                s = (s + 1) & S.hmask;
            }
        }
        __syncwarp();
    }
    return TILE_GENERIC;
}

// ------------------------------------------------------------ tile pass ---

struct RowStats {
    unsigned long long numzero, pairs, scanned;
    long long hmin_key;  // order-preserving integer image of the minimum value
};

__device__ __forceinline__ long long dkey(double x)
{
    long long b = __double_as_longlong(x);
    return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}

static inline double key_to_double(long long k)
{
    long long b = k >= 0 ? k : (k ^ 0x7fffffffffffffffLL);
    double x;
    memcpy(&x, &b, 8);
    return x;
}

constexpr int TR = 64;   // rows of c1 per chunk
constexpr int TK = 64;   // columns of c2 per chunk
constexpr int WARPS = 8;
// Resident blocks per SM the tile kernel is compiled for (caps registers at
// 65536 / (256 * blocks)).
#ifndef PCI_TILES_MIN_BLOCKS
#define PCI_TILES_MIN_BLOCKS 3
#endif
constexpr int QCAP = 64;

// Per-warp shared memory, occupation lists sized for NE electrons.
template <int NE>
struct WarpSmem {
    union {
        TileCache tc;    // generic tiles
        TilePlan plan;   // one- and two-orbital tiles
    } c;
    int64_t rowbase[TR];
    int64_t rowend[TR];      // end of each row's slots (fill pass)
    int32_t rowcnt[TR];
    uint16_t drow[TR * NE];
    uint16_t orow[TR * NE];  // orbital of each row m-state
    uint8_t trow[TR * NE];   // Gaunt-table type of each row m-state
    union {
        // radial keys of a generic tile: used only while its cache is
        // filled, before its columns are staged
        unsigned long long keys[TILE_KEYS];
        struct {
            uint32_t queue[QCAP];   // candidate pairs (row << 16 | column) in tile order
            uint16_t dcol[TK * NE];
            uint8_t tcol[TK * NE];
        } t;
    } u;
};

struct Tally {
    unsigned long long nzero, npairs, nscan;
    double hmin;
};

// Evaluate the first `cnt` queued pairs (one per lane) and write or count the
// non-zeros.  Rows receive their columns in queue order, which is ascending.
template <int NE, int KIND, int FILL, typename VT>
__device__ __forceinline__ void eval_queue(const DevSys &S, WarpSmem<NE> *ws, int tkind, int cnt,
                                           int64_t rabs0, int64_t kabs0, int32_t *col, VT *val, Tally &ty,
                                           int lane)
{
    const unsigned lt = (1u << lane) - 1;
    int r = TR + lane;
    bool nz = false;
    double v = 0.0;
    int64_t k = 0;
    if (lane < cnt) {
        uint32_t e = ws->u.t.queue[lane];
        r = (int)(e >> 16);
        const int kk = (int)(e & 0xffffu);
        k = kabs0 + kk;
        uint16_t d1[NE], d2[NE];
#pragma unroll
        for (int q = 0; q < NE; q++) { d1[q] = ws->drow[r * NE + q]; d2[q] = ws->u.t.dcol[kk * NE + q]; }
        Diff<NE> df = d_diff<NE>(d1, d2);
        if (KIND == 0) {
            ty.npairs++;
            if (tkind == TILE_TWO) {
                // Gint(q1,q2,p1,p2), orbitals (B0,B1,A0,A1)
                const int tq1 = ws->u.t.tcol[kk * NE + df.jp1], tq2 = ws->u.t.tcol[kk * NE + df.jp2];
                const int tp1 = ws->trow[r * NE + df.ip1], tp2 = ws->trow[r * NE + df.ip2];
                v = 0.0 + plan_gint(S, ws->c.plan.t[0], tq1, tq2, tp1, tp2) * df.is;
                if (S.gj != 0.0) v = v + S.gj * d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
            } else if (tkind == TILE_ONE) {
                const TilePlan &P = ws->c.plan;
                if (df.nf == 2) {
                    // Gint(q1,q2,p1,p2): one electron moved A0 -> B0, one changed m in spectator orbital s
                    const int s2 = ws->orow[r * NE + df.ip1] + ws->orow[r * NE + df.ip2] - P.a0;
                    int x = 0;
                    while (x + 1 < P.nspec && P.spec[x] != s2) x++;
                    const int tq1 = ws->u.t.tcol[kk * NE + df.jp1], tq2 = ws->u.t.tcol[kk * NE + df.jp2];
                    const int tp1 = ws->trow[r * NE + df.ip1], tp2 = ws->trow[r * NE + df.ip2];
                    v = 0.0 + plan_gint(S, P.t[2 * x + 1], tq1, tq2, tp1, tp2) * df.is;
                    if (S.gj != 0.0) v = v + S.gj * d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
                } else {
                    // nf = 1: sum of Gint(q,x,p,x) over the spectators x of det1, then Hint(q,p)
                    const int tq = ws->u.t.tcol[kk * NE + df.jp1], tp = ws->trow[r * NE + df.ip1];
                    double t = 0.0;
#pragma unroll
                    for (int iq = 0; iq < NE; iq++) {
                        if (iq != df.ip1) {
                            const int so = ws->orow[r * NE + iq];
                            int x = 0;
                            while (x + 1 < P.nspec && P.spec[x] != so) x++;
                            const int tx = ws->trow[r * NE + iq];
                            t = t + plan_gint(S, P.t[2 * x], tq, tx, tp, tx) * df.is;
                        }
                    }
                    v = t + d_hint(S, ms_get(S, df.q1), ms_get(S, df.p1)) * df.is;
                }
            } else {
                v = d_hmltn<NE>(S, &ws->c.tc, d1, df);
            }
            if (v != 0.0) nz = true; else ty.nzero++;
        } else {
            v = df.nf == 0 ? d_fj2_diag<NE>(S, d1) : d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
            nz = v != 0.0;
        }
    }
    const unsigned nzm = __ballot_sync(FULL_MASK, nz);
    if (nzm) {
        const unsigned same = __match_any_sync(FULL_MASK, r) & nzm;
        int cur = 0;
        if (nz) cur = ws->rowcnt[r];
        __syncwarp();
        if (nz) {
            VT vs = (VT)v;
            double vd = (double)vs;
            if (vd < ty.hmin) ty.hmin = vd;
            if (FILL) {
                int64_t pos = ws->rowbase[r] + cur + __popc(same & lt);
                if (pos < ws->rowend[r]) {
                    col[pos] = (int32_t)k;
                    val[pos] = vs;
                } else {
                    atomicOr(S.err, DERR_ROW_SLOTS);
                }
            }
            if ((same & lt) == 0) ws->rowcnt[r] = cur + __popc(same);
        }
    }
    __syncwarp();
    (void)rabs0;
}

// One warp per work item (row configuration c1, a chunk of its rows), items
// taken heaviest first.  For each adjacent configuration c2 (ascending) the
// warp fills the tile cache and stages the column determinants; lanes compare
// 32 pairs at a time and push the pairs with difference <= 2 into a FIFO;
// every 32 queued pairs are evaluated together, so the Slater-Condon work
// runs with full warps.  Non-zeros are compacted per row with
// __match_any_sync + __ballot_sync, every row receiving its columns in
// ascending order.
// KIND 0: Hamiltonian; KIND 1: J^2 (diagonal tile only, nf in {0, 2}).
// FILL 0: per-row non-zero counts into rowinfo (values evaluated).
// FILL 1: rowinfo holds each row's first slot; non-zeros are written there
//         and, when rowcnt_out is given, each row's count goes to rowcnt_out.
template <int NE, int KIND, int FILL, typename VT>
__global__ void __launch_bounds__(WARPS * 32, PCI_TILES_MIN_BLOCKS) k_tiles(DevSys S, const int4 *items, int64_t nitems,
                                                      unsigned long long *counter, int64_t *rowinfo, int32_t *col,
                                                      VT *val, RowStats *stats, int64_t *rowcnt_out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31;
    WarpSmem<NE> *ws = reinterpret_cast<WarpSmem<NE> *>(smem_raw) + (threadIdx.x >> 5);
    if (KIND == 0)
        for (int i = lane; i < CACHE_SLOTS; i += 32) ws->c.tc.key[i] = 0ULL;
    __syncwarp();
    Tally ty = {0, 0, 0, INFINITY};
    const unsigned lt = (1u << lane) - 1;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ULL);
        t = __shfl_sync(FULL_MASK, t, 0);
        if (t >= (unsigned long long)nitems) break;
        const int4 it = items[t];
        const int c1 = it.x;
        const int64_t cs1 = S.conf_start[c1];
        const int64_t r0 = cs1 + it.y;
        const int nr = it.z;
        uint16_t o1[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) o1[e] = S.conf_orb[(int64_t)c1 * NE + e];
        const int64_t a0 = KIND == 0 ? S.adj_ptr[c1] : 0, a1 = KIND == 0 ? S.adj_ptr[c1 + 1] : 1;
        for (int rc = 0; rc < nr; rc += TR) {
            const int nrc = min(TR, nr - rc);
            const int64_t rb = r0 + rc;   // absolute index of the chunk's first row
            for (int i = lane; i < nrc * NE; i += 32) {
                const uint16_t m = S.occ[rb * NE + i];
                ws->drow[i] = m;
                const uint32_t w = __ldg(&S.msd[m]);
                ws->trow[i] = (uint8_t)((w >> 10) & 63u);
                ws->orow[i] = (uint16_t)(w & 1023u);
            }
            for (int i = lane; i < nrc; i += 32) {
                ws->rowcnt[i] = 0;
                ws->rowbase[i] = FILL == 1 ? rowinfo[rb + i] : 0;
                ws->rowend[i] = FILL == 1 ? rowinfo[rb + i + 1] : 0;
            }
            __syncwarp();
            for (int64_t a = a0; a < a1; a++) {
                const int c2 = KIND == 0 ? S.adj[a] : c1;
                const int64_t k0 = S.conf_start[c2];
                const int nk = (int)(S.conf_start[c2 + 1] - k0);
                const bool diag = c2 == c1;
                int tkind = TILE_GENERIC;
                if (KIND == 0) {
                    uint16_t o2[NE];
#pragma unroll
                    for (int e = 0; e < NE; e++) o2[e] = S.conf_orb[(int64_t)c2 * NE + e];
                    tkind = prepare_tile<NE>(S, &ws->c.tc, &ws->c.plan, ws->u.keys, o1, o2, lane);
                }
                for (int kc = 0; kc < nk; kc += TK) {
                    const int nkc = min(TK, nk - kc);
                    if (diag && k0 + kc > rb + nrc - 1) break;  // whole chunk above the diagonal
                    __syncwarp();
                    for (int i = lane; i < nkc * NE; i += 32) {
                        const uint16_t m = S.occ[(k0 + kc) * NE + i];
                        ws->u.t.dcol[i] = m;
                        ws->u.t.tcol[i] = (uint8_t)((__ldg(&S.msd[m]) >> 10) & 63u);
                    }
                    __syncwarp();
                    // pair idx = r * nkc + kk, lane + 32 s at step s: (r, kk) advance
                    // by (32 / nkc, 32 % nkc) per step with a carry, no division
                    const int np = nrc * nkc;
                    const int dr = 32 / nkc, dk = 32 - dr * nkc;
                    int r = lane / nkc;
                    int kk = lane - r * nkc;
                    int qn = 0;
                    for (int base = 0; base < np; base += 32) {
                        bool cand = false;
                        if (base + lane < np && !(diag && k0 + kc + kk > rb + r)) {
                            ty.nscan++;
                            uint16_t d1[NE], d2[NE];
#pragma unroll
                            for (int e = 0; e < NE; e++) { d1[e] = ws->drow[r * NE + e]; d2[e] = ws->u.t.dcol[kk * NE + e]; }
                            unsigned ma = 0;
#pragma unroll
                            for (int i = 0; i < NE; i++)
#pragma unroll
                                for (int j = 0; j < NE; j++)
                                    if (d1[i] == d2[j]) ma |= 1u << i;
                            const int nf = NE - __popc(ma);
                            cand = KIND == 0 ? nf <= 2 : (nf == 0 || nf == 2);
                        }
                        const unsigned cm = __ballot_sync(FULL_MASK, cand);
                        if (cand) ws->u.t.queue[qn + __popc(cm & lt)] = ((uint32_t)r << 16) | (uint32_t)kk;
                        qn += __popc(cm);
                        __syncwarp();
                        if (qn >= 32) {
                            eval_queue<NE, KIND, FILL, VT>(S, ws, tkind, 32, rb, k0 + kc, col, val, ty, lane);
                            if (lane < qn - 32) ws->u.t.queue[lane] = ws->u.t.queue[32 + lane];
                            qn -= 32;
                            __syncwarp();
                        }
                        r += dr;
                        kk += dk;
                        if (kk >= nkc) { kk -= nkc; r++; }
                    }
                    if (qn > 0) eval_queue<NE, KIND, FILL, VT>(S, ws, tkind, qn, rb, k0 + kc, col, val, ty, lane);
                }
            }
            __syncwarp();
            if (FILL != 1)
                for (int i = lane; i < nrc; i += 32) rowinfo[rb + i] = ws->rowcnt[i];
            else if (rowcnt_out)
                for (int i = lane; i < nrc; i += 32) rowcnt_out[rb + i] = ws->rowcnt[i];
            __syncwarp();
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ty.nzero += __shfl_down_sync(FULL_MASK, ty.nzero, o);
        ty.npairs += __shfl_down_sync(FULL_MASK, ty.npairs, o);
        ty.nscan += __shfl_down_sync(FULL_MASK, ty.nscan, o);
        ty.hmin = fmin(ty.hmin, __shfl_down_sync(FULL_MASK, ty.hmin, o));
    }
    if (lane == 0 && stats) {
        atomicAdd(&stats->numzero, ty.nzero);
        atomicAdd(&stats->pairs, ty.npairs);
        atomicAdd(&stats->scanned, ty.nscan);
        if (ty.hmin < INFINITY) atomicMin(&stats->hmin_key, dkey(ty.hmin));
    }
}

// ------------------------------------------------------ candidate bound ---

// Pairs of m values (2m units) of two electrons placed in orbitals with 2j =
// j0 and j1 (the same orbital when same: distinct, unordered) whose sum is
// m2.  All 2m values are odd and m2 is even, so the odd members of an
// interval are counted in closed form.
__device__ __forceinline__ int pair_fillings(int j0, int j1, bool same, int m2)
{
    int lo, hi;
    if (!same) {
        lo = max(-j0, m2 - j1);
        hi = min(j0, m2 + j1);
    } else {
        // m0 < m1 = m2 - m0 <= j0
        lo = max(-j0, m2 - j0);
        const int h = m2 / 2;
        hi = (h & 1) ? h - 2 : h - 1;
    }
    return hi >= lo ? (hi - lo) / 2 + 1 : 0;
}

// Upper bound on the candidate pairs (difference <= 2) of every row, from
// the configurations alone.  For a tile whose configurations differ by two
// orbitals, C+{A0,A1} against C+{B0,B1}, with no A or B orbital in C, a
// column determinant is a candidate exactly when it holds the row's
// m-states in C, and then its two electrons in B0, B1 must carry the m of
// the row's two electrons in A0, A1: the count is pair_fillings.  Other
// tiles count every column determinant (the diagonal tile: those up to the
// row).  One lane per row; the next 32 tiles' descriptions are loaded one
// per lane.
template <int NE>
__global__ void __launch_bounds__(256) k_bound(DevSys S, const int4 *items, int64_t nitems, unsigned long long *counter,
                                               int64_t *bound)
{
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ULL);
        t = __shfl_sync(FULL_MASK, t, 0);
        if (t >= (unsigned long long)nitems) break;
        const int4 it = items[t];
        const int c1 = it.x;
        const int64_t cs1 = S.conf_start[c1];
        uint16_t o1[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) o1[e] = S.conf_orb[(int64_t)c1 * NE + e];
        const int64_t a0 = S.adj_ptr[c1], a1 = S.adj_ptr[c1 + 1];
        for (int rp = 0; rp < it.z; rp += 32) {
            const int64_t n = cs1 + it.y + rp + lane;
            const bool mine = rp + lane < it.z;
            int ro[NE], rjz[NE];
#pragma unroll
            for (int e = 0; e < NE; e++) {
                const uint32_t w = mine ? __ldg(&S.msd[S.occ[n * NE + e]]) : 0u;
                ro[e] = (int)(w & 1023u);
                rjz[e] = (int)((w >> 16) & 255u) - 128;
            }
            int64_t cnt = 0;
            for (int64_t ab = a0; ab < a1; ab += 32) {
                const int64_t al = ab + lane;
                int c2l = c1;
                int64_t k0l = 0, k1l = 0;
                uint32_t o2l[(NE + 1) / 2];
#pragma unroll
                for (int e = 0; e < (NE + 1) / 2; e++) o2l[e] = 0u;
                if (al < a1) {
                    c2l = S.adj[al];
                    k0l = S.conf_start[c2l];
                    k1l = S.conf_start[c2l + 1];
#pragma unroll
                    for (int e = 0; e < NE; e++)
                        o2l[e >> 1] |= (uint32_t)S.conf_orb[(int64_t)c2l * NE + e] << (16 * (e & 1));
                }
                const int na = (int)(a1 - ab < 32 ? a1 - ab : 32);
                for (int j = 0; j < na; j++) {
                    const int c2 = __shfl_sync(FULL_MASK, c2l, j);
                    const int64_t k0 = __shfl_sync(FULL_MASK, k0l, j);
                    const int64_t nk = __shfl_sync(FULL_MASK, k1l, j) - k0;
                    if (c2 == c1) {
                        cnt += n - cs1 + 1;
                        continue;
                    }
                    int o2[NE];
#pragma unroll
                    for (int e = 0; e < NE; e++) o2[e] = (int)((__shfl_sync(FULL_MASK, o2l[e >> 1], j) >> (16 * (e & 1))) & 0xffffu);
                    // multiset differences A = c1 - c2, B = c2 - c1 and the common part
                    int A[NE], B[NE], Cm[NE], nA = 0, nB = 0, nC = 0;
                    {
                        int i = 0, k = 0;
                        while (i < NE && k < NE) {
                            if (o1[i] == o2[k]) { Cm[nC++] = o1[i]; i++; k++; }
                            else if (o1[i] < o2[k]) A[nA++] = o1[i++];
                            else B[nB++] = o2[k++];
                        }
                        while (i < NE) A[nA++] = o1[i++];
                        while (k < NE) B[nB++] = o2[k++];
                    }
                    bool typical = nA == 2;
                    for (int x = 0; x < nC && typical; x++)
                        if (Cm[x] == A[0] || Cm[x] == A[1] || Cm[x] == B[0] || Cm[x] == B[1]) typical = false;
                    if (!typical) {
                        cnt += nk;
                        continue;
                    }
                    int m2 = 0;
#pragma unroll
                    for (int e = 0; e < NE; e++)
                        if (ro[e] == A[0] || ro[e] == A[1]) m2 += rjz[e];
                    cnt += pair_fillings(S.orb_j[B[0]], S.orb_j[B[1]], B[0] == B[1], m2);
                }
            }
            if (mine) bound[n] = cnt;
        }
    }
}

// Work items (configuration, first row, row count), heaviest first.  A
// configuration's rows are split so that no item holds much more than
// `target` determinant pairs; for J^2 every configuration is one item.
static inline void make_items(const pci_gpu *h, const std::vector<unsigned long long> &rowwork, int kind, int nwarps,
                       std::vector<int4> &items)
{
    items.clear();
    const int nc = h->nc;
    if (kind == 1) {
        for (int c = 0; c < nc; c++)
            if (h->h_ndc[c] > 0) items.push_back(make_int4(c, 0, h->h_ndc[c], 0));
        return;
    }
    double total = 0.0;
    for (int c = 0; c < nc; c++) total += (double)rowwork[c] * h->h_ndc[c];
    const double target = std::max(1.0, total / (6.0 * nwarps));
    std::vector<std::pair<double, int4>> tmp;
    for (int c = 0; c < nc; c++) {
        int nr = h->h_ndc[c];
        if (nr == 0 || rowwork[c] == 0) continue;   // no pairs: outside a windowed adjacency
        double w = std::max(1.0, (double)rowwork[c]);
        int R = (int)std::max(1.0, std::min((double)TR, std::floor(target / w)));
        for (int r = 0; r < nr; r += R) {
            int cnt = std::min(R, nr - r);
            tmp.push_back({w * cnt, make_int4(c, r, cnt, 0)});
        }
    }
    std::stable_sort(tmp.begin(), tmp.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    items.reserve(tmp.size());
    for (auto &p : tmp) items.push_back(p.second);
}

// Which FormH layout to build: the single-evaluation build (a bound on the
// candidate pairs of each row from the configurations, values evaluated
// once into rows padded to it, then compacted) needs slots for every bound; the two-pass build (count, then
// fill) needs exactly NumH slots but evaluates every value twice.
// PCI_FORMH=exact|padded forces one; by default padded is taken when its
// slots and the compaction buffer fit in free device memory.
static inline int formh_mode_env()
{
    const char *e = getenv("PCI_FORMH");
    if (!e) return -1;
    if (!strcmp(e, "exact")) return 0;
    if (!strcmp(e, "padded")) return 1;
    return -1;
}

// Compaction buffer of the padded build, in entries.
constexpr int64_t COMPACT_CHUNK = 1LL << 24;

// Buffer `which` (0 rowptr, 1 col, 2 val) of the H being built: the retired
// H's buffer when it fits, else a new allocation.
static inline void *csr_buf(pci_gpu *h, int which, size_t bytes, int *rc)
{
    if (void *p = spare_take(h, which, bytes)) {
        *rc = PCI_OK;
        return p;
    }
    return dev_alloc(h, bytes, rc);
}

template <int NE, int KIND>
static int rows_impl(pci_gpu *h, int value_prec, Csr &out, RowStats *hs)
{
    int rc = 0;
    DevSys S = make_devsys(h);
    const int64_t nd = h->nd;
    const int vb = value_prec == 32 ? 4 : 8;
    if (KIND == 0) csr_retire(h, out);
    else csr_free(out);
    out.nrows = nd;
    int64_t *cnt = nullptr, *pptr = nullptr;
    RowStats *d_stats = nullptr;
    int4 *d_items = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
    auto cleanup = [&](int code) {
        dev_free(cnt); dev_free(pptr); dev_free(d_stats); dev_free(d_items);
        if (KIND == 0) spare_release(h);   // what the new H did not reuse
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (e2) cudaEventDestroy(e2);
        if (e3) cudaEventDestroy(e3);
        return code;
    };
    out.rowptr = (int64_t *)(KIND == 0 ? csr_buf(h, 0, (nd + 1) * 8, &rc) : dev_alloc(h, (nd + 1) * 8, &rc));
    if (rc) return cleanup(rc);
    cnt = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
    if (rc) return cleanup(rc);
    d_stats = (RowStats *)dev_alloc(h, sizeof(RowStats) + 16, &rc);
    if (rc) return cleanup(rc);
    unsigned long long *d_counter = (unsigned long long *)((char *)d_stats + sizeof(RowStats));
    RowStats init = {0, 0, 0, 0x7fffffffffffffffLL};
    PCI_CUDA(h, cudaMemcpyAsync(d_stats, &init, sizeof(RowStats), cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_counter, 0, 8, h->st));
    PCI_CUDA(h, cudaMemsetAsync(cnt, 0, (nd + 1) * 8, h->st));
    const size_t smem = sizeof(WarpSmem<NE>) * WARPS;
    auto kc64 = k_tiles<NE, KIND, 0, double>;
    auto kc32 = k_tiles<NE, KIND, 0, float>;
    auto kf64 = k_tiles<NE, KIND, 1, double>;
    auto kf32 = k_tiles<NE, KIND, 1, float>;
    cudaFuncSetAttribute(kc64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(kc32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(kf64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(kf32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc64, WARPS * 32, smem);
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
    const int blocks = dev_sms * std::max(per_sm, 1);
    std::vector<int4> items;
    make_items(h, h->h_rowwork, KIND, blocks * WARPS, items);
    d_items = (int4 *)dev_alloc(h, std::max<size_t>(items.size(), 1) * sizeof(int4), &rc);
    if (rc) return cleanup(rc);
    PCI_CUDA(h, cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, h->st));
    const int64_t nit = (int64_t)items.size();
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, out.rowptr + 1, nd, h->st);
    if ((rc = ensure_tmp(h, tb))) return cleanup(rc);
    auto check_derr = [&]() -> int {
        unsigned int derr = 0;
        PCI_CUDA(h, cudaMemcpy(&derr, h->d_err, 4, cudaMemcpyDeviceToHost));
        if (!derr) return PCI_OK;
        PCI_CUDA(h, cudaMemset(h->d_err, 0, 4));
        if (derr & DERR_MISSING_INTEGRAL) return set_err(h, PCI_E_MISSING_INTEGRAL, "Gint: integral is absent");
        if (derr & DERR_ROW_SLOTS) return set_err(h, PCI_E_CUDA, "FormH: a row produced more elements than its slots");
        return set_err(h, PCI_E_INPUT, "Gint error: ma+mb /= mc+md (determinant list inconsistent)");
    };
    auto launch_fill = [&](int64_t *rowinfo, int64_t *rowcnt_out, RowStats *st) {
        PCI_CUDA(h, cudaMemsetAsync(d_counter, 0, 8, h->st));
        if (value_prec == 32)
            kf32<<<blocks, WARPS * 32, smem, h->st>>>(S, d_items, nit, d_counter, rowinfo, out.col, (float *)out.val, st,
                                                      rowcnt_out);
        else
            kf64<<<blocks, WARPS * 32, smem, h->st>>>(S, d_items, nit, d_counter, rowinfo, out.col, (double *)out.val, st,
                                                      rowcnt_out);
        PCI_CUDA(h, cudaGetLastError());
        return PCI_OK;
    };
    const int forced = KIND == 0 ? formh_mode_env() : 0;
    if (KIND == 0) {
        h->st_formh_padded = 0;
        h->st_formh_compact = 0;
        h->st_formh_compact_launches = 0;
    }
    float t01 = 0, t12 = 0, t23 = 0;
    bool done = false;
    cudaEventRecord(e0, h->st);
    if (KIND == 0 && forced != 0) {
        // Single evaluation: candidate bound per row, padded fill, compaction.
        k_bound<NE><<<dev_sms * 8, 256, 0, h->st>>>(S, d_items, nit, d_counter, cnt);
        PCI_CUDA(h, cudaGetLastError());
        pptr = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
        if (rc) return cleanup(rc);
        PCI_CUDA(h, cudaMemsetAsync(pptr, 0, 8, h->st));
        cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, pptr + 1, nd, h->st);
        int64_t ncand = 0;
        PCI_CUDA(h, cudaMemcpyAsync(&ncand, pptr + nd, 8, cudaMemcpyDeviceToHost, h->st));
        PCI_CUDA(h, cudaStreamSynchronize(h->st));
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        fr += h->spare.col_bytes + h->spare.val_bytes;   // the retired H's buffers count as free
        const int64_t chunk = std::min<int64_t>(COMPACT_CHUNK, std::max<int64_t>(ncand, 1));
        const double need = (double)(ncand + chunk) * (4 + vb) + (double)(nd + 1) * 8 + (512.0 * (1 << 20));
        if (forced == 1 || need <= (double)fr) {
            out.nnz = ncand;
            out.val_f32 = value_prec == 32;
            out.col = (int32_t *)csr_buf(h, 1, std::max<int64_t>(ncand, 1) * 4, &rc);
            if (rc) return cleanup(rc);
            out.val = csr_buf(h, 2, std::max<int64_t>(ncand, 1) * vb, &rc);
            if (rc) return cleanup(rc);
            out.cap = ncand;
            cudaEventRecord(e1, h->st);
            if ((rc = launch_fill(pptr, cnt, d_stats))) return cleanup(rc);
            cudaEventRecord(e2, h->st);
            cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, out.rowptr + 1, nd, h->st);
            PCI_CUDA(h, cudaMemsetAsync(out.rowptr, 0, 8, h->st));
            PCI_CUDA(h, cudaStreamSynchronize(h->st));
            if ((rc = check_derr())) return cleanup(rc);
            if ((rc = hb_compact(h, pptr, out.rowptr, nd, out.col, out.val, vb, chunk))) return cleanup(rc);
            PCI_CUDA(h, cudaMemcpyAsync(&out.nnz, out.rowptr + nd, 8, cudaMemcpyDeviceToHost, h->st));
            cudaEventRecord(e3, h->st);
            PCI_CUDA(h, cudaStreamSynchronize(h->st));
            cudaEventElapsedTime(&t01, e0, e1);
            cudaEventElapsedTime(&t12, e1, e2);
            cudaEventElapsedTime(&t23, e2, e3);
            h->st_formh_padded = 1;
            h->st_formh_slots = (double)ncand;
            h->st_formh_compact = t23;
            done = true;
        } else {
            // does not fit: the two-pass build below (the scan time is kept in the count figure)
            dev_free(pptr);
            pptr = nullptr;
            PCI_CUDA(h, cudaMemsetAsync(d_counter, 0, 8, h->st));
            PCI_CUDA(h, cudaMemcpyAsync(d_stats, &init, sizeof(RowStats), cudaMemcpyHostToDevice, h->st));
        }
    }
    if (!done) {
        if (value_prec == 32)
            kc32<<<blocks, WARPS * 32, smem, h->st>>>(S, d_items, nit, d_counter, cnt, nullptr, nullptr, d_stats, nullptr);
        else
            kc64<<<blocks, WARPS * 32, smem, h->st>>>(S, d_items, nit, d_counter, cnt, nullptr, nullptr, d_stats, nullptr);
        PCI_CUDA(h, cudaGetLastError());
        PCI_CUDA(h, cudaMemsetAsync(out.rowptr, 0, 8, h->st));
        cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, out.rowptr + 1, nd, h->st);
        int64_t nnz = 0;
        PCI_CUDA(h, cudaMemcpyAsync(&nnz, out.rowptr + nd, 8, cudaMemcpyDeviceToHost, h->st));
        cudaEventRecord(e1, h->st);
        PCI_CUDA(h, cudaStreamSynchronize(h->st));
        if ((rc = check_derr())) return cleanup(rc);
        out.nnz = nnz;
        out.val_f32 = value_prec == 32;
        out.col = (int32_t *)(KIND == 0 ? csr_buf(h, 1, std::max<int64_t>(nnz, 1) * 4, &rc)
                                        : dev_alloc(h, std::max<int64_t>(nnz, 1) * 4, &rc));
        if (rc) return cleanup(rc);
        out.val = KIND == 0 ? csr_buf(h, 2, std::max<int64_t>(nnz, 1) * vb, &rc)
                            : dev_alloc(h, std::max<int64_t>(nnz, 1) * vb, &rc);
        if (rc) return cleanup(rc);
        if ((rc = launch_fill(out.rowptr, nullptr, nullptr))) return cleanup(rc);
        cudaEventRecord(e2, h->st);
        PCI_CUDA(h, cudaStreamSynchronize(h->st));
        cudaEventElapsedTime(&t01, e0, e1);
        cudaEventElapsedTime(&t12, e1, e2);
    }
    PCI_CUDA(h, cudaMemcpyAsync(hs, d_stats, sizeof(RowStats), cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    if (KIND == 0) {
        h->st_formh_count = t01;
        h->st_formh_fill = t12;
        h->st_formh = t01 + t12 + t23;
    } else {
        h->st_formj = t01 + t12;
    }
    return cleanup(PCI_OK);
}
