// Determinant-pair Hamiltonian build (FormH) and J^2 build (FormJ) on sm_100a.
//
// Compiled with -fmad=false: every floating-point expression keeps the
// reference's evaluation order with separately rounded multiplies and adds,
// so matrix elements are bit-identical to a straight restatement of
// Hmltn/Gint (src/pconf.F90:1653-1692, src/integrals.f90:153-293).
//
// Work decomposition.  Determinants come grouped by configuration.  The
// reference screens every (row n, configuration block) pair with CompD
// against the block's first determinant (src/pconf.F90:1238-1247).  Here the
// configuration-level screen is done once per configuration pair on the
// device (adjacency lists: c2 <= c1 with CompD <= 2), and one warp owns one
// row: it walks the adjacent blocks in ascending order, 32 columns at a time,
// compares occupation lists (Ne <= 8 m-states packed as uint16), evaluates
// the element and compacts the non-zeros with __ballot_sync/__popc so columns
// stay ascending.  Two passes: count (values evaluated, zeros dropped) and,
// after a scan, fill straight into CSR.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "pci_internal.h"

#define FULL_MASK 0xffffffffu

// ----------------------------------------------------------------- host ---

// Gaunt (src/integrals.f90:509-561): symmetry folds onto the j1 <= j2, m1 > 0
// half of the CONF.GNT table, absent entries give 0.
double host_gaunt(int nlx, const double *lut, int64_t nlut, int k, double xj1, double xm1,
                  double xj2, double xm2)
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
                if (im % 2 != 0) is = -is;
            }
            if (m1 <= 0.0) {
                m1 = -m1; m2 = -m2;
                int ij = (int)(k + j1 - j2);
                if (ij % 2 != 0) is = -is;
            }
            int ib1 = 2 * nlx + 1;
            int ib2 = ib1 * ib1;
            int64_t ind = (int64_t)(ib2 * (ib2 * k + 2 * (ib1 * j1 + j2)) + ib1 * (j1 + m1) + (j2 + m2));
            if (ind >= 0 && ind <= nlut - 1) return lut[ind] * is;
        }
    }
    return g * is;
}

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

__global__ void k_hash_insert(unsigned long long *keys, unsigned int *pos, unsigned long long mask,
                              const int32_t *iint2, const int32_t *iint3, int64_t n, unsigned int *err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int a = iint2[i], b = iint3[i];
        if (a <= 0 || b <= 0) { atomicOr(err, DERR_BAD_INDEX); continue; }
        unsigned long long key = hkey(a, b);
        unsigned long long s = hmix(key) & mask;
        int p = 0;
        for (; p < PCI_MAX_PROBE; p++) {
            unsigned long long prev = atomicCAS(&keys[s], 0ULL, key);
            if (prev == 0ULL || prev == key) {
                atomicMin(&pos[s], (unsigned int)i);  // first occurrence wins, as in FindGint
                break;
            }
            s = (s + 1) & mask;
        }
        if (p == PCI_MAX_PROBE) atomicOr(err, DERR_BAD_INDEX);
    }
}

template <typename RT>
__global__ void k_hash_fill(const unsigned long long *keys, const unsigned int *pos, double *vals,
                            unsigned long long cap, const RT *r2, int stride)
{
    for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap;
         s += (unsigned long long)gridDim.x * blockDim.x) {
        if (keys[s] != 0ULL) {
            unsigned long long p = pos[s];
            for (int c = 0; c < stride; c++) vals[s * stride + c] = (double)r2[p * stride + c];
        }
    }
}

int hb_build_hash(pci_gpu *h, int64_t ngint, int kbrt, int r2_is_f64, const void *rint2,
                  const int32_t *iint2, const int32_t *iint3)
{
    if (ngint <= 0 || ngint >= 0xffffffffLL) return set_err(h, PCI_E_INPUT, "Ngint out of range");
    unsigned long long cap = 1024;
    while (cap < 2ULL * (unsigned long long)ngint) cap <<= 1;
    int stride = kbrt ? 2 : 1;
    int rc = 0;
    dev_free(h->d_hkey);
    dev_free(h->d_hval);
    h->d_hkey = (unsigned long long *)dev_alloc(h, cap * 8, &rc);
    if (rc) return rc;
    h->d_hval = (double *)dev_alloc(h, cap * 8 * stride, &rc);
    if (rc) return rc;
    h->hcap = cap;
    size_t esz = r2_is_f64 ? 8 : 4;
    size_t need = cap * 4 + (size_t)ngint * (8 + esz * stride);
    if ((rc = ensure_tmp(h, need))) return rc;
    unsigned int *d_pos = (unsigned int *)h->d_tmp;
    int32_t *d_i2 = (int32_t *)((char *)h->d_tmp + cap * 4);
    int32_t *d_i3 = d_i2 + ngint;
    void *d_r2 = (void *)(d_i3 + ngint);
    PCI_CUDA(h, cudaMemsetAsync(h->d_hkey, 0, cap * 8, h->st));
    PCI_CUDA(h, cudaMemsetAsync(h->d_hval, 0, cap * 8 * stride, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_pos, 0xff, cap * 4, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_i2, iint2, ngint * 4, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_i3, iint3, ngint * 4, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_r2, rint2, (size_t)ngint * esz * stride, cudaMemcpyHostToDevice, h->st));
    k_hash_insert<<<148 * 8, 256, 0, h->st>>>(h->d_hkey, d_pos, cap - 1, d_i2, d_i3, ngint, h->d_err);
    if (r2_is_f64)
        k_hash_fill<double><<<148 * 8, 256, 0, h->st>>>(h->d_hkey, d_pos, h->d_hval, cap, (const double *)d_r2, stride);
    else
        k_hash_fill<float><<<148 * 8, 256, 0, h->st>>>(h->d_hkey, d_pos, h->d_hval, cap, (const float *)d_r2, stride);
    PCI_CUDA(h, cudaGetLastError());
    unsigned int e = 0;
    PCI_CUDA(h, cudaMemcpyAsync(&e, h->d_err, 4, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    if (e & DERR_BAD_INDEX) {
        PCI_CUDA(h, cudaMemset(h->d_err, 0, 4));
        return set_err(h, PCI_E_INPUT, "Iint2/Iint3 hold a non-positive key or the hash table overflowed");
    }
    h->kbrt = kbrt;
    return PCI_OK;
}

// ------------------------------------------------------- device physics ---

__device__ __forceinline__ double d_lookup(const DevSys &S, int iac, int ibd, int comp)
{
    unsigned long long key = hkey(iac, ibd);
    unsigned long long s = hmix(key) & S.hmask;
    int stride = S.kbrt ? 2 : 1;
    for (int p = 0; p < PCI_MAX_PROBE; p++) {
        unsigned long long k = __ldg(&S.hkey[s]);
        if (k == key) return __ldg(&S.hval[s * stride + comp]);
        if (k == 0ULL) break;
        s = (s + 1) & S.hmask;
    }
    atomicOr(S.err, DERR_MISSING_INTEGRAL);
    return 0.0;
}

// Hint (src/integrals.f90:122-151); m-states are 0-based.
__device__ __forceinline__ double d_hint(const DevSys &S, int ia, int ib)
{
    if (S.ms_jz[ia] != S.ms_jz[ib]) return 0.0;
    return __ldg(&S.h1[S.ms_orb[ia] * S.nsu + S.ms_orb[ib]]);
}

__device__ __forceinline__ double d_gaunt(const DevSys &S, int k, int t1, int t2)
{
    return __ldg(&S.gaunt[((size_t)k * S.ntype + t1) * S.ntype + t2]);
}

// Gint (src/integrals.f90:153-293) with Ksig < 2 and no SMS term.  Orbital
// indices are 0-based here, so the 1-based na-Nso-1 of the key becomes oa-Nso.
__device__ double d_gint(const DevSys &S, int i1, int i2, int i3, int i4)
{
    const bool l_br = S.kbrt != 0;
    double e = 0.0;
    int is = 1;
    int ia = i1, ib = i2, ic = i3, id = i4;
    for (int ii = 0; ii < 2; ii++) {
        int ma = S.ms_jz[ia], mb = S.ms_jz[ib], mc = S.ms_jz[ic], md = S.ms_jz[id];
        if (ma + mb != mc + md) { atomicOr(S.err, DERR_M_NOT_CONSERVED); return 0.0; }
        int na = S.ms_orb[ia], nb = S.ms_orb[ib], nc = S.ms_orb[ic], nd = S.ms_orb[id];
        int la = S.orb_l[na], lb = S.orb_l[nb], lc = S.orb_l[nc], ld = S.orb_l[nd];
        if (((la + lb + lc + ld) & 1) == 0) {
            int ja = S.orb_j[na], jb = S.orb_j[nb], jc = S.orb_j[nc], jd = S.orb_j[nd];
            int ta = S.ms_type[ia], tb = S.ms_type[ib], tc = S.ms_type[ic], td = S.ms_type[id];
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
                    double rabcd = d_lookup(S, iac, ibd0, 0);
                    if (l_br) rabcd = rabcd + is_br * d_lookup(S, iac, ibd0, 1);
                    double g1 = d_gaunt(S, k, ta, tc);
                    double g2 = d_gaunt(S, k, td, tb);
                    e = e + ((is * g1) * g2) * rabcd;
                }
            }
        }
        int t = ic; ic = id; id = t;
        is = -is;
    }
    return e;
}

// Plj (src/formj2.f90:48-67)
__device__ __forceinline__ double d_plj(const DevSys &S, int ia, int ib)
{
    int na = S.ms_orb[ia], nb = S.ms_orb[ib];
    if (na == nb) {
        int ma = S.ms_jz[ia], mb = S.ms_jz[ib];
        if (ma == mb + 2) {
            int ja = S.orb_j[na];
            return sqrt((double)(ja * (ja + 2) - ma * mb));
        }
    }
    return 0.0;
}

// F_J2, nf = 0 (src/formj2.f90:23-38)
template <int NE>
__device__ double d_fj2_diag(const DevSys &S, const uint16_t *d)
{
    double t = (double)(S.mj * S.mj);
#pragma unroll
    for (int iq = 0; iq < NE; iq++) {
        int a = d[iq];
        int ja = S.orb_j[S.ms_orb[a]], ma = S.ms_jz[a];
        t = t + (double)(ja * (ja + 2) - ma * ma);
#pragma unroll
        for (int jq = iq + 1; jq < NE; jq++) {
            int b = d[jq];
            double p1 = d_plj(S, a, b), p2 = d_plj(S, b, a);
            t = t - p1 * p1 - p2 * p2;
        }
    }
    return t;
}

// F_J2, nf = 2 (src/formj2.f90:39-41), arguments (ia, ic, ib, id)
__device__ __forceinline__ double d_fj2_two(const DevSys &S, int is, int ia, int ic, int ib, int id)
{
    return is * (d_plj(S, ia, ic) * d_plj(S, id, ib) + d_plj(S, ic, ia) * d_plj(S, ib, id)
                 - d_plj(S, ia, id) * d_plj(S, ic, ib) - d_plj(S, id, ia) * d_plj(S, ib, ic));
}

// Difference of two sorted occupation lists.  Positions of the differing
// m-states are list positions, so the fermion sign of Rspq_phase2
// (src/determinants.f90:709-724), (-1)^(|j2-i2| + |j3-i3|), is the parity of
// the sum of the four positions.
template <int NE>
struct Diff {
    int nf;
    int p1, p2, q1, q2;  // m-states: det1 (row) earlier/later, det2 (column) earlier/later
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
    r.is = 1;
    if (r.nf == 1 || r.nf == 2) {
        unsigned ua = (~ma) & ((1u << NE) - 1), ub = (~mb) & ((1u << NE) - 1);
        int ip1 = __ffs(ua) - 1, jp1 = __ffs(ub) - 1;
        int par = ip1 + jp1;
        r.p1 = d1[ip1];
        r.q1 = d2[jp1];
        if (r.nf == 2) {
            int ip2 = 31 - __clz(ua), jp2 = 31 - __clz(ub);
            par += ip2 + jp2;
            r.p2 = d1[ip2];
            r.q2 = d2[jp2];
        }
        r.is = (par & 1) ? -1 : 1;
    }
    return r;
}

// Hmltn (src/pconf.F90:1653-1692) as called from FormH with
// (i2, i1, j2, j1) = (jIndexes(3), iIndexes(3), jIndexes(2), iIndexes(2)).
template <int NE>
__device__ double d_hmltn(const DevSys &S, const uint16_t *d1, const Diff<NE> &df)
{
    double t = 0.0;
    if (df.nf == 2) {
        // Gint(i2, j2, i1, j1) = Gint(q1, q2, p1, p2)
        t = t + d_gint(S, df.q1, df.q2, df.p1, df.p2) * df.is;
        if (S.gj != 0.0) t = t + S.gj * d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
    } else if (df.nf == 1) {
        // j2 = q (det2), j1 = p (det1)
#pragma unroll
        for (int iq = 0; iq < NE; iq++) {
            int a = d1[iq];
            if (a != df.p1) t = t + d_gint(S, df.q1, a, df.p1, a) * df.is;
        }
        t = t + d_hint(S, df.q1, df.p1) * df.is;
    } else {
#pragma unroll
        for (int iq = 0; iq < NE; iq++) {
            int a = d1[iq];
#pragma unroll
            for (int jq = iq + 1; jq < NE; jq++) {
                int b = d1[jq];
                t = t + d_gint(S, a, b, a, b) * 1;
            }
            t = t + d_hint(S, a, a) * 1;
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
template <int NE, int FILL>
__global__ void __launch_bounds__(256) k_adjacency(DevSys S, const int32_t *ndc, int64_t *cnt, int32_t *adj)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c1 = warp; c1 < S.nc; c1 += nwarps) {
        if (ndc[c1] == 0) {
            if (!FILL && lane == 0) cnt[c1] = 0;
            continue;
        }
        uint16_t a[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) a[e] = S.conf_orb[c1 * NE + e];
        int64_t base = FILL ? cnt[c1] : 0, c = 0;
        for (int64_t c2b = 0; c2b <= c1; c2b += 32) {
            int64_t c2 = c2b + lane;
            bool ok = false;
            if (c2 <= c1 && ndc[c2] > 0) {
                uint16_t b[NE];
#pragma unroll
                for (int e = 0; e < NE; e++) b[e] = S.conf_orb[c2 * NE + e];
                ok = d_compd<NE>(a, b) <= 2;
            }
            unsigned m = __ballot_sync(FULL_MASK, ok);
            if (FILL && ok) adj[base + c + __popc(m & ((1u << lane) - 1))] = (int32_t)c2;
            c += __popc(m);
        }
        if (!FILL && lane == 0) cnt[c1] = c;
    }
}

template <int NE>
static int adjacency_impl(pci_gpu *h, DevSys S, const int32_t *d_ndc)
{
    int rc = 0;
    int64_t nc = h->nc;
    int64_t *cnt = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) return rc;
    k_adjacency<NE, 0><<<148 * 8, 256, 0, h->st>>>(S, d_ndc, cnt, nullptr);
    PCI_CUDA(h, cudaGetLastError());
    dev_free(h->d_adj_ptr);
    h->d_adj_ptr = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) { dev_free(cnt); return rc; }
    PCI_CUDA(h, cudaMemsetAsync(h->d_adj_ptr, 0, 8, h->st));
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, h->d_adj_ptr + 1, nc, h->st);
    if ((rc = ensure_tmp(h, tb))) { dev_free(cnt); return rc; }
    cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, h->d_adj_ptr + 1, nc, h->st);
    int64_t nadj = 0;
    PCI_CUDA(h, cudaMemcpyAsync(&nadj, h->d_adj_ptr + nc, 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    dev_free(h->d_adj);
    h->d_adj = (int32_t *)dev_alloc(h, std::max<int64_t>(nadj, 1) * 4, &rc);
    if (rc) { dev_free(cnt); return rc; }
    S.adj_ptr = h->d_adj_ptr;
    k_adjacency<NE, 1><<<148 * 8, 256, 0, h->st>>>(S, d_ndc, h->d_adj_ptr, h->d_adj);
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    dev_free(cnt);
    h->n_adj = nadj;
    return PCI_OK;
}

int hb_build_adjacency(pci_gpu *h)
{
    int rc = 0;
    int32_t *d_ndc = (int32_t *)dev_alloc(h, (size_t)h->nc * 4, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_ndc, h->h_ndc.data(), (size_t)h->nc * 4, cudaMemcpyHostToDevice, h->st));
    DevSys S = make_devsys(h);
    switch (h->ne) {
    case 1: rc = adjacency_impl<1>(h, S, d_ndc); break;
    case 2: rc = adjacency_impl<2>(h, S, d_ndc); break;
    case 3: rc = adjacency_impl<3>(h, S, d_ndc); break;
    case 4: rc = adjacency_impl<4>(h, S, d_ndc); break;
    case 5: rc = adjacency_impl<5>(h, S, d_ndc); break;
    case 6: rc = adjacency_impl<6>(h, S, d_ndc); break;
    case 7: rc = adjacency_impl<7>(h, S, d_ndc); break;
    case 8: rc = adjacency_impl<8>(h, S, d_ndc); break;
    default: rc = set_err(h, PCI_E_INPUT, "Ne outside 1..8");
    }
    dev_free(d_ndc);
    return rc;
}

// ------------------------------------------------------------ row pass ---

struct RowStats {
    unsigned long long numzero, pairs, scanned;
    long long hmin_key;  // order-preserving integer image of the minimum value
};

__device__ __forceinline__ long long dkey(double x)
{
    long long b = __double_as_longlong(x);
    return b >= 0 ? b : (b ^ 0x7fffffffffffffffLL);
}

static double key_to_double(long long k)
{
    long long b = k >= 0 ? k : (k ^ 0x7fffffffffffffffLL);
    double x;
    memcpy(&x, &b, 8);
    return x;
}

// KIND 0: Hamiltonian over adjacent configuration blocks, k <= n.
// KIND 1: J^2 inside the row's own configuration block, k <= n, nf in {0, 2}.
// FILL 0: per-row counts into rowinfo[n]; FILL 1: rowinfo is the CSR rowptr.
template <int NE, int KIND, int FILL, typename VT>
__global__ void __launch_bounds__(256) k_rows(DevSys S, unsigned long long *row_counter,
                                               int64_t *rowinfo, int32_t *col, VT *val, RowStats *stats)
{
    const int lane = threadIdx.x & 31;
    unsigned long long nzero = 0, npairs = 0, nscan = 0;
    double hmin = INFINITY;
    while (true) {
        unsigned long long n = 0;
        if (lane == 0) n = atomicAdd(row_counter, 1ULL);
        n = __shfl_sync(FULL_MASK, n, 0);
        if (n >= (unsigned long long)S.nd) break;
        uint16_t d1[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) d1[e] = S.occ[n * NE + e];
        const int c1 = S.conf_of[n];
        int64_t base = FILL ? rowinfo[n] : 0, c = 0;
        int64_t a0 = KIND == 0 ? S.adj_ptr[c1] : 0, a1 = KIND == 0 ? S.adj_ptr[c1 + 1] : 1;
        for (int64_t a = a0; a < a1; a++) {
            const int c2 = KIND == 0 ? S.adj[a] : c1;
            const int64_t k0 = S.conf_start[c2];
            const int64_t k1 = min(S.conf_start[c2 + 1], (int64_t)n + 1);
            for (int64_t kb = k0; kb < k1; kb += 32) {
                const int64_t k = kb + lane;
                bool nz = false;
                double v = 0.0;
                if (k < k1) {
                    nscan++;
                    uint16_t d2[NE];
#pragma unroll
                    for (int e = 0; e < NE; e++) d2[e] = S.occ[k * NE + e];
                    Diff<NE> df = d_diff<NE>(d1, d2);
                    if (KIND == 0) {
                        if (df.nf <= 2) {
                            npairs++;
                            v = d_hmltn<NE>(S, d1, df);
                            if (v != 0.0) nz = true; else nzero++;
                        }
                    } else {
                        if (df.nf == 0) v = d_fj2_diag<NE>(S, d1);
                        else if (df.nf == 2) v = d_fj2_two(S, df.is, df.q1, df.p1, df.q2, df.p2);
                        nz = (df.nf == 0 || df.nf == 2) && v != 0.0;
                    }
                }
                unsigned m = __ballot_sync(FULL_MASK, nz);
                if (nz) {
                    VT vs = (VT)v;
                    double vd = (double)vs;
                    if (vd < hmin) hmin = vd;
                    if (FILL) {
                        int64_t p = base + c + __popc(m & ((1u << lane) - 1));
                        col[p] = (int32_t)k;
                        val[p] = vs;
                    }
                }
                c += __popc(m);
            }
        }
        if (!FILL && lane == 0) rowinfo[n] = c;
    }
    // warp reductions, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) {
        nzero += __shfl_down_sync(FULL_MASK, nzero, o);
        npairs += __shfl_down_sync(FULL_MASK, npairs, o);
        nscan += __shfl_down_sync(FULL_MASK, nscan, o);
        hmin = fmin(hmin, __shfl_down_sync(FULL_MASK, hmin, o));
    }
    if (lane == 0 && stats) {
        atomicAdd(&stats->numzero, nzero);
        atomicAdd(&stats->pairs, npairs);
        atomicAdd(&stats->scanned, nscan);
        if (hmin < INFINITY) atomicMin(&stats->hmin_key, dkey(hmin));
    }
}

template <int NE, int KIND>
static int rows_impl(pci_gpu *h, int value_prec, Csr &out, RowStats *hs)
{
    int rc = 0;
    DevSys S = make_devsys(h);
    const int64_t nd = h->nd;
    csr_free(out);
    out.nrows = nd;
    out.rowptr = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
    if (rc) return rc;
    int64_t *cnt = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
    if (rc) return rc;
    RowStats *d_stats = nullptr;
    unsigned long long *d_counter = nullptr;
    d_stats = (RowStats *)dev_alloc(h, sizeof(RowStats) + 16, &rc);
    if (rc) { dev_free(cnt); return rc; }
    d_counter = (unsigned long long *)((char *)d_stats + sizeof(RowStats));
    RowStats init = {0, 0, 0, 0x7fffffffffffffffLL};
    PCI_CUDA(h, cudaMemcpyAsync(d_stats, &init, sizeof(RowStats), cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_counter, 0, 8, h->st));
    int blocks = 148 * 8;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
    cudaEventRecord(e0, h->st);
    if (value_prec == 32)
        k_rows<NE, KIND, 0, float><<<blocks, 256, 0, h->st>>>(S, d_counter, cnt, nullptr, nullptr, d_stats);
    else
        k_rows<NE, KIND, 0, double><<<blocks, 256, 0, h->st>>>(S, d_counter, cnt, nullptr, nullptr, d_stats);
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaMemsetAsync(out.rowptr, 0, 8, h->st));
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, out.rowptr + 1, nd, h->st);
    if ((rc = ensure_tmp(h, tb))) return rc;
    cub::DeviceScan::InclusiveSum(h->d_tmp, tb, cnt, out.rowptr + 1, nd, h->st);
    int64_t nnz = 0;
    PCI_CUDA(h, cudaMemcpyAsync(&nnz, out.rowptr + nd, 8, cudaMemcpyDeviceToHost, h->st));
    cudaEventRecord(e1, h->st);
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    unsigned int derr = 0;
    PCI_CUDA(h, cudaMemcpy(&derr, h->d_err, 4, cudaMemcpyDeviceToHost));
    if (derr) {
        dev_free(cnt); dev_free(d_stats);
        PCI_CUDA(h, cudaMemset(h->d_err, 0, 4));
        if (derr & DERR_MISSING_INTEGRAL) return set_err(h, PCI_E_MISSING_INTEGRAL, "Gint: integral is absent");
        return set_err(h, PCI_E_INPUT, "Gint error: ma+mb /= mc+md (determinant list inconsistent)");
    }
    out.nnz = nnz;
    out.val_f32 = value_prec == 32;
    out.col = (int32_t *)dev_alloc(h, std::max<int64_t>(nnz, 1) * 4, &rc);
    if (rc) return rc;
    out.val = dev_alloc(h, std::max<int64_t>(nnz, 1) * (out.val_f32 ? 4 : 8), &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemsetAsync(d_counter, 0, 8, h->st));
    if (value_prec == 32)
        k_rows<NE, KIND, 1, float><<<blocks, 256, 0, h->st>>>(S, d_counter, out.rowptr, out.col, (float *)out.val, nullptr);
    else
        k_rows<NE, KIND, 1, double><<<blocks, 256, 0, h->st>>>(S, d_counter, out.rowptr, out.col, (double *)out.val, nullptr);
    PCI_CUDA(h, cudaGetLastError());
    cudaEventRecord(e2, h->st);
    PCI_CUDA(h, cudaMemcpyAsync(hs, d_stats, sizeof(RowStats), cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    float t01 = 0, t12 = 0;
    cudaEventElapsedTime(&t01, e0, e1);
    cudaEventElapsedTime(&t12, e1, e2);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    if (KIND == 0) {
        h->st_formh_count = t01;
        h->st_formh_fill = t12;
        h->st_formh = t01 + t12;
    } else {
        h->st_formj = t01 + t12;
    }
    dev_free(cnt);
    dev_free(d_stats);
    return PCI_OK;
}

template <int KIND>
static int rows_dispatch(pci_gpu *h, int value_prec, Csr &out, RowStats *hs)
{
    switch (h->ne) {
    case 1: return rows_impl<1, KIND>(h, value_prec, out, hs);
    case 2: return rows_impl<2, KIND>(h, value_prec, out, hs);
    case 3: return rows_impl<3, KIND>(h, value_prec, out, hs);
    case 4: return rows_impl<4, KIND>(h, value_prec, out, hs);
    case 5: return rows_impl<5, KIND>(h, value_prec, out, hs);
    case 6: return rows_impl<6, KIND>(h, value_prec, out, hs);
    case 7: return rows_impl<7, KIND>(h, value_prec, out, hs);
    case 8: return rows_impl<8, KIND>(h, value_prec, out, hs);
    }
    return set_err(h, PCI_E_INPUT, "Ne outside 1..8");
}

int hb_form_h(pci_gpu *h, int value_prec, int64_t *numh, int64_t *numzero, double *hmin)
{
    if (!h->have_basis || !h->have_ints) return set_err(h, PCI_E_STATE, "form_h before set_basis/set_integrals");
    if (value_prec != 64 && value_prec != 32) return set_err(h, PCI_E_INPUT, "value_prec must be 64 or 32");
    int rc;
    cudaEvent_t a0, a1;
    cudaEventCreate(&a0); cudaEventCreate(&a1);
    cudaEventRecord(a0, h->st);
    if ((rc = hb_build_adjacency(h))) return rc;
    cudaEventRecord(a1, h->st);
    cudaEventSynchronize(a1);
    float tadj = 0;
    cudaEventElapsedTime(&tadj, a0, a1);
    cudaEventDestroy(a0); cudaEventDestroy(a1);
    RowStats hs;
    if ((rc = rows_dispatch<0>(h, value_prec, h->H, &hs))) return rc;
    h->st_adj = tadj;
    h->st_formh += tadj;
    h->st_pairs = (double)hs.pairs;
    h->st_scanned = (double)hs.scanned;
    // adjacency: 2 passes + scan (2 kernels) + memset; rows: 2 passes + scan (2) + 2 memsets
    h->st_launches = 11;
    csr_free(h->Hfull);
    h->numh = h->H.nnz;
    h->numzero = (int64_t)hs.numzero;
    h->hmin = h->H.nnz ? key_to_double(hs.hmin_key) : 0.0;
    if (numh) *numh = h->numh;
    if (numzero) *numzero = h->numzero;
    if (hmin) *hmin = h->hmin;
    return PCI_OK;
}

int hb_form_j(pci_gpu *h, int64_t *numj)
{
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "form_j before set_basis");
    RowStats hs;
    int rc = rows_dispatch<1>(h, 64, h->J, &hs);
    if (rc) return rc;
    h->numj = h->J.nnz;
    if (numj) *numj = h->numj;
    return PCI_OK;
}
