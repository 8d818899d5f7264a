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
// row configuration c1: for each adjacent c2 it evaluates the whole
// Ndc(c1) x Ndc(c2) tile of determinant pairs 32 at a time.  Every Gint call
// inside a tile uses radial integrals of the same few orbital quadruples, so
// the warp looks them up once per tile into a shared-memory cache.  Pairs are
// compared on occupation lists (Ne <= 8 m-states as uint16); non-zeros are
// compacted per row with __match_any_sync/__ballot_sync/__popc so each row's
// columns stay ascending.  Two builds: single evaluation (bound the
// candidate pairs of each row from the configurations alone, evaluate once
// into rows padded to that bound, squeeze the rows into CSR), taken when the
// padded rows fit in device memory; otherwise two passes (count with values
// evaluated and zeros dropped, then, after a scan, fill straight into CSR).
// The fill checks every write against its row's slots.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pci_internal.h"

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

#include "hbuild_impl.cuh"

__global__ void k_hash_insert(unsigned long long *htab, int hw, unsigned int *pos, unsigned long long mask,
                              const int32_t *iint2, const int32_t *iint3, int64_t n, unsigned int *err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int a = iint2[i], b = iint3[i];
        if (a <= 0 || b <= 0) { atomicOr(err, DERR_BAD_INDEX); continue; }
        unsigned long long key = hkey(a, b);
        unsigned long long s = hmix(key) & mask;
        int p = 0;
        for (; p < PCI_MAX_PROBE; p++) {
            unsigned long long prev = atomicCAS(&htab[s * hw], 0ULL, key);
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
__global__ void k_hash_fill(unsigned long long *htab, int hw, const unsigned int *pos, unsigned long long cap,
                            const RT *r2, int stride)
{
    for (unsigned long long s = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; s < cap;
         s += (unsigned long long)gridDim.x * blockDim.x) {
        if (htab[s * hw] != 0ULL) {
            unsigned long long p = pos[s];
            for (int c = 0; c < stride; c++)
                htab[s * hw + 1 + c] = (unsigned long long)__double_as_longlong((double)r2[p * stride + c]);
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
    // key and value(s) of a slot share one 16-byte (32 with Breit) line, so
    // a probe reads both with one load
    const int hw = stride == 2 ? 4 : 2;
    dev_free(h->d_htab);
    h->d_htab = (unsigned long long *)dev_alloc(h, cap * 8 * hw, &rc);
    if (rc) return rc;
    h->hw = hw;
    h->hcap = cap;
    size_t esz = r2_is_f64 ? 8 : 4;
    size_t need = cap * 4 + (size_t)ngint * (8 + esz * stride);
    if ((rc = ensure_tmp(h, need))) return rc;
    unsigned int *d_pos = (unsigned int *)h->d_tmp;
    int32_t *d_i2 = (int32_t *)((char *)h->d_tmp + cap * 4);
    int32_t *d_i3 = d_i2 + ngint;
    void *d_r2 = (void *)(d_i3 + ngint);
    PCI_CUDA(h, cudaMemsetAsync(h->d_htab, 0, cap * 8 * hw, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_pos, 0xff, cap * 4, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_i2, iint2, ngint * 4, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_i3, iint3, ngint * 4, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_r2, rint2, (size_t)ngint * esz * stride, cudaMemcpyHostToDevice, h->st));
    k_hash_insert<<<148 * 8, 256, 0, h->st>>>(h->d_htab, hw, d_pos, cap - 1, d_i2, d_i3, ngint, h->d_err);
    if (r2_is_f64)
        k_hash_fill<double><<<148 * 8, 256, 0, h->st>>>(h->d_htab, hw, d_pos, cap, (const double *)d_r2, stride);
    else
        k_hash_fill<float><<<148 * 8, 256, 0, h->st>>>(h->d_htab, hw, d_pos, cap, (const float *)d_r2, stride);
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

// ----------------------------------------------------------- compaction ---

// Smallest gap (entries) worth a direct in-place move; below it rows go
// through the buffer.  Zeros are spread over the rows, so the gap grows with
// the position and only the first rows need the buffer.
constexpr int64_t COMPACT_DIRECT_MIN = 1LL << 20;

// One warp per row: copy the row's entries from its padded slot to its CSR
// position, relative to the chunk's first CSR position qa.  The source and
// destination may be the same arrays as long as the chunk's destination
// range ends before its source range starts.
template <typename VT>
__global__ void k_compact_gather(const int64_t *pptr, const int64_t *rowptr, int64_t ra, int64_t rb, int64_t qa,
                                 const int32_t *col, const VT *val, int32_t *tcol, VT *tval)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ra + w; r < rb; r += nw) {
        const int64_t src = pptr[r], dst = rowptr[r] - qa, n = rowptr[r + 1] - rowptr[r];
        int64_t i = lane;
        // four loads of each array in flight per lane before the stores
        for (; i + 96 < n; i += 128) {
            int32_t c[4];
            VT v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) { c[u] = col[src + i + 32 * u]; v[u] = val[src + i + 32 * u]; }
#pragma unroll
            for (int u = 0; u < 4; u++) { tcol[dst + i + 32 * u] = c[u]; tval[dst + i + 32 * u] = v[u]; }
        }
        for (; i < n; i += 32) {
            tcol[dst + i] = col[src + i];
            tval[dst + i] = val[src + i];
        }
    }
}

int hb_compact(pci_gpu *h, const int64_t *pptr, const int64_t *rowptr, int64_t nrows, int32_t *col, void *val,
               int vbytes, int64_t chunk)
{
    std::vector<int64_t> p(nrows + 1), q(nrows + 1);
    PCI_CUDA(h, cudaMemcpyAsync(p.data(), pptr, (nrows + 1) * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(q.data(), rowptr, (nrows + 1) * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    // rows that start where their padded slot starts are already in place
    int64_t ra = 0;
    while (ra < nrows && p[ra] == q[ra]) ra++;
    if (q[nrows] == p[nrows]) return PCI_OK;
    int64_t maxrow = 0;
    for (int64_t r = ra; r < nrows; r++) maxrow = std::max(maxrow, q[r + 1] - q[r]);
    chunk = std::max(chunk, maxrow);
    // the buffer lives in the handle's scratch (kept across calls); values
    // first so both arrays stay aligned
    int rc = 0;
    if ((rc = ensure_tmp(h, (size_t)chunk * (vbytes + 4) + 256))) return rc;
    void *tval = h->d_tmp;
    int32_t *tcol = (int32_t *)((char *)h->d_tmp + (((size_t)chunk * vbytes + 255) & ~(size_t)255));
    while (ra < nrows) {
        // Direct move: once the gap p[ra] - q[ra] left by the zeros dropped
        // so far covers a whole run of rows, their CSR range ends before
        // their padded range starts and they move in place without a buffer.
        const int64_t gap = p[ra] - q[ra];
        if (gap >= COMPACT_DIRECT_MIN) {
            int64_t rb = std::upper_bound(q.begin() + ra + 1, q.end(), q[ra] + gap) - q.begin() - 1;
            if (rb > ra) {
                if (vbytes == 4)
                    k_compact_gather<float><<<148 * 8, 256, 0, h->st>>>(pptr, rowptr, ra, rb, 0, col, (const float *)val,
                                                                         col, (float *)val);
                else
                    k_compact_gather<double><<<148 * 8, 256, 0, h->st>>>(pptr, rowptr, ra, rb, 0, col,
                                                                          (const double *)val, col, (double *)val);
                PCI_CUDA(h, cudaGetLastError());
                h->st_formh_compact_launches += 1;
                ra = rb;
                continue;
            }
        }
        // largest rb with q[rb] - q[ra] <= chunk (at least one row)
        int64_t rb = std::upper_bound(q.begin() + ra + 1, q.end(), q[ra] + chunk) - q.begin() - 1;
        rb = std::max(rb, ra + 1);
        const int64_t n = q[rb] - q[ra];
        if (n > 0) {
            if (vbytes == 4)
                k_compact_gather<float><<<148 * 8, 256, 0, h->st>>>(pptr, rowptr, ra, rb, q[ra], col, (const float *)val,
                                                                     tcol, (float *)tval);
            else
                k_compact_gather<double><<<148 * 8, 256, 0, h->st>>>(pptr, rowptr, ra, rb, q[ra], col,
                                                                      (const double *)val, tcol, (double *)tval);
            PCI_CUDA(h, cudaGetLastError());
            h->st_formh_compact_launches += 1;
            PCI_CUDA(h, cudaMemcpyAsync(col + q[ra], tcol, n * 4, cudaMemcpyDeviceToDevice, h->st));
            PCI_CUDA(h, cudaMemcpyAsync((char *)val + q[ra] * vbytes, tval, n * vbytes, cudaMemcpyDeviceToDevice, h->st));
        }
        ra = rb;
    }
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    return PCI_OK;
}

// ------------------------------------------------------ per-Ne dispatch ---

#define PCI_DECL_NE(n)                                                                   \
    int hb_adjacency_ne##n(pci_gpu *h, DevSys S, const int32_t *d_ndc);                  \
    int hb_rows_ne##n(pci_gpu *h, int kind, int value_prec, Csr &out, RowStatsOut *hs);
PCI_DECL_NE(1) PCI_DECL_NE(2) PCI_DECL_NE(3) PCI_DECL_NE(4)
PCI_DECL_NE(5) PCI_DECL_NE(6) PCI_DECL_NE(7) PCI_DECL_NE(8)

int hb_build_adjacency(pci_gpu *h, int w_c1, int w_c0, int w_c2)
{
    int rc = 0;
    h->adj_win_c1 = w_c1;
    h->adj_win_c0 = w_c0;
    h->adj_win_c2 = w_c2;
    int32_t *d_ndc = (int32_t *)dev_alloc(h, (size_t)h->nc * 4, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_ndc, h->h_ndc.data(), (size_t)h->nc * 4, cudaMemcpyHostToDevice, h->st));
    DevSys S = make_devsys(h);
    switch (h->ne) {
    case 1: rc = hb_adjacency_ne1(h, S, d_ndc); break;
    case 2: rc = hb_adjacency_ne2(h, S, d_ndc); break;
    case 3: rc = hb_adjacency_ne3(h, S, d_ndc); break;
    case 4: rc = hb_adjacency_ne4(h, S, d_ndc); break;
    case 5: rc = hb_adjacency_ne5(h, S, d_ndc); break;
    case 6: rc = hb_adjacency_ne6(h, S, d_ndc); break;
    case 7: rc = hb_adjacency_ne7(h, S, d_ndc); break;
    case 8: rc = hb_adjacency_ne8(h, S, d_ndc); break;
    default: rc = set_err(h, PCI_E_INPUT, "Ne outside 1..8");
    }
    dev_free(d_ndc);
    return rc;
}

static int rows_dispatch(pci_gpu *h, int kind, int value_prec, Csr &out, RowStatsOut *hs)
{
    switch (h->ne) {
    case 1: return hb_rows_ne1(h, kind, value_prec, out, hs);
    case 2: return hb_rows_ne2(h, kind, value_prec, out, hs);
    case 3: return hb_rows_ne3(h, kind, value_prec, out, hs);
    case 4: return hb_rows_ne4(h, kind, value_prec, out, hs);
    case 5: return hb_rows_ne5(h, kind, value_prec, out, hs);
    case 6: return hb_rows_ne6(h, kind, value_prec, out, hs);
    case 7: return hb_rows_ne7(h, kind, value_prec, out, hs);
    case 8: return hb_rows_ne8(h, kind, value_prec, out, hs);
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
    RowStatsOut hs;
    h->h_from_tiles = false;
    if ((rc = rows_dispatch(h, 0, value_prec, h->H, &hs))) {
        csr_free(h->H);   // no half-built matrix stays resident
        return rc;
    }
    h->st_adj = tadj;
    h->st_formh += tadj;
    h->st_pairs = (double)hs.pairs;
    h->st_scanned = (double)hs.scanned;
    // adjacency: 2 passes + scan (2 kernels); tiles: 2 passes + scan (2);
    // the single-evaluation build adds a second scan and its compaction
    h->st_launches = h->st_formh_padded ? 10 + h->st_formh_compact_launches : 8;
    csr_free(h->Hfull);
    h->h_from_tiles = true;
    h->h_pt_nd1 = -1;
    h->numh = h->H.nnz;
    h->numzero = (int64_t)hs.numzero;
    h->hmin = hs.hmin;
    if (numh) *numh = h->numh;
    if (numzero) *numzero = h->numzero;
    if (hmin) *hmin = h->hmin;
    return PCI_OK;
}

// conf_pt's PT block: the rows of the PT determinants row_lo..row_hi-1
// (within nd1..Nd-1) against the first nd0 columns and their own
// configuration's diagonal block (for H_ii), through the tile kernel over a
// windowed adjacency.  Other rows stay empty, so the stored elements are
// those PTE (conf_pt.f90:751-952) reads for these rows and none of the PT x PT
// block beyond the diagonal configurations.
int hb_form_h_pt(pci_gpu *h, int64_t nd1, int64_t nd0, int64_t row_lo, int64_t row_hi, int value_prec,
                 int64_t *numh)
{
    if (!h->have_basis || !h->have_ints) return set_err(h, PCI_E_STATE, "form_h_pt before set_basis/set_integrals");
    if (value_prec != 64 && value_prec != 32) return set_err(h, PCI_E_INPUT, "value_prec must be 64 or 32");
    if (nd0 < 1 || nd0 > nd1 || nd1 > h->nd) return set_err(h, PCI_E_INPUT, "form_h_pt: need 1 <= Nd0 <= Nd1 <= Nd");
    if (row_lo < nd1 || row_hi <= row_lo || row_hi > h->nd)
        return set_err(h, PCI_E_INPUT, "form_h_pt: need Nd1 <= row_lo < row_hi <= Nd");
    // configuration index at which determinant n starts (n must end a configuration)
    auto conf_at = [&](int64_t n) -> int {
        int64_t s = 0;
        for (int c = 0; c < h->nc; c++) {
            if (s == n) return c;
            s += h->h_ndc[c];
        }
        return s == n ? h->nc : -1;
    };
    const int c1 = conf_at(row_lo), c2 = conf_at(row_hi), c0 = conf_at(nd0);
    if (conf_at(nd1) < 0 || c0 < 0 || c1 < 0 || c2 < 0)
        return set_err(h, PCI_E_INPUT, "form_h_pt: Nd1, Nd0, row_lo and row_hi must end a configuration");
    int rc;
    cudaEvent_t a0, a1;
    cudaEventCreate(&a0); cudaEventCreate(&a1);
    cudaEventRecord(a0, h->st);
    if ((rc = hb_build_adjacency(h, c1, c0, c2))) { cudaEventDestroy(a0); cudaEventDestroy(a1); return rc; }
    cudaEventRecord(a1, h->st);
    cudaEventSynchronize(a1);
    float tadj = 0;
    cudaEventElapsedTime(&tadj, a0, a1);
    cudaEventDestroy(a0); cudaEventDestroy(a1);
    RowStatsOut hs;
    h->h_pt_nd1 = -1;
    h->h_from_tiles = false;
    if ((rc = rows_dispatch(h, 0, value_prec, h->H, &hs))) {
        csr_free(h->H);   // no half-built matrix stays resident
        return rc;
    }
    h->st_adj = tadj;
    h->st_formh += tadj;
    h->st_pairs = (double)hs.pairs;
    h->st_scanned = (double)hs.scanned;
    h->st_launches = h->st_formh_padded ? 10 + h->st_formh_compact_launches : 8;
    csr_free(h->Hfull);
    h->h_from_tiles = false;   // the adjacency is windowed; nothing else may walk it with this H
    h->h_pt_nd1 = nd1;
    h->h_pt_nd0 = nd0;
    h->h_pt_lo = row_lo;
    h->h_pt_hi = row_hi;
    h->numh = h->H.nnz;
    h->numzero = (int64_t)hs.numzero;
    h->hmin = hs.hmin;
    if (numh) *numh = h->numh;
    return PCI_OK;
}

int hb_form_j(pci_gpu *h, int64_t *numj)
{
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "form_j before set_basis");
    RowStatsOut hs;
    int rc = rows_dispatch(h, 1, 64, h->J, &hs);
    if (rc) return rc;
    h->numj = h->J.nnz;
    if (numj) *numj = h->numj;
    return PCI_OK;
}
