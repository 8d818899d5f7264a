// CSF basis (kCSF = 1): jbasis, formh_sym and unsym (src/csf.f90) on the GPU.
//
// jbasis: for every configuration the J^2 block of its determinants (the
// diagonal blocks of the FormJ matrix) is diagonalised, and the eigenvectors
// with 2J = Mj are the configuration's CSFs (src/csf.f90:17-407).  Here one
// thread block per configuration loads its block into shared memory and runs
// cyclic Jacobi rotations (round-robin order, disjoint pairs per step); the
// host picks the eigenvectors (the same J test as the reference) and a
// gather kernel packs the CSF coefficients C_c (ndc x ncsf, column-major per
// configuration).
//
// formh_sym: the CSF Hamiltonian H_csf = C^T H C (src/csf.f90:538-1006),
// kept as a lower-triangle CSR over the CSFs (configurations in order, CSFs
// of a configuration in eigenvector order).  One thread block per row
// configuration c1 walks its adjacency list (c2 <= c1, ascending, CompD <=
// 2, built by FormH): the determinant block H[c1, c2] is scattered from the
// lower-triangle CSR into shared memory (a cursor per row advances through
// its sorted columns as c2 grows; the diagonal block is symmetrised), then
// T = H[c1, c2] C_c2 and B = C_c1^T T, and B (its lower triangle for c2 =
// c1) is written to the CSF rows.
//
// unsym: determinant vectors x_n = sum_i C_c[n, i] y_(c, i) (src/csf.f90:
// 1088-1134).
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pci_internal.h"

namespace {

constexpr int CSF_MAX_NDC = 112;   // determinants per configuration (two m x m FP64 arrays in shared memory)

// Eigenpairs of each configuration's J^2 block: eigenvalues into w[n0 + i],
// eigenvectors column-major into ev[off_c + i * m + r].
__global__ void __launch_bounds__(256) k_csf_jblocks(const int64_t *__restrict__ conf_start,
                                                     const int64_t *__restrict__ jrow, const int32_t *__restrict__ jcol,
                                                     const double *__restrict__ jval, const int64_t *__restrict__ evoff,
                                                     double *w, double *ev, int *bad)
{
    const int c = blockIdx.x, t = threadIdx.x;
    const int64_t n0 = conf_start[c];
    const int m = (int)(conf_start[c + 1] - n0);
    if (m == 0) return;
    const int mp = m + (m & 1), h = mp / 2;
    extern __shared__ double sm[];
    double *A = sm, *V = sm + mp * mp;
    __shared__ int pp[CSF_MAX_NDC / 2], qq[CSF_MAX_NDC / 2];
    __shared__ double cc[CSF_MAX_NDC / 2], sn[CSF_MAX_NDC / 2];
    __shared__ double red[2][8];
    __shared__ int stop;
    for (int e = t; e < mp * mp; e += blockDim.x) {
        A[e] = 0.0;
        V[e] = (e / mp == e % mp) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int r = t; r < m; r += blockDim.x) {
        const int64_t n = n0 + r;
        for (int64_t l = jrow[n]; l < jrow[n + 1]; l++) {
            const int64_t k = jcol[l];
            if (k < n0 || k > n) continue;   // J^2 couples determinants of one configuration only
            const int q = (int)(k - n0);
            A[r * mp + q] = jval[l];
            A[q * mp + r] = jval[l];
        }
    }
    __syncthreads();
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int e = t; e < mp * mp; e += blockDim.x) {
            const double a = A[e];
            tot += a * a;
            if (e / mp != e % mp) off += a * a;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_down_sync(0xffffffffu, off, o);
            tot += __shfl_down_sync(0xffffffffu, tot, o);
        }
        if ((t & 31) == 0) { red[0][t >> 5] = off; red[1][t >> 5] = tot; }
        __syncthreads();
        if (t == 0) {
            double o2 = 0.0, t2 = 0.0;
            for (int x = 0; x < (int)(blockDim.x >> 5); x++) { o2 += red[0][x]; t2 += red[1][x]; }
            stop = !(o2 > 1e-30 * t2);
            if (sweep == 59 && !stop) atomicOr(bad, 1);
        }
        __syncthreads();
        if (stop) break;
        for (int rr = 0; rr < mp - 1; rr++) {
            if (t < h) {
                int p, q;
                if (t == 0) { p = mp - 1; q = rr; }
                else { p = (rr + t) % (mp - 1); q = (rr - t + mp - 1) % (mp - 1); }
                if (p > q) { const int x = p; p = q; q = x; }
                const double apq = A[p * mp + q];
                double c1 = 1.0, s1 = 0.0;
                if (apq != 0.0) {
                    // rotation angle as in Golub & Van Loan, Matrix Computations, sec. 8.5
                    const double th = (A[q * mp + q] - A[p * mp + p]) / (2.0 * apq);
                    const double at = fabs(th);
                    const double tt = at > 1e150 ? 0.5 / th : (th >= 0.0 ? 1.0 : -1.0) / (at + sqrt(th * th + 1.0));
                    c1 = 1.0 / sqrt(tt * tt + 1.0);
                    s1 = tt * c1;
                }
                pp[t] = p; qq[t] = q; cc[t] = c1; sn[t] = s1;
            }
            __syncthreads();
            for (int x = t; x < mp * h; x += blockDim.x) {   // columns: A <- A R, V <- V R
                const int k = x % mp, i = x / mp;
                const int p = pp[i], q = qq[i];
                const double c1 = cc[i], s1 = sn[i];
                const double ap = A[k * mp + p], aq = A[k * mp + q];
                A[k * mp + p] = c1 * ap - s1 * aq;
                A[k * mp + q] = s1 * ap + c1 * aq;
                const double vp = V[k * mp + p], vq = V[k * mp + q];
                V[k * mp + p] = c1 * vp - s1 * vq;
                V[k * mp + q] = s1 * vp + c1 * vq;
            }
            __syncthreads();
            for (int x = t; x < mp * h; x += blockDim.x) {   // rows: A <- R^T A
                const int k = x % mp, i = x / mp;
                const int p = pp[i], q = qq[i];
                const double c1 = cc[i], s1 = sn[i];
                const double ap = A[p * mp + k], aq = A[q * mp + k];
                A[p * mp + k] = c1 * ap - s1 * aq;
                A[q * mp + k] = s1 * ap + c1 * aq;
            }
            __syncthreads();
        }
    }
    for (int i = t; i < m; i += blockDim.x) w[n0 + i] = A[i * mp + i];
    for (int e = t; e < m * m; e += blockDim.x) {
        const int i = e / m, r = e % m;   // eigenvector i (column i of V), row r
        ev[evoff[c] + e] = V[r * mp + i];
    }
}

// C_c = the selected eigenvectors of configuration c: sel[cs_c + s] is the
// eigenvector index of CSF s; C[coff_c + s * m + r].
__global__ void k_csf_gather(const int64_t *__restrict__ conf_start, const int64_t *__restrict__ csf_start,
                             const int32_t *__restrict__ sel, const int64_t *__restrict__ evoff,
                             const int64_t *__restrict__ coff, const double *__restrict__ ev, double *C)
{
    const int c = blockIdx.x;
    const int m = (int)(conf_start[c + 1] - conf_start[c]);
    const int64_t s0 = csf_start[c];
    const int ns = (int)(csf_start[c + 1] - s0);
    for (int e = threadIdx.x; e < ns * m; e += blockDim.x) {
        const int s = e / m, r = e % m;
        C[coff[c] + e] = ev[evoff[c] + (int64_t)sel[s0 + s] * m + r];
    }
}

// Off-diagonal CSF columns of each row configuration: the CSFs of the
// adjacent configurations c2 < c1.
__global__ void k_csf_rowcount(const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj,
                               const int64_t *__restrict__ csf_start, int nc, int64_t *out)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c1 = warp; c1 < nc; c1 += nwarps) {
        int64_t s = 0;
        for (int64_t a = adj_ptr[c1] + lane; a < adj_ptr[c1 + 1]; a += 32) {
            const int c2 = adj[a];
            if (c2 < c1) s += csf_start[c2 + 1] - csf_start[c2];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) out[c1] = s;
    }
}

// H_csf rows of configuration c1 (one thread block): blocks C_c1^T H[c1, c2]
// C_c2 for the adjacent c2 <= c1 in ascending order.
__global__ void __launch_bounds__(256) k_csf_fill(const int64_t *__restrict__ conf_start,
                                                  const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj,
                                                  const int64_t *__restrict__ hrow, const int32_t *__restrict__ hcol,
                                                  const double *__restrict__ hval, const int64_t *__restrict__ csf_start,
                                                  const int64_t *__restrict__ coff, const double *__restrict__ C,
                                                  const int64_t *__restrict__ rowptr, int32_t *ocol, double *oval,
                                                  int maxm)
{
    const int c1 = blockIdx.x, t = threadIdx.x;
    const int64_t n0 = conf_start[c1];
    const int m1 = (int)(conf_start[c1 + 1] - n0);
    const int64_t cs1 = csf_start[c1];
    const int ns1 = (int)(csf_start[c1 + 1] - cs1);
    if (ns1 == 0 || m1 == 0) return;
    extern __shared__ double smf[];
    double *tile = smf;                           // m1 x m2 determinant block
    double *T = tile + (size_t)maxm * maxm;       // m1 x ns2
    int64_t *cur = reinterpret_cast<int64_t *>(T + (size_t)maxm * maxm);   // per-row cursor into the CSR
    const double *C1 = C + coff[c1];
    for (int r = t; r < m1; r += blockDim.x) cur[r] = hrow[n0 + r];
    int64_t colpos = 0;   // CSF columns written so far in each row of c1
    __syncthreads();
    for (int64_t a = adj_ptr[c1]; a < adj_ptr[c1 + 1]; a++) {
        const int c2 = adj[a];
        const int64_t k0 = conf_start[c2];
        const int m2 = (int)(conf_start[c2 + 1] - k0);
        const int64_t cs2 = csf_start[c2];
        const int ns2 = (int)(csf_start[c2 + 1] - cs2);
        const bool diag = c2 == c1;
        for (int e = t; e < m1 * m2; e += blockDim.x) tile[e] = 0.0;
        __syncthreads();
        for (int r = t; r < m1; r += blockDim.x) {
            int64_t l = cur[r];
            const int64_t l1 = hrow[n0 + r + 1];
            while (l < l1 && hcol[l] < k0 + m2) {
                const int64_t k = hcol[l];
                if (k >= k0) {
                    const int q = (int)(k - k0);
                    tile[r * m2 + q] = hval[l];
                    if (diag) tile[q * m2 + r] = hval[l];
                }
                l++;
            }
            cur[r] = l;
        }
        __syncthreads();
        if (ns2 > 0) {
            const double *C2 = C + coff[c2];
            for (int e = t; e < m1 * ns2; e += blockDim.x) {   // T = tile C2
                const int r = e / ns2, j = e % ns2;
                double s = 0.0;
                for (int q = 0; q < m2; q++) s += tile[r * m2 + q] * C2[(int64_t)j * m2 + q];
                T[r * ns2 + j] = s;
            }
            __syncthreads();
            for (int e = t; e < ns1 * ns2; e += blockDim.x) {   // B = C1^T T, written to the CSF rows
                const int i = e / ns2, j = e % ns2;
                if (diag && j > i) continue;
                double s = 0.0;
                for (int r = 0; r < m1; r++) s += C1[(int64_t)i * m1 + r] * T[r * ns2 + j];
                const int64_t pos = rowptr[cs1 + i] + colpos + j;
                ocol[pos] = (int32_t)(cs2 + j);
                oval[pos] = s;
            }
            colpos += ns2;
        }
        __syncthreads();
    }
}

// unsym: x[v * nd + n] = sum_s C_c[n - n0, s] y[v * ncsf + cs_c + s].
__global__ void k_csf_to_det(const int32_t *__restrict__ conf_of, const int64_t *__restrict__ conf_start,
                             const int64_t *__restrict__ csf_start, const int64_t *__restrict__ coff,
                             const double *__restrict__ C, const double *__restrict__ y, int64_t ncsf, int64_t nd,
                             int nv, double *x)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        const int c = conf_of[n];
        const int64_t n0 = conf_start[c];
        const int m = (int)(conf_start[c + 1] - n0), r = (int)(n - n0);
        const int64_t cs = csf_start[c];
        const int ns = (int)(csf_start[c + 1] - cs);
        for (int v = 0; v < nv; v++) {
            double s = 0.0;
            for (int i = 0; i < ns; i++) s += C[coff[c] + (int64_t)i * m + r] * y[(int64_t)v * ncsf + cs + i];
            x[(int64_t)v * nd + n] = s;
        }
    }
}

struct CsfBuf {
    void *p = nullptr;
    ~CsfBuf() { dev_free(p); }
};

}  // namespace

extern "C" {

int pci_gpu_form_csf(pci_gpu_t *h, int64_t *ncsf_out, int64_t *numh_out)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!h->have_basis) return set_err(h, PCI_E_STATE, "form_csf before set_basis");
    if (!h->H.rowptr || h->H.val_f32 || !h->h_from_tiles || h->H.nrows != h->nd || !h->d_adj)
        return set_err(h, PCI_E_STATE, "form_csf needs the FP64 determinant H of pci_gpu_form_h(64)");
    if (!h->J.rowptr) return set_err(h, PCI_E_STATE, "form_csf needs J^2 (pci_gpu_form_j)");
    const int nc = h->nc;
    int maxm = 1;
    for (int c = 0; c < nc; c++) maxm = std::max(maxm, (int)h->h_ndc[c]);
    if (maxm > CSF_MAX_NDC) return set_err(h, PCI_E_INPUT, "form_csf: a configuration has more than 112 determinants");
    int rc = 0;
    // jbasis: eigenpairs of every configuration's J^2 block
    std::vector<int64_t> evoff(nc + 1, 0), conf_start(nc + 1, 0);
    for (int c = 0; c < nc; c++) {
        conf_start[c + 1] = conf_start[c] + h->h_ndc[c];
        evoff[c + 1] = evoff[c] + (int64_t)h->h_ndc[c] * h->h_ndc[c];
    }
    CsfBuf d_evoff, d_w, d_ev, d_bad;
    d_evoff.p = dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) return rc;
    d_w.p = dev_alloc(h, std::max<int64_t>(h->nd, 1) * 8, &rc);
    if (rc) return rc;
    d_ev.p = dev_alloc(h, std::max<int64_t>(evoff[nc], 1) * 8, &rc);
    if (rc) return rc;
    d_bad.p = dev_alloc(h, 4, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_evoff.p, evoff.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(d_bad.p, 0, 4, h->st));
    const size_t smj = (size_t)2 * (maxm + 1) * (maxm + 1) * 8;
    PCI_CUDA(h, cudaFuncSetAttribute(k_csf_jblocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smj));
    k_csf_jblocks<<<nc, 256, smj, h->st>>>(h->d_conf_start, h->J.rowptr, h->J.col, (const double *)h->J.val,
                                           (const int64_t *)d_evoff.p, (double *)d_w.p, (double *)d_ev.p,
                                           (int *)d_bad.p);
    PCI_CUDA(h, cudaGetLastError());
    std::vector<double> w(h->nd);
    int bad = 0;
    PCI_CUDA(h, cudaMemcpyAsync(w.data(), d_w.p, h->nd * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(&bad, d_bad.p, 4, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    if (bad) return set_err(h, PCI_E_CUDA, "form_csf: Jacobi rotations of a J^2 block did not converge");
    // the eigenvectors with 2J = Mj (src/csf.f90:190-215)
    std::vector<int64_t> csf_start(nc + 1, 0), coff(nc + 1, 0);
    std::vector<int32_t> sel;
    for (int c = 0; c < nc; c++) {
        int ns = 0;
        for (int64_t i = 0; i < h->h_ndc[c]; i++) {
            const double tj = 0.5 * (sqrt(1.0 + w[conf_start[c] + i]) - 1.0);
            const int jtt = (int)(2 * tj + 0.0001);
            if (fabs(2 * tj - jtt) > 1e-7)
                return set_err(h, PCI_E_INPUT, "form_csf: J of a J^2 eigenvector is not integer or half-integer in "
                                                "configuration " + std::to_string(c + 1));
            if (jtt == h->mj) {
                sel.push_back((int32_t)i);
                ns++;
            }
        }
        csf_start[c + 1] = csf_start[c] + ns;
        coff[c + 1] = coff[c] + (int64_t)ns * h->h_ndc[c];
    }
    const int64_t ncsf = csf_start[nc];
    if (ncsf == 0) return set_err(h, PCI_E_INPUT, "form_csf: no configuration state has 2J = Mj");
    dev_free(h->d_csf_C); dev_free(h->d_csf_start); dev_free(h->d_csf_coff);
    h->d_csf_C = nullptr; h->d_csf_start = nullptr; h->d_csf_coff = nullptr;
    CsfBuf d_sel;
    d_sel.p = dev_alloc(h, std::max<size_t>(sel.size(), 1) * 4, &rc);
    if (rc) return rc;
    h->d_csf_start = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) return rc;
    h->d_csf_coff = (int64_t *)dev_alloc(h, (nc + 1) * 8, &rc);
    if (rc) return rc;
    h->d_csf_C = (double *)dev_alloc(h, std::max<int64_t>(coff[nc], 1) * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_sel.p, sel.data(), sel.size() * 4, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(h->d_csf_start, csf_start.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(h->d_csf_coff, coff.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, h->st));
    k_csf_gather<<<nc, 256, 0, h->st>>>(h->d_conf_start, h->d_csf_start, (const int32_t *)d_sel.p,
                                        (const int64_t *)d_evoff.p, h->d_csf_coff, (const double *)d_ev.p, h->d_csf_C);
    PCI_CUDA(h, cudaGetLastError());
    // formh_sym: row counts, row pointers, the blocks C1^T H C2
    CsfBuf d_cnt;
    d_cnt.p = dev_alloc(h, (size_t)nc * 8, &rc);
    if (rc) return rc;
    k_csf_rowcount<<<148 * 8, 256, 0, h->st>>>(h->d_adj_ptr, h->d_adj, h->d_csf_start, nc, (int64_t *)d_cnt.p);
    PCI_CUDA(h, cudaGetLastError());
    std::vector<int64_t> cnt(nc);
    PCI_CUDA(h, cudaMemcpyAsync(cnt.data(), d_cnt.p, (size_t)nc * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    std::vector<int64_t> rowptr(ncsf + 1, 0);
    for (int c = 0; c < nc; c++)
        for (int64_t i = 0; i < csf_start[c + 1] - csf_start[c]; i++)
            rowptr[csf_start[c] + i + 1] = rowptr[csf_start[c] + i] + cnt[c] + i + 1;
    const int64_t nnz = rowptr[ncsf];
    Csr out;
    out.nrows = ncsf;
    out.nnz = nnz;
    out.val_f32 = 0;
    out.rowptr = (int64_t *)dev_alloc(h, (ncsf + 1) * 8, &rc);
    if (rc) return rc;
    out.col = (int32_t *)dev_alloc(h, std::max<int64_t>(nnz, 1) * 4, &rc);
    if (rc) { csr_free(out); return rc; }
    out.val = dev_alloc(h, std::max<int64_t>(nnz, 1) * 8, &rc);
    if (rc) { csr_free(out); return rc; }
    PCI_CUDA(h, cudaMemcpyAsync(out.rowptr, rowptr.data(), (ncsf + 1) * 8, cudaMemcpyHostToDevice, h->st));
    const size_t smf = (size_t)2 * maxm * maxm * 8 + (size_t)maxm * 8;
    PCI_CUDA(h, cudaFuncSetAttribute(k_csf_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smf));
    k_csf_fill<<<nc, 256, smf, h->st>>>(h->d_conf_start, h->d_adj_ptr, h->d_adj, h->H.rowptr, h->H.col,
                                        (const double *)h->H.val, h->d_csf_start, h->d_csf_coff, h->d_csf_C,
                                        out.rowptr, out.col, (double *)out.val, maxm);
    PCI_CUDA(h, cudaGetLastError());
    // Hamil%minval of the CSF matrix
    double *d_min = nullptr;
    size_t tb = 0;
    cub::DeviceReduce::Min(nullptr, tb, (const double *)out.val, d_min, nnz, h->st);
    if ((rc = ensure_tmp(h, tb + 16))) { csr_free(out); return rc; }
    d_min = (double *)((char *)h->d_tmp + ((tb + 7) / 8) * 8);
    cub::DeviceReduce::Min(h->d_tmp, tb, (const double *)out.val, d_min, nnz, h->st);
    double hmin = 0.0;
    PCI_CUDA(h, cudaMemcpyAsync(&hmin, d_min, 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    // the CSF matrix takes the determinant matrix's place
    csr_retire(h, h->H);
    spare_release(h);
    csr_free(h->Hfull);
    h->H = out;
    h->h_from_tiles = false;
    h->h_pt_nd1 = -1;
    h->hmin = hmin;
    h->numh = nnz;
    h->h_csf_start = csf_start;
    h->ncsf = ncsf;
    if (ncsf_out) *ncsf_out = ncsf;
    if (numh_out) *numh_out = nnz;
    return PCI_OK;
}

int pci_gpu_csf_counts(pci_gpu_t *h, int32_t *per_conf)
{
    if (!h || !per_conf) return PCI_E_INPUT;
    if (h->ncsf == 0 || (int)h->h_csf_start.size() != h->nc + 1) return set_err(h, PCI_E_STATE, "no CSF basis");
    for (int c = 0; c < h->nc; c++) per_conf[c] = (int32_t)(h->h_csf_start[c + 1] - h->h_csf_start[c]);
    return PCI_OK;
}

int pci_gpu_csf_to_det(pci_gpu_t *h, const double *Y, int32_t nv, double *X)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    if (!Y || !X) return set_err(h, PCI_E_INPUT, "null array");
    if (h->ncsf == 0 || !h->d_csf_C) return set_err(h, PCI_E_STATE, "csf_to_det before form_csf");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "csf_to_det: nv must be 1..64");
    int rc = 0;
    CsfBuf d_y, d_x;
    d_y.p = dev_alloc(h, (size_t)h->ncsf * nv * 8, &rc);
    if (rc) return rc;
    d_x.p = dev_alloc(h, (size_t)h->nd * nv * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpyAsync(d_y.p, Y, (size_t)h->ncsf * nv * 8, cudaMemcpyHostToDevice, h->st));
    k_csf_to_det<<<148 * 8, 256, 0, h->st>>>(h->d_conf_of, h->d_conf_start, h->d_csf_start, h->d_csf_coff,
                                            h->d_csf_C, (const double *)d_y.p, h->ncsf, h->nd, nv, (double *)d_x.p);
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaMemcpyAsync(X, d_x.p, (size_t)h->nd * nv * 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    return PCI_OK;
}

}  // extern "C"
