// Second-order CI+PT energies (conf_pt's PTE, src/conf_pt.f90:751-952) on the
// resident determinant Hamiltonian.
//
// The reference loops over the determinants i of the PT space (beyond the
// Nd1 determinants of the CI space), forms the row H_ik against the first
// Nd0 determinants (its own FormH, conf_pt.f90:1319-1351), and accumulates
// x_in = sum_k H_ik X0_kn, dE_n += x_in^2 / del and c_in = x_in / del.  Here
// the whole list (CI + PT determinants) is one FormH matrix, so x = H X0 with
// X0 zero beyond Nd0 is one SpMM over all rows (rows beyond Nd1 see only
// columns below Nd0, and the Hmin shift of the SpMM vanishes there since X0
// is zero), and one thread per PT determinant forms its terms.  Energies and
// the denominator are in the engine's convention: del = E_n - H_ii with E_n
// the level's energy as an eigenvalue of H, so dE_n is negative for a lowest
// level (the reference's Ey(n), in its positive binding convention, is
// -dE_n) and c_in is the first-order coefficient x_in / (E_n - H_ii).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "pci_internal.h"

namespace {

struct PtBuf {
    void *p = nullptr;
    ~PtBuf() { dev_free(p); }
};

// Row-major X (nd x nv, zero beyond nd0) from column-major X0 (nd0 x nv).
__global__ void k_pt_pack(const double *__restrict__ x0, int64_t nd0, int nv, double *x)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nd0 * nv;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e % nd0;
        const int v = (int)(e / nd0);
        x[k * nv + v] = x0[e];
    }
}

// H_ii of the rows beyond nd1 (the last stored element of a lower-triangle
// row, when it is the diagonal; an exact zero is not stored).
__global__ void k_pt_diag(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col, const void *val,
                          int f32, int64_t nd1, int64_t nd, double *d)
{
    for (int64_t i = nd1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nd;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t l = rowptr[i + 1] - 1;
        double v = 0.0;
        if (l >= rowptr[i] && col[l] == i)
            v = f32 ? (double)((const float *)val)[l] : ((const double *)val)[l];
        d[i - nd1] = v;
    }
}

// average_diag (src/conf_pt.f90:710-724) for PT configuration c: the mean of
// its determinants' H_ii goes to the position the reference writes,
// Diag(n + kx) inside its k loop, which is the configuration's last
// determinant.
__global__ void k_pt_avg(const int64_t *__restrict__ conf_start, int c0, int nc, int64_t nd1, double *d)
{
    for (int c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int64_t a = conf_start[c], b = conf_start[c + 1];
        if (b == a) continue;
        double s = 0.0;
        for (int64_t i = a; i < b; i++) s += d[i - nd1];
        d[b - 1 - nd1] = s / (double)(b - a);
    }
}

// dE_v += y^2 / (E_v - H_ii) and c = y / (E_v - H_ii) for the PT rows lo..hi-1
// (d holds H_ii of rows nd1..Nd-1).
__global__ void __launch_bounds__(256) k_pt_terms(const double *__restrict__ y, const double *__restrict__ d,
                                                  const double *__restrict__ e, int64_t nd1, int64_t lo, int64_t hi,
                                                  int64_t nd, int nv, double *de, double *cpt)
{
    __shared__ double red[8][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double acc[64];
    for (int v = 0; v < nv; v++) acc[v] = 0.0;
    for (int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < hi;
         i += (int64_t)gridDim.x * blockDim.x) {
        for (int v = 0; v < nv; v++) {
            const double x = y[i * nv + v];
            const double del = e[v] - d[i - nd1];
            acc[v] += x * x / del;
            if (cpt) cpt[(int64_t)v * nd + i] = x / del;
        }
    }
    for (int v = 0; v < nv; v++) {
        double s = acc[v];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[w][v] = s;
    }
    __syncthreads();
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        double s = 0.0;
        for (int x = 0; x < (int)(blockDim.x >> 5); x++) s += red[x][v];
        atomicAdd(&de[v], s);
    }
}

// PTE's per-configuration sums (conf_pt.f90:871-872): for group g (rows
// grp[g]..grp[g+1]-1, clipped to lo..hi-1), dEg[g * nv + v] = sum of
// y^2 / (E_v - H_ii) and dVg[g * nv + v] = sum of (y / (E_v - H_ii))^2.  One
// thread block per group.
__global__ void __launch_bounds__(256) k_pt_groups(const double *__restrict__ y, const double *__restrict__ d,
                                                   const double *__restrict__ e, const int64_t *__restrict__ grp,
                                                   int ngrp, int64_t nd1, int64_t lo, int64_t hi, int nv, double *deg,
                                                   double *dvg)
{
    __shared__ double red[2][8][64];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int g = blockIdx.x; g < ngrp; g += gridDim.x) {
        const int64_t a = grp[g] > lo ? grp[g] : lo, b = grp[g + 1] < hi ? grp[g + 1] : hi;
        double ae[64], av[64];
        for (int v = 0; v < nv; v++) { ae[v] = 0.0; av[v] = 0.0; }
        for (int64_t i = a + threadIdx.x; i < b; i += blockDim.x) {
            for (int v = 0; v < nv; v++) {
                const double x = y[i * nv + v];
                const double del = e[v] - d[i - nd1];
                const double c = x / del;
                ae[v] += x * x / del;
                av[v] += c * c;
            }
        }
        for (int v = 0; v < nv; v++) {
            double s = ae[v], t = av[v];
            for (int o = 16; o > 0; o >>= 1) {
                s += __shfl_down_sync(0xffffffffu, s, o);
                t += __shfl_down_sync(0xffffffffu, t, o);
            }
            if (lane == 0) { red[0][w][v] = s; red[1][w][v] = t; }
        }
        __syncthreads();
        for (int v = threadIdx.x; v < nv; v += blockDim.x) {
            double s = 0.0, t = 0.0;
            for (int x = 0; x < (int)(blockDim.x >> 5); x++) { s += red[0][x][v]; t += red[1][x][v]; }
            deg[(int64_t)g * nv + v] = s;
            dvg[(int64_t)g * nv + v] = t;
        }
        __syncthreads();
    }
}

int pt2_impl(pci_gpu *h, int64_t nd1, int64_t nd0, const double *X0, int32_t nv, const double *E, int32_t avg_diag,
             const int64_t *grp, int32_t ngrp, double *dE, double *dEg, double *dVg, double *Xpt)
{
    if (!X0 || !E || !dE) return set_err(h, PCI_E_INPUT, "null array");
    if (!h->have_basis || !h->H.rowptr || h->H.nrows != h->nd)
        return set_err(h, PCI_E_STATE, "pt2 needs the determinant H of pci_gpu_form_h or pci_gpu_form_h_pt");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "pt2: nv must be 1..64");
    // conf_pt's Hmltn (conf_pt.f90:1353-1398) has no Gj J^2 term
    if (h->gj != 0.0) return set_err(h, PCI_E_INPUT, "pt2: H must be built with Gj = 0, as conf_pt's Hmltn");
    const int64_t nd = h->nd;
    if (nd0 < 1 || nd0 > nd1 || nd1 > nd) return set_err(h, PCI_E_INPUT, "pt2: need 1 <= Nd0 <= Nd1 <= Nd");
    // Nd1 and Nd0 end configurations (conf_pt.f90:669-676)
    std::vector<int64_t> cs(h->nc + 1, 0);
    for (int c = 0; c < h->nc; c++) cs[c + 1] = cs[c] + h->h_ndc[c];
    auto at_boundary = [&](int64_t n) { return std::binary_search(cs.begin(), cs.end(), n); };
    if (!at_boundary(nd1) || !at_boundary(nd0))
        return set_err(h, PCI_E_INPUT, "pt2: Nd1 and Nd0 must end a configuration");
    if (h->h_pt_nd1 >= 0 && (h->h_pt_nd1 != nd1 || h->h_pt_nd0 != nd0))
        return set_err(h, PCI_E_INPUT, "pt2: the resident PT block was built for another Nd1 / Nd0");
    const int cpt0 = (int)(std::lower_bound(cs.begin(), cs.end(), nd1) - cs.begin());   // first PT configuration
    if (ngrp < 0 || (ngrp > 0 && (!grp || !dEg || !dVg))) return set_err(h, PCI_E_INPUT, "pt2: bad groups");
    for (int g = 0; g < ngrp; g++)
        if (grp[g] < nd1 || grp[g + 1] < grp[g] || grp[g + 1] > nd)
            return set_err(h, PCI_E_INPUT, "pt2: groups must be ascending determinant offsets within Nd1..Nd");
    int rc = 0;
    PtBuf d_x0, d_x, d_y, d_d, d_e, d_de, d_c, d_grp, d_eg, d_vg;
    if (ngrp > 0) {
        d_grp.p = dev_alloc(h, (size_t)(ngrp + 1) * 8, &rc);
        if (rc) return rc;
        d_eg.p = dev_alloc(h, (size_t)ngrp * nv * 8, &rc);
        if (rc) return rc;
        d_vg.p = dev_alloc(h, (size_t)ngrp * nv * 8, &rc);
        if (rc) return rc;
    }
    d_x0.p = dev_alloc(h, (size_t)nd0 * nv * 8, &rc);
    if (rc) return rc;
    d_x.p = dev_alloc(h, (size_t)nd * nv * 8, &rc);
    if (rc) return rc;
    d_y.p = dev_alloc(h, (size_t)nd * nv * 8, &rc);
    if (rc) return rc;
    d_d.p = dev_alloc(h, (size_t)std::max<int64_t>(nd - nd1, 1) * 8, &rc);
    if (rc) return rc;
    d_e.p = dev_alloc(h, (size_t)nv * 8, &rc);
    if (rc) return rc;
    d_de.p = dev_alloc(h, (size_t)nv * 8, &rc);
    if (rc) return rc;
    if (Xpt) {
        d_c.p = dev_alloc(h, (size_t)nd * nv * 8, &rc);
        if (rc) return rc;
        PCI_CUDA(h, cudaMemsetAsync(d_c.p, 0, (size_t)nd * nv * 8, h->st));
    }
    cudaStream_t st = h->st;
    PCI_CUDA(h, cudaMemcpyAsync(d_x0.p, X0, (size_t)nd0 * nv * 8, cudaMemcpyHostToDevice, st));
    PCI_CUDA(h, cudaMemcpyAsync(d_e.p, E, (size_t)nv * 8, cudaMemcpyHostToDevice, st));
    PCI_CUDA(h, cudaMemsetAsync(d_x.p, 0, (size_t)nd * nv * 8, st));
    PCI_CUDA(h, cudaMemsetAsync(d_de.p, 0, (size_t)nv * 8, st));
    k_pt_pack<<<148 * 4, 256, 0, st>>>((const double *)d_x0.p, nd0, nv, (double *)d_x.p);
    PCI_CUDA(h, cudaGetLastError());
    for (int v0 = 0; v0 < nv; v0 += 16)   // the SpMM takes up to 16 vectors per call
        if ((rc = sp_spmm(h, (const double *)d_x.p + v0, nv, (double *)d_y.p + v0, nv, std::min(16, nv - v0), st)))
            return rc;
    if (nd > nd1) {
        k_pt_diag<<<148 * 4, 256, 0, st>>>(h->H.rowptr, h->H.col, h->H.val, h->H.val_f32, nd1, nd, (double *)d_d.p);
        PCI_CUDA(h, cudaGetLastError());
        if (avg_diag) {
            k_pt_avg<<<148, 256, 0, st>>>(h->d_conf_start, cpt0, h->nc, nd1, (double *)d_d.p);
            PCI_CUDA(h, cudaGetLastError());
        }
        // a PT block holds rows h_pt_lo..h_pt_hi-1 only; the others are another block's
        const bool blk = h->h_pt_nd1 >= 0;
        const int64_t lo = blk ? h->h_pt_lo : nd1, hi = blk ? h->h_pt_hi : nd;
        k_pt_terms<<<148 * 4, 256, 0, st>>>((const double *)d_y.p, (const double *)d_d.p, (const double *)d_e.p, nd1,
                                            lo, hi, nd, nv, (double *)d_de.p, Xpt ? (double *)d_c.p : nullptr);
        PCI_CUDA(h, cudaGetLastError());
        if (ngrp > 0) {
            PCI_CUDA(h, cudaMemcpyAsync(d_grp.p, grp, (size_t)(ngrp + 1) * 8, cudaMemcpyHostToDevice, st));
            k_pt_groups<<<std::min(ngrp, 148 * 8), 256, 0, st>>>((const double *)d_y.p, (const double *)d_d.p,
                                                                 (const double *)d_e.p, (const int64_t *)d_grp.p,
                                                                 ngrp, nd1, lo, hi, nv, (double *)d_eg.p,
                                                                 (double *)d_vg.p);
            PCI_CUDA(h, cudaGetLastError());
        }
    } else if (ngrp > 0) {
        PCI_CUDA(h, cudaMemsetAsync(d_eg.p, 0, (size_t)ngrp * nv * 8, st));
        PCI_CUDA(h, cudaMemsetAsync(d_vg.p, 0, (size_t)ngrp * nv * 8, st));
    }
    if (ngrp > 0) {
        PCI_CUDA(h, cudaMemcpyAsync(dEg, d_eg.p, (size_t)ngrp * nv * 8, cudaMemcpyDeviceToHost, st));
        PCI_CUDA(h, cudaMemcpyAsync(dVg, d_vg.p, (size_t)ngrp * nv * 8, cudaMemcpyDeviceToHost, st));
    }
    PCI_CUDA(h, cudaMemcpyAsync(dE, d_de.p, (size_t)nv * 8, cudaMemcpyDeviceToHost, st));
    if (Xpt) PCI_CUDA(h, cudaMemcpyAsync(Xpt, d_c.p, (size_t)nd * nv * 8, cudaMemcpyDeviceToHost, st));
    PCI_CUDA(h, cudaStreamSynchronize(st));
    return PCI_OK;
}

}  // namespace

extern "C" {

int pci_gpu_pt2(pci_gpu_t *h, int64_t nd1, int64_t nd0, const double *X0, int32_t nv, const double *E,
                int32_t avg_diag, double *dE, double *Xpt)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    return pt2_impl(h, nd1, nd0, X0, nv, E, avg_diag, nullptr, 0, dE, nullptr, nullptr, Xpt);
}

int pci_gpu_pt2_groups(pci_gpu_t *h, int64_t nd1, int64_t nd0, const double *X0, int32_t nv, const double *E,
                       int32_t avg_diag, const int64_t *grp, int32_t ngrp, double *dE, double *dEg, double *dVg,
                       double *Xpt)
{
    if (!h) return PCI_E_INPUT;
    cudaSetDevice(h->device);
    return pt2_impl(h, nd1, nd0, X0, nv, E, avg_diag, grp, ngrp, dE, dEg, dVg, Xpt);
}

}  // extern "C"
