// Sparse products of the Davidson loop: Y = (H - Hmin I) X over a block of
// vectors (Mxmpy, src/davidson.f90:572-647) and <x|J^2|x> (J_av,
// src/formj2.f90:355-387).
//
// The reference stores the lower triangle and scatters the transpose part
// (y_k += H_nk x_n) one vector at a time, with an Allreduce per vector.  Here
// the SpMM works on all Nlv vectors at once from a full symmetric CSR built
// once on the device from the lower triangle, so each output row is one
// warp-private gather with no atomics: a group of NV lanes owns one stored
// element, lane v multiplies x_k[v] (one coalesced read of the NV-wide row of
// X), and the groups are reduced with shuffles at the end of the row.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pci_internal.h"

#define FULL_MASK 0xffffffffu

void csr_free(Csr &c)
{
    dev_free(c.rowptr);
    dev_free(c.col);
    dev_free(c.val);
    c.rowptr = nullptr;
    c.col = nullptr;
    c.val = nullptr;
    c.nrows = c.nnz = 0;
}

void spare_release(pci_gpu *h)
{
    dev_free(h->spare.rowptr);
    dev_free(h->spare.col);
    dev_free(h->spare.val);
    h->spare = pci_gpu::Spare();
}

size_t spare_bytes(const pci_gpu *h)
{
    return h->spare.rowptr_bytes + h->spare.col_bytes + h->spare.val_bytes;
}

void csr_retire(pci_gpu *h, Csr &c)
{
    if (!c.col) {
        csr_free(c);
        return;
    }
    spare_release(h);
    const int64_t slots = std::max(c.cap, c.nnz);
    h->spare.rowptr = c.rowptr;
    h->spare.rowptr_bytes = c.rowptr ? (size_t)(c.nrows + 1) * 8 : 0;
    h->spare.col = c.col;
    h->spare.col_bytes = (size_t)slots * 4;
    h->spare.val = c.val;
    h->spare.val_bytes = (size_t)slots * (c.val_f32 ? 4 : 8);
    c = Csr();
}

void *spare_take(pci_gpu *h, int which, size_t bytes)
{
    void **p = which == 0 ? &h->spare.rowptr : which == 1 ? &h->spare.col : &h->spare.val;
    size_t *n = which == 0 ? &h->spare.rowptr_bytes : which == 1 ? &h->spare.col_bytes : &h->spare.val_bytes;
    // reused only when at most about twice the size asked for
    if (!*p || *n < bytes || *n > 2 * bytes + ((size_t)64 << 20)) return nullptr;
    void *r = *p;
    *p = nullptr;
    *n = 0;
    return r;
}

// --------------------------------------------------------- full CSR ---

__global__ void k_count_upper(const int64_t *rowptr, const int32_t *col, int64_t nd, unsigned int *cntU)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n = warp; n < nd; n += nwarps) {
        for (int64_t l = rowptr[n] + lane; l < rowptr[n + 1]; l += 32) {
            int k = col[l];
            if (k != n) atomicAdd(&cntU[k], 1u);
        }
    }
}

__global__ void k_full_counts(const int64_t *rowptr, const unsigned int *cntU, int64_t nd, int64_t *fullcnt)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        fullcnt[n] = (rowptr[n + 1] - rowptr[n]) + cntU[n];
}

template <typename VT>
__global__ void k_full_fill(const int64_t *rowptr, const int32_t *col, const VT *val, int64_t nd,
                            const int64_t *frow, unsigned int *cursor, int32_t *fcol, VT *fval)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n = warp; n < nd; n += nwarps) {
        int64_t r0 = rowptr[n], r1 = rowptr[n + 1];
        int64_t f0 = frow[n];
        for (int64_t l = r0 + lane; l < r1; l += 32) {
            int k = col[l];
            VT v = val[l];
            fcol[f0 + (l - r0)] = k;   // lower part keeps its order
            fval[f0 + (l - r0)] = v;
            if (k != n) {
                int64_t lowk = rowptr[k + 1] - rowptr[k];
                int64_t p = frow[k] + lowk + atomicAdd(&cursor[k], 1u);
                fcol[p] = (int32_t)n;
                fval[p] = v;
            }
        }
    }
}

int sp_build_full(pci_gpu *h)
{
    if (h->Hfull.rowptr) return PCI_OK;
    Csr &L = h->H;
    if (!L.rowptr) return set_err(h, PCI_E_STATE, "no Hamiltonian resident");
    int rc = 0;
    const int64_t nd = L.nrows;
    unsigned int *cntU = (unsigned int *)dev_alloc(h, nd * 4 + 16, &rc);
    if (rc) return rc;
    int64_t *fullcnt = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemsetAsync(cntU, 0, nd * 4, h->st));
    k_count_upper<<<148 * 16, 256, 0, h->st>>>(L.rowptr, L.col, nd, cntU);
    k_full_counts<<<148 * 4, 256, 0, h->st>>>(L.rowptr, cntU, nd, fullcnt);
    Csr &F = h->Hfull;
    F.nrows = nd;
    F.val_f32 = L.val_f32;
    F.rowptr = (int64_t *)dev_alloc(h, (nd + 1) * 8, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemsetAsync(F.rowptr, 0, 8, h->st));
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, fullcnt, F.rowptr + 1, nd, h->st);
    if ((rc = ensure_tmp(h, tb))) return rc;
    cub::DeviceScan::InclusiveSum(h->d_tmp, tb, fullcnt, F.rowptr + 1, nd, h->st);
    PCI_CUDA(h, cudaMemcpyAsync(&F.nnz, F.rowptr + nd, 8, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    size_t vs = F.val_f32 ? 4 : 8;
    F.col = (int32_t *)dev_alloc(h, F.nnz * 4, &rc);
    if (rc) return rc;
    F.val = dev_alloc(h, F.nnz * vs, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemsetAsync(cntU, 0, nd * 4, h->st));
    if (F.val_f32) {
        k_full_fill<float><<<148 * 16, 256, 0, h->st>>>(L.rowptr, L.col, (const float *)L.val, nd, F.rowptr, cntU,
                                                        F.col, (float *)F.val);
    } else {
        k_full_fill<double><<<148 * 16, 256, 0, h->st>>>(L.rowptr, L.col, (const double *)L.val, nd, F.rowptr, cntU,
                                                         F.col, (double *)F.val);
    }
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    dev_free(cntU);
    dev_free(fullcnt);
    return PCI_OK;
}

// ------------------------------------------------------------- SpMM ---

// One warp per row; NV lanes per stored element, 32/NV elements per step.
template <int NV, typename VT, typename XT>
__global__ void __launch_bounds__(256) k_spmm(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                                               const VT *__restrict__ val, int64_t nd, double hmin,
                                               const XT *__restrict__ X, int ldx, XT *__restrict__ Y, int ldy)
{
    constexpr int G = 32 / NV;
    const int lane = threadIdx.x & 31;
    const int g = lane / NV, v = lane - g * NV;
    const bool active = g < G;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n = warp; n < nd; n += nwarps) {
        const int64_t r0 = rowptr[n], r1 = rowptr[n + 1];
        XT acc = 0;
        if (active) {
            int64_t l = r0 + g;
            for (; l + 3 * G < r1; l += 4 * G) {
                int k0 = __ldg(&col[l]), k1 = __ldg(&col[l + G]), k2 = __ldg(&col[l + 2 * G]), k3 = __ldg(&col[l + 3 * G]);
                XT t0 = (XT)__ldg(&val[l]), t1 = (XT)__ldg(&val[l + G]), t2 = (XT)__ldg(&val[l + 2 * G]),
                   t3 = (XT)__ldg(&val[l + 3 * G]);
                if (k0 == n) t0 -= (XT)hmin;
                if (k1 == n) t1 -= (XT)hmin;
                if (k2 == n) t2 -= (XT)hmin;
                if (k3 == n) t3 -= (XT)hmin;
                XT x0 = __ldg(&X[(int64_t)k0 * ldx + v]), x1 = __ldg(&X[(int64_t)k1 * ldx + v]);
                XT x2 = __ldg(&X[(int64_t)k2 * ldx + v]), x3 = __ldg(&X[(int64_t)k3 * ldx + v]);
                acc += t0 * x0;
                acc += t1 * x1;
                acc += t2 * x2;
                acc += t3 * x3;
            }
            for (; l < r1; l += G) {
                int k = __ldg(&col[l]);
                XT t = (XT)__ldg(&val[l]);
                if (k == n) t -= (XT)hmin;
                acc += t * __ldg(&X[(int64_t)k * ldx + v]);
            }
        }
#pragma unroll
        for (int gg = 1; gg < G; gg++) {
            XT o = __shfl_sync(FULL_MASK, acc, (lane + gg * NV) & 31);
            if (g == 0) acc += o;
        }
        if (g == 0) Y[n * (int64_t)ldy + v] = acc;
    }
}

// --------------------------------------------- lower-triangle SpMM ---
//
// Y += (H - hmin I) X from the stored lower triangle alone, for matrices too
// large to hold twice.  One warp owns 32 consecutive rows (lane = row) and
// walks the union of their sorted column lists in windows of WIN columns:
// each lane consumes its row's entries inside the window, adding h x_k to a
// register accumulator (row part) and h x_n into a shared-memory window
// buffer (transpose part, k != n).  At the end of a window the buffer goes to
// Y with one global atomic per (column, vector); the row accumulators go to Y
// once at the end.  Rows of one configuration share their column structure,
// so a window collects many transpose contributions per atomic.  Y must be
// zero on entry.
constexpr int LW_ROWS = 32;
constexpr int LW_WIN = 32;
constexpr int LW_WARPS = 4;

// Transpose contributions inside a window are summed in shared memory as
// 64-bit fixed point (scale 2^55, |window sum| < 256): integer atomics are
// exact, so the window sums do not depend on the order lanes arrive in.
constexpr double LW_SCALE = 36028797018963968.0;  // 2^55

template <int NV, typename VT, typename XT>
__global__ void __launch_bounds__(LW_WARPS * 32) k_spmm_lower(const int64_t *__restrict__ rowptr,
                                                               const int32_t *__restrict__ col,
                                                               const VT *__restrict__ val, int64_t nd, double hmin,
                                                               const XT *__restrict__ X, int ldx, XT *Y,
                                                               int ldy, unsigned long long *counter)
{
    __shared__ unsigned long long tbuf[LW_WARPS][LW_WIN * NV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long *tb = tbuf[w];
    const int64_t nitems = (nd + LW_ROWS - 1) / LW_ROWS;
    for (int i = lane; i < LW_WIN * NV; i += 32) tb[i] = 0ULL;
    __syncwarp();
    while (true) {
        unsigned long long it = 0;
        if (lane == 0) it = atomicAdd(counter, 1ULL);
        it = __shfl_sync(FULL_MASK, it, 0);
        if (it >= (unsigned long long)nitems) break;
        const int64_t n = (int64_t)it * LW_ROWS + lane;
        const bool mine = n < nd;
        int64_t cur = mine ? rowptr[n] : 0, end = mine ? rowptr[n + 1] : 0;
        XT xn[NV], acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
            xn[v] = mine ? X[n * ldx + v] : (XT)0;
            acc[v] = (XT)0;
        }
        int ck = cur < end ? __ldg(&col[cur]) : INT_MAX;
        while (true) {
            int wmin = ck;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) wmin = min(wmin, __shfl_xor_sync(FULL_MASK, wmin, o));
            if (wmin == INT_MAX) break;
            const int wend = wmin + LW_WIN;
            while (ck < wend) {
                const XT h0 = (XT)__ldg(&val[cur]);
                const XT h = ck == n ? h0 - (XT)hmin : h0;
                const XT *xk = X + (int64_t)ck * ldx;
#pragma unroll
                for (int v = 0; v < NV; v++) acc[v] += h * __ldg(&xk[v]);
                if (ck != n) {
                    unsigned long long *t = tb + (ck - wmin) * NV;
#pragma unroll
                    for (int v = 0; v < NV; v++)
                        atomicAdd(&t[v], (unsigned long long)__double2ll_rn((double)(h * xn[v]) * LW_SCALE));
                }
                cur++;
                ck = cur < end ? __ldg(&col[cur]) : INT_MAX;
            }
            __syncwarp();
            for (int i = lane; i < LW_WIN * NV; i += 32) {
                const long long q = (long long)tb[i];
                if (q != 0) {
                    const int64_t k = wmin + i / NV;
                    atomicAdd(&Y[k * ldy + (i % NV)], (XT)((double)q / LW_SCALE));
                    tb[i] = 0ULL;
                }
            }
            __syncwarp();
        }
        if (mine)
#pragma unroll
            for (int v = 0; v < NV; v++) atomicAdd(&Y[n * ldy + v], acc[v]);
    }
}

// ------------------------------- lower-triangle SpMM along the tiles ---
//
// Same product, for an H built here: its rows are grouped by configuration
// and every stored element lies in a tile (c1, c2) of adjacent
// configurations, columns ascending tile by tile.  One warp takes up to 32
// rows of one configuration c1 (lane = row) and walks c1's adjacency list:
// for each tile the lanes consume their row's entries inside c2's column
// range, the row part into registers and the transpose part into a
// shared-memory buffer of c2's columns (64-bit fixed point, as above), which
// goes to Y with one global atomic per touched (column, vector) per tile.
// All rows of a configuration share the tile sequence, so the buffer
// collects every row's contribution to a column before its one atomic.
constexpr int LT_WARPS = 8;
constexpr int LT_WIN = 64;   // columns of a tile per buffer flush
constexpr int LT_ROWS = 32;

template <int NV, typename VT, typename XT>
__global__ void __launch_bounds__(LT_WARPS * 32) k_spmm_lower_tiles(
    const int64_t *__restrict__ rowptr, const int32_t *__restrict__ col, const VT *__restrict__ val, double hmin,
    const int64_t *__restrict__ conf_start, const int64_t *__restrict__ adj_ptr, const int32_t *__restrict__ adj,
    const int2 *__restrict__ items, int64_t nitems, const XT *__restrict__ X, int ldx, XT *Y, int ldy,
    unsigned long long *counter)
{
    extern __shared__ unsigned long long lt_smem[];
    const int lane = threadIdx.x & 31;
    unsigned long long *tb = lt_smem + (size_t)(threadIdx.x >> 5) * LT_WIN * NV;
    for (int i = lane; i < LT_WIN * NV; i += 32) tb[i] = 0ULL;
    __syncwarp();
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(counter, 1ULL);
        t = __shfl_sync(FULL_MASK, t, 0);
        if (t >= (unsigned long long)nitems) break;
        const int2 it = items[t];
        const int c1 = it.x;
        const int64_t cend = conf_start[c1 + 1];
        const int64_t n = conf_start[c1] + it.y + lane;
        const bool mine = n < cend && lane < LT_ROWS;
        int64_t cur = mine ? rowptr[n] : 0;
        const int64_t end = mine ? rowptr[n + 1] : 0;
        XT xn[NV], acc[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
            xn[v] = mine ? X[n * ldx + v] : (XT)0;
            acc[v] = (XT)0;
        }
        int ck = cur < end ? __ldg(&col[cur]) : INT_MAX;
        // an element outside the tile being walked (not produced by this
        // build) goes straight to Y
        auto direct = [&]() {
            const XT h0 = (XT)__ldg(&val[cur]);
            const XT h = ck == n ? h0 - (XT)hmin : h0;
#pragma unroll
            for (int v = 0; v < NV; v++) {
                acc[v] += h * __ldg(&X[(int64_t)ck * ldx + v]);
                if (ck != n) atomicAdd(&Y[(int64_t)ck * ldy + v], h * xn[v]);
            }
            cur++;
            ck = cur < end ? __ldg(&col[cur]) : INT_MAX;
        };
        const int64_t a1 = adj_ptr[c1 + 1];
        for (int64_t a = adj_ptr[c1]; a < a1; a++) {
            const int c2 = adj[a];
            const int64_t k0 = conf_start[c2], k1 = conf_start[c2 + 1];
            for (int64_t w0 = k0; w0 < k1; w0 += LT_WIN) {
                const int64_t w1 = min(k1, w0 + LT_WIN);
                while (ck < w0) direct();
                while (ck < w1) {
                    const XT h0 = (XT)__ldg(&val[cur]);
                    const XT h = ck == n ? h0 - (XT)hmin : h0;
                    const XT *xk = X + (int64_t)ck * ldx;
#pragma unroll
                    for (int v = 0; v < NV; v++) acc[v] += h * __ldg(&xk[v]);
                    if (ck != n) {
                        unsigned long long *tt = tb + (ck - w0) * NV;
#pragma unroll
                        for (int v = 0; v < NV; v++)
                            atomicAdd(&tt[v], (unsigned long long)__double2ll_rn((double)(h * xn[v]) * LW_SCALE));
                    }
                    cur++;
                    ck = cur < end ? __ldg(&col[cur]) : INT_MAX;
                }
                __syncwarp();
                const int nw = (int)(w1 - w0) * NV;
                for (int i = lane; i < nw; i += 32) {
                    const long long q = (long long)tb[i];
                    if (q != 0) {
                        atomicAdd(&Y[(w0 + i / NV) * ldy + (i % NV)], (XT)((double)q / LW_SCALE));
                        tb[i] = 0ULL;
                    }
                }
                __syncwarp();
            }
        }
        while (ck != INT_MAX) direct();
        if (mine)
#pragma unroll
            for (int v = 0; v < NV; v++) atomicAdd(&Y[n * ldy + v], acc[v]);
    }
}

// ------------------------- lower-triangle SpMM with transpose reductions ---
//
// Same product, one warp per row with NV lanes per stored element (as the
// full-copy kernel): the row part accumulates in registers and is reduced
// across the element groups at the row's end; the transpose part of every
// element goes to Y with a global reduction (no return value) per vector.
// The columns of one row are distinct, so a warp never reduces twice into
// one address in a step; rows of other warps meet in L2.
template <int NV, typename VT, typename XT>
__global__ void __launch_bounds__(256) k_spmm_lower_red(const int64_t *__restrict__ rowptr,
                                                         const int32_t *__restrict__ col,
                                                         const VT *__restrict__ val, int64_t nd, double hmin,
                                                         const XT *__restrict__ X, int ldx, XT *Y, int ldy)
{
    constexpr int G = 32 / NV;
    const int lane = threadIdx.x & 31;
    const int g = lane / NV, v = lane - g * NV;
    const bool active = g < G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n = warp; n < nd; n += nwarps) {
        const int64_t r0 = rowptr[n], r1 = rowptr[n + 1];
        const XT xn = active ? __ldg(&X[n * (int64_t)ldx + v]) : (XT)0;
        XT acc = 0;
        if (active) {
            int64_t l = r0 + g;
            // four elements per step: their loads are issued before any use
            for (; l + 3 * G < r1; l += 4 * G) {
                int k[4];
                XT t[4], xk[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    k[u] = __ldg(&col[l + u * G]);
                    t[u] = (XT)__ldg(&val[l + u * G]);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) xk[u] = __ldg(&X[(int64_t)k[u] * ldx + v]);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (k[u] == n) {
                        t[u] -= (XT)hmin;
                    } else {
                        atomicAdd(&Y[(int64_t)k[u] * ldy + v], t[u] * xn);
                    }
                    acc += t[u] * xk[u];
                }
            }
            for (; l < r1; l += G) {
                const int k = __ldg(&col[l]);
                XT t = (XT)__ldg(&val[l]);
                if (k == n) {
                    t -= (XT)hmin;
                } else {
                    atomicAdd(&Y[(int64_t)k * ldy + v], t * xn);
                }
                acc += t * __ldg(&X[(int64_t)k * ldx + v]);
            }
        }
#pragma unroll
        for (int gg = 1; gg < G; gg++) {
            XT o = __shfl_sync(FULL_MASK, acc, (lane + gg * NV) & 31);
            if (g == 0) acc += o;
        }
        if (g == 0) atomicAdd(&Y[n * (int64_t)ldy + v], acc);
    }
}

template <typename VT, typename XT>
static int spmm_lower_red_dispatch(pci_gpu *h, const XT *X, int ldx, XT *Y, int ldy, int nv, cudaStream_t st);

template <typename XT>
__global__ void k_zero_block(XT *Y, int ldy, int64_t nd, int nv)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nd * nv; i += (int64_t)gridDim.x * blockDim.x)
        Y[(i / nv) * ldy + (i % nv)] = (XT)0;
}

// Work items of the tile kernel: (configuration, first row) chunks of up to
// LT_ROWS rows, heaviest first (determinant pairs per row x rows).
static void lower_tile_items(const pci_gpu *h, std::vector<int2> &items)
{
    std::vector<std::pair<double, int2>> tmp;
    for (int c = 0; c < h->nc; c++) {
        const int nr = h->h_ndc[c];
        const double w = c < (int)h->h_rowwork.size() ? (double)h->h_rowwork[c] : 1.0;
        for (int r = 0; r < nr; r += LT_ROWS) tmp.push_back({w * std::min(LT_ROWS, nr - r), make_int2(c, r)});
    }
    std::stable_sort(tmp.begin(), tmp.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
    items.resize(tmp.size());
    for (size_t i = 0; i < tmp.size(); i++) items[i] = tmp[i].second;
}

template <typename VT, typename XT>
static int spmm_lower_tiles_dispatch(pci_gpu *h, const XT *X, int ldx, XT *Y, int ldy, int nv, cudaStream_t st)
{
    const Csr &L = h->H;
    std::vector<int2> items;
    lower_tile_items(h, items);
    int rc = 0;
    if ((rc = ensure_tmp(h, 64 + items.size() * sizeof(int2)))) return rc;
    unsigned long long *counter = (unsigned long long *)h->d_tmp;
    int2 *d_items = (int2 *)((char *)h->d_tmp + 64);
    PCI_CUDA(h, cudaMemsetAsync(counter, 0, 8, st));
    PCI_CUDA(h, cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    k_zero_block<<<148 * 8, 256, 0, st>>>(Y, ldy, L.nrows, nv);
    const VT *val = (const VT *)L.val;
    const int64_t nit = (int64_t)items.size();
#define CASE(N)                                                                                                 \
    case N: {                                                                                                   \
        auto kf = k_spmm_lower_tiles<N, VT, XT>;                                                                \
        const int smem = LT_WARPS * LT_WIN * N * 8;                                                             \
        cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);                            \
        int per_sm = 1;                                                                                         \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, LT_WARPS * 32, smem);                        \
        kf<<<148 * std::max(per_sm, 1), LT_WARPS * 32, smem, st>>>(L.rowptr, L.col, val, h->hmin, h->d_conf_start, \
                                                                  h->d_adj_ptr, h->d_adj, d_items, nit, X, ldx, Y, \
                                                                  ldy, counter);                                 \
        break;                                                                                                  \
    }
    switch (nv) {
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
        CASE(9) CASE(10) CASE(11) CASE(12) CASE(13) CASE(14) CASE(15) CASE(16)
    default: return set_err(h, PCI_E_INPUT, "SpMM supports 1..16 vectors");
    }
#undef CASE
    PCI_CUDA(h, cudaGetLastError());
    return PCI_OK;
}

template <typename VT, typename XT>
static int spmm_lower_dispatch(pci_gpu *h, const XT *X, int ldx, XT *Y, int ldy, int nv, cudaStream_t st)
{
    const Csr &L = h->H;
    // Default: warp per row with global reductions for the transpose part.
    // Measured per call (10 vectors): 279 ms FP64 / 178 ms FP32 on config 2
    // against 795 / 736 ms for the window kernel and 930 ms for the tile
    // walk; 8.2 / 3.2 ms on the 86k-determinant system against 43 / 41 ms.
    // PCI_SPMM_LOWER=windows|tiles selects the others (the tile walk needs
    // the adjacency of an H built here).
    const char *e = getenv("PCI_SPMM_LOWER");
    if (e && !strcmp(e, "tiles") && h->h_from_tiles && h->d_adj && h->have_basis)
        return spmm_lower_tiles_dispatch<VT, XT>(h, X, ldx, Y, ldy, nv, st);
    if (!(e && !strcmp(e, "windows"))) return spmm_lower_red_dispatch<VT, XT>(h, X, ldx, Y, ldy, nv, st);
    int rc = 0;
    if ((rc = ensure_tmp(h, 64))) return rc;
    unsigned long long *counter = (unsigned long long *)h->d_tmp;
    PCI_CUDA(h, cudaMemsetAsync(counter, 0, 8, st));
    k_zero_block<<<148 * 8, 256, 0, st>>>(Y, ldy, L.nrows, nv);
    const int blocks = 148 * 8;
    const VT *val = (const VT *)L.val;
#define CASE(N)                                                                                           \
    case N:                                                                                               \
        k_spmm_lower<N, VT, XT><<<blocks, LW_WARPS * 32, 0, st>>>(L.rowptr, L.col, val, L.nrows, h->hmin, \
                                                                      X, ldx, Y, ldy, counter);           \
        break;
    switch (nv) {
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
        CASE(9) CASE(10) CASE(11) CASE(12) CASE(13) CASE(14) CASE(15) CASE(16)
    default: return set_err(h, PCI_E_INPUT, "SpMM supports 1..16 vectors");
    }
#undef CASE
    PCI_CUDA(h, cudaGetLastError());
    return PCI_OK;
}

template <typename VT, typename XT>
static int spmm_lower_red_dispatch(pci_gpu *h, const XT *X, int ldx, XT *Y, int ldy, int nv, cudaStream_t st)
{
    const Csr &L = h->H;
    k_zero_block<<<148 * 8, 256, 0, st>>>(Y, ldy, L.nrows, nv);
    const VT *val = (const VT *)L.val;
    // 4 thread blocks per SM (measured 1.5% faster than 16 on config 2)
#define CASE(N)                                                                                               \
    case N:                                                                                                   \
        k_spmm_lower_red<N, VT, XT><<<148 * 4, 256, 0, st>>>(L.rowptr, L.col, val, L.nrows, h->hmin, X, ldx, Y, ldy); \
        break;
    switch (nv) {
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
        CASE(9) CASE(10) CASE(11) CASE(12) CASE(13) CASE(14) CASE(15) CASE(16)
    default: return set_err(h, PCI_E_INPUT, "SpMM supports 1..16 vectors");
    }
#undef CASE
    PCI_CUDA(h, cudaGetLastError());
    return PCI_OK;
}

template <typename VT, typename XT>
static int spmm_dispatch(pci_gpu *h, const XT *X, int ldx, XT *Y, int ldy, int nv, cudaStream_t st)
{
    Csr &F = h->Hfull;
    const VT *val = (const VT *)F.val;
    int blocks = 148 * 16;
    double hm = h->hmin;
#define CASE(N) \
    case N: k_spmm<N, VT, XT><<<blocks, 256, 0, st>>>(F.rowptr, F.col, val, F.nrows, hm, X, ldx, Y, ldy); break;
    switch (nv) {
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
        CASE(9) CASE(10) CASE(11) CASE(12) CASE(13) CASE(14) CASE(15) CASE(16)
    default: return set_err(h, PCI_E_INPUT, "SpMM supports 1..16 vectors");
    }
#undef CASE
    PCI_CUDA(h, cudaGetLastError());
    return PCI_OK;
}

// The full symmetric copy is used when it fits beside everything else on the
// device (or PCI_SPMM=full); otherwise the lower-triangle kernel (or PCI_SPMM=lower).
static bool use_lower(pci_gpu *h)
{
    if (h->spmm_mode == 2) return true;
    if (h->spmm_mode == 1 || h->Hfull.rowptr) return false;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const size_t vs = h->H.val_f32 ? 4 : 8;
    const size_t need = (size_t)(2 * h->H.nnz) * (4 + vs) + (size_t)(h->H.nrows + 1) * 16;
    return need + ((size_t)2 << 30) > fr;
}

int sp_spmm(pci_gpu *h, const double *X, int ldx, double *Y, int ldy, int nv, cudaStream_t st)
{
    if (use_lower(h)) {
        h->spmm_lower_used = 1;
        return h->H.val_f32 ? spmm_lower_dispatch<float, double>(h, X, ldx, Y, ldy, nv, st)
                            : spmm_lower_dispatch<double, double>(h, X, ldx, Y, ldy, nv, st);
    }
    h->spmm_lower_used = 0;
    int rc = sp_build_full(h);
    if (rc) return rc;
    if (h->Hfull.val_f32) return spmm_dispatch<float, double>(h, X, ldx, Y, ldy, nv, st);
    return spmm_dispatch<double, double>(h, X, ldx, Y, ldy, nv, st);
}

int sp_spmm_f32(pci_gpu *h, const float *X, int ldx, float *Y, int ldy, int nv, cudaStream_t st)
{
    if (use_lower(h)) {
        h->spmm_lower_used = 1;
        return h->H.val_f32 ? spmm_lower_dispatch<float, float>(h, X, ldx, Y, ldy, nv, st)
                            : spmm_lower_dispatch<double, float>(h, X, ldx, Y, ldy, nv, st);
    }
    h->spmm_lower_used = 0;
    int rc = sp_build_full(h);
    if (rc) return rc;
    if (h->Hfull.val_f32) return spmm_dispatch<float, float>(h, X, ldx, Y, ldy, nv, st);
    return spmm_dispatch<double, float>(h, X, ldx, Y, ldy, nv, st);
}

// ------------------------------------------------------------- J_av ---

// sums[v] += sum over stored (n, k), n,k < nlim, of t x_k x_n (doubled off the
// diagonal); element (n, v) of X is X[n*sn + v*sv].
__global__ void k_jav(const int64_t *rowptr, const int32_t *col, const double *val, int64_t nlim,
                      const double *X, int64_t sn, int64_t sv, int nv, double *sums)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int v = 0; v < nv; v++) {
        double acc = 0.0;
        for (int64_t n = warp; n < nlim; n += nwarps) {
            double xn = X[n * sn + v * sv];
            for (int64_t l = rowptr[n] + lane; l < rowptr[n + 1]; l += 32) {
                int k = col[l];
                if (k < nlim) {
                    double r = val[l] * X[(int64_t)k * sn + v * sv] * xn;
                    if (k != n) r = r + r;
                    acc += r;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL_MASK, acc, o);
        if (lane == 0) atomicAdd(&sums[v], acc);
    }
}

int sp_jav_strided(pci_gpu *h, const double *X, int64_t sn, int64_t sv, int nv, int64_t nlim, double *out_host)
{
    if (!h->J.rowptr) return set_err(h, PCI_E_STATE, "J^2 not formed");
    if (nv < 1 || nv > 64) return set_err(h, PCI_E_INPUT, "J_av: nv must be 1..64");
    if (nlim < 0 || nlim > h->J.nrows) return set_err(h, PCI_E_INPUT, "J_av: nlim outside 0..Nd");
    int rc = 0;
    if ((rc = ensure_tmp(h, 8 * 64))) return rc;
    double *sums = (double *)h->d_tmp;
    PCI_CUDA(h, cudaMemsetAsync(sums, 0, 8 * nv, h->st));
    k_jav<<<148 * 4, 256, 0, h->st>>>(h->J.rowptr, h->J.col, (const double *)h->J.val, nlim, X, sn, sv, nv, sums);
    PCI_CUDA(h, cudaGetLastError());
    std::vector<double> s(nv);
    PCI_CUDA(h, cudaMemcpyAsync(s.data(), sums, 8 * nv, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    for (int v = 0; v < nv; v++) out_host[v] = 0.5 * (sqrt(1.0 + s[v]) - 1.0);
    return PCI_OK;
}

int sp_jav(pci_gpu *h, const double *X, int ldx, int nv, int64_t nlim, double *out_host)
{
    return sp_jav_strided(h, X, ldx, 1, nv, nlim, out_host);
}
