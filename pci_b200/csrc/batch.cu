// Batched form: many independent CI blocks solved together on one GPU.
//
// The reference runs one block per pconf job (Diag4, pconf.F90:238, and the
// Davidson module davidson.f90: Nlv roots, N_it iterations, residual
// criterion Crt4).  Here every block keeps its own lower-triangle FP32 CSR
// where its H-build left it (no concatenation copy); a table of per-block
// pointers lets one persistent SpMM kernel walk the rows of all blocks, and
// all vectors live in shared tall arrays (rows of every block stacked,
// column-major, leading dimension = total rows).
//
// The solver is a block Davidson with the diagonal correction and a thick
// restart, run in lock step over the blocks: each step of an iteration (SpMM,
// Gram update, projected eigensolve, residuals, correction,
// orthonormalisation) is ONE launch over all blocks, per-block reductions go
// through per-chunk partial sums added in a fixed order (deterministic), and
// the per-block decisions (convergence, restart, dropped directions) are
// taken on the device, so the iterations replay from a CUDA graph with one
// 4-byte read-back per replay.  A converged block drops out of every kernel.
//
// Iteration for block b with orthonormal basis V (m columns), W = H V:
//   G = V^T W (only the new columns are formed), G = E diag(w) E^T (Jacobi),
//   x_j = V e_j, r_j = W e_j - w_j x_j for the nlv lowest w_j,
//   t_j = r_j / (w_j - H_nn) for unconverged roots,
//   restart V <- V E[:, :keep] when the basis would exceed max_sub,
//   t <- normalised, two classical Gram-Schmidt passes against V, two
//   Cholesky-QR passes (dependent directions dropped), appended to V.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "pci_internal.h"
#include "mlp_tc.cuh"
#include "../../include/pci_batch.h"

#define FULL_MASK 0xffffffffu

namespace {

constexpr int BT_CH = 1024;                                  // rows per chunk
constexpr int BT_TR = 32;                                    // rows per tile of the TN products
constexpr int BT_MS = PCI_BATCH_MAX_SUB;
constexpr int BT_LV = PCI_BATCH_MAX_LV;
constexpr int BT_PW = BT_MS * BT_LV;                         // partial words per chunk
constexpr int BT_ROT_THREADS = 128;
constexpr int BT_FIN_THREADS = 512;                          // threads of the per-block reductions

struct BlkCsr {
    const int64_t *rowptr;
    const int32_t *col;
    const void *val;   // float, double when f64, or (hi, lo) float pairs when split
    int64_t r0, nd;
    int32_t full;      // 1: both triangles stored (row-wise gather, no reductions)
    int32_t f64;
    int32_t split;     // 1: val holds float2 {hi, lo} with hi + lo = the FP64 value to 2^-48
    int32_t pad;
    const uint8_t *orbs;   // [nd][8] occupied orbitals of each row (0xff = empty), or null
};

struct Chunk {
    int32_t blk, pad;
    int64_t row0, row1;
};

// Per-block solver state, on the device.
struct BState {
    int m;        // basis vectors (the last knew of them still need H V)
    int knew;
    int done;     // 0 running, 1 converged, 2 iteration limit, 3 no new direction
    int iters;
    int restart;  // rotate V, W to `base` Ritz vectors this iteration
    int base;     // basis vectors the corrections are orthogonalised against
    int kk;       // corrections formed this iteration
    int k1, k2;   // corrections left after the first and second Cholesky-QR
    int phase;    // 0: SpMM on FP32 vectors with FP32 sums; 1: FP64 SpMM
    int sw;       // this iteration ends phase 0: restart on the Ritz vectors, recompute H V in FP64
    int it32;     // iterations spent in phase 0
    int stall;    // phase-0 iterations without a 10% drop of the largest residual
    int swit;     // iteration at which phase 0 ended
    double best;  // smallest largest-residual seen in phase 0
    int jsel[BT_LV];
    int lrn[BT_LV];          // learned correction still used for root j
    double theta[BT_LV];
    double rnorm[BT_LV];
    double prev[BT_LV];      // residual of root j at the previous iteration
    double scale[BT_LV];
};

struct Bufs {
    double *V, *W, *R, *T, *T2, *P, *Q, *G, *EV, *EW, *part, *coef, *D;
    float *P32, *Q32;
    double *Xk;   // Ritz vectors of the iteration (written only while harvesting samples)
    int64_t ld;
    int msub, nlv, keep, max_it;
    double tol, swtol;
    int stall_max;
};

enum { TN_GRAM = 0, TN_TT = 1, TN_VT = 2, TN_T2 = 3 };
enum { FIN_GRAM = 0, FIN_NORM = 1, FIN_VT1 = 2, FIN_VT2 = 3, FIN_CHOL1 = 4, FIN_CHOL2 = 5, FIN_RESID = 6 };

// ------------------------------------------------------------ setup ---

__global__ void k_to_f32(const double *a, float *b, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// In place: a[i] (double) becomes the float pair {hi, lo}, hi = fl32(a[i]),
// lo = fl32(a[i] - hi), so hi + lo equals a[i] to about 2^-48 relative.
__global__ void k_split(double *a, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = a[i];
        const float hi = (float)v;
        const float lo = (float)(v - (double)hi);
        reinterpret_cast<float2 *>(a)[i] = make_float2(hi, lo);
    }
}

// Diagonal of one block's lower-triangle CSR (values FP64, FP32 or split pairs).
__global__ void kb_diag_blk(const int64_t *rowptr, const int32_t *col, const void *val, int f64, int split, int64_t nd,
                            double *D)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int64_t l = rowptr[n + 1] - 1; l >= rowptr[n]; l--)
            if (col[l] == n) {
                if (f64) d = ((const double *)val)[l];
                else if (split) {
                    const float2 hl = ((const float2 *)val)[l];
                    d = (double)hl.x + (double)hl.y;
                } else d = (double)((const float *)val)[l];
                break;
            }
        D[n] = d;
    }
}

__global__ void kb_set_units(double *V, int64_t ld, const int64_t *pos, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) V[pos[i]] = 1.0;
}

// ------------------------------------------------------------- SpMM ---

// Stored value kinds of a block: FP32, FP64, or split FP32 pairs.
enum { VK_F32 = 0, VK_F64 = 1, VK_SPLIT = 2 };

// Value of stored element l as the arithmetic type XT of the SpMM: FP32
// vectors take the FP32 value (hi of a split pair), FP64 vectors the FP64
// value (hi + lo of a split pair).  The kind is a template parameter so the
// element loop has no branch on it and its loads issue back to back.
template <typename XT, int VK>
__device__ __forceinline__ XT blk_val(const void *val, int64_t l)
{
    if constexpr (VK == VK_F64) {
        return (XT)__ldg(&((const double *)val)[l]);
    } else if constexpr (VK == VK_SPLIT) {
        const float2 hl = __ldg(&((const float2 *)val)[l]);
        if constexpr (sizeof(XT) == 4) return (XT)hl.x;
        else return (XT)((double)hl.x + (double)hl.y);
    } else {
        return (XT)__ldg(&((const float *)val)[l]);
    }
}

__device__ __forceinline__ int blk_kind(const BlkCsr &B)
{
    return B.f64 ? VK_F64 : (B.split ? VK_SPLIT : VK_F32);
}

// Row n (local row ln) of block B for vector v: the row part of the product
// (returned; both triangles for a full copy) and, for a lower triangle, the
// transpose part added to Y by global reductions.  XT is the vector and sum
// type (double, or float in the first phase of the mixed-precision form).
template <int NV, int G, typename XT, int VK>
__device__ __forceinline__ XT spmm_row(const BlkCsr &B, int64_t ln, int64_t n, int g, int v,
                                       const XT *__restrict__ X, XT *Y)
{
    const void *val = B.val;
    const int64_t l0 = __ldg(&B.rowptr[ln]), l1 = __ldg(&B.rowptr[ln + 1]);
    XT acc = 0;
    int64_t l = l0 + g;
    if (B.full) {
        for (; l + 3 * G < l1; l += 4 * G) {
            int k[4];
            XT t[4], xk[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                k[u] = __ldg(&B.col[l + u * G]);
                t[u] = blk_val<XT, VK>(val, l + u * G);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) xk[u] = __ldg(&X[(B.r0 + k[u]) * NV + v]);
#pragma unroll
            for (int u = 0; u < 4; u++) acc += t[u] * xk[u];
        }
        for (; l < l1; l += G) acc += blk_val<XT, VK>(val, l) * __ldg(&X[(B.r0 + __ldg(&B.col[l])) * NV + v]);
        return acc;
    }
    const XT xn = __ldg(&X[n * NV + v]);
    // four elements per step: their loads are issued before any use
    for (; l + 3 * G < l1; l += 4 * G) {
        int k[4];
        XT t[4], xk[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            k[u] = __ldg(&B.col[l + u * G]);
            t[u] = blk_val<XT, VK>(val, l + u * G);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) xk[u] = __ldg(&X[(B.r0 + k[u]) * NV + v]);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (k[u] != ln) atomicAdd(&Y[(B.r0 + k[u]) * NV + v], t[u] * xn);
            acc += t[u] * xk[u];
        }
    }
    for (; l < l1; l += G) {
        const int k = __ldg(&B.col[l]);
        const XT t = blk_val<XT, VK>(val, l);
        const int64_t kg = B.r0 + k;
        if (k != ln) atomicAdd(&Y[kg * NV + v], t * xn);
        acc += t * __ldg(&X[kg * NV + v]);
    }
    return acc;
}

// Y = H X over the rows of every running block in SpMM phase `phase`
// (blocks in the other phase are skipped), X and Y row-major with NV
// vectors.  A team of SUB lanes owns a row; within it NV lanes share one
// stored element (lane v takes vector v) and SUB/NV elements go per step.
// Lower-triangle blocks: the transpose part of each element goes to Y as a
// global reduction, and so does the row part (other rows add into it), so Y
// starts at zero.  Blocks stored with both triangles: a plain row gather and
// store, with no reductions.
template <int NV, int SUB, typename XT>
__global__ void __launch_bounds__(256) kb_spmm(const BlkCsr *__restrict__ blks, const int32_t *__restrict__ row_blk,
                                               const BState *__restrict__ bst, int64_t rows, int phase,
                                               const XT *__restrict__ X, XT *Y)
{
    constexpr int G = SUB / NV;
    constexpr int TPW = 32 / SUB;
    static_assert(G >= 1, "fewer lanes per row than vectors");
    const int lane = threadIdx.x & 31;
    const int sl = lane % SUB;
    const int g = sl / NV, v = sl - g * NV;
    const bool act = g < G;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n0 = warp * TPW; n0 < rows; n0 += nwarps * TPW) {
        const int64_t n = n0 + lane / SUB;
        bool ok = n < rows;
        const int b = ok ? __ldg(&row_blk[n]) : 0;
        ok = ok && bst[b].done == 0 && bst[b].phase == phase;
        XT acc = 0;
        bool full = false;
        if (ok && act) {
            const BlkCsr B = blks[b];
            full = B.full != 0;
            const int vk = blk_kind(B);
            if (vk == VK_F64) acc = spmm_row<NV, G, XT, VK_F64>(B, n - B.r0, n, g, v, X, Y);
            else if (vk == VK_SPLIT) acc = spmm_row<NV, G, XT, VK_SPLIT>(B, n - B.r0, n, g, v, X, Y);
            else acc = spmm_row<NV, G, XT, VK_F32>(B, n - B.r0, n, g, v, X, Y);
        }
#pragma unroll
        for (int gg = 1; gg < G; gg++) {
            const XT o = __shfl_sync(FULL_MASK, acc, g == 0 ? lane + gg * NV : lane);
            if (g == 0) acc += o;
        }
        if (ok && act && g == 0) {
            if (full) Y[n * NV + v] = acc;
            else atomicAdd(&Y[n * NV + v], acc);
        }
    }
}

constexpr int N_SUB = 3, N_CTAS = 4;
constexpr int SUBS[N_SUB] = {32, 16, 8};
constexpr int CTAS[N_CTAS] = {4, 8, 16, 32};
constexpr int N_VARIANTS = N_SUB * N_CTAS;
constexpr int DEFAULT_VARIANT = 2;   // 32 lanes per row, 16 blocks per SM

template <int NV, typename XT>
void launch_spmm_nv(int sub, int grid, cudaStream_t st, const BlkCsr *blks, const int32_t *row_blk, const BState *bst,
                    int64_t rows, int phase, const XT *X, XT *Y)
{
    if (sub == 32) kb_spmm<NV, 32, XT><<<grid, 256, 0, st>>>(blks, row_blk, bst, rows, phase, X, Y);
    else if constexpr (NV <= 16) {
        if (sub == 16) kb_spmm<NV, 16, XT><<<grid, 256, 0, st>>>(blks, row_blk, bst, rows, phase, X, Y);
        else if constexpr (NV <= 8) kb_spmm<NV, 8, XT><<<grid, 256, 0, st>>>(blks, row_blk, bst, rows, phase, X, Y);
    }
}

bool variant_ok(int nv, int variant)
{
    return variant >= 0 && variant < N_VARIANTS && SUBS[variant / N_CTAS] >= nv;
}

// One SpMM launch of every running block in `phase` (1: FP64 vectors X, Y;
// 0: FP32 vectors X, Y).
template <typename XT>
void launch_spmm(int nv, int variant, int nsm, cudaStream_t st, const BlkCsr *blks, const int32_t *row_blk,
                 const BState *bst, int64_t rows, int phase, const XT *X, XT *Y)
{
    const int sub = SUBS[variant / N_CTAS];
    const int grid = nsm * CTAS[variant % N_CTAS];
    switch (nv) {
    case 1: launch_spmm_nv<1, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 2: launch_spmm_nv<2, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 3: launch_spmm_nv<3, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 4: launch_spmm_nv<4, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 5: launch_spmm_nv<5, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 6: launch_spmm_nv<6, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 7: launch_spmm_nv<7, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 8: launch_spmm_nv<8, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 9: launch_spmm_nv<9, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 10: launch_spmm_nv<10, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    case 11: launch_spmm_nv<11, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    default: launch_spmm_nv<12, XT>(sub, grid, st, blks, row_blk, bst, rows, phase, X, Y); break;
    }
}

// ------------------------------------------------------ per-row steps ---

// P[n, s] = V[n, m-knew+s] (s < knew), 0 otherwise; Q = 0 for the SpMM.
// Blocks in phase 0 pack FP32 copies into P32 / Q32.
__global__ void kb_pack(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const int c0 = s.m - s.knew, kn = s.knew, nv = B.nlv;
    if (s.phase == 0) {
        for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
            for (int c = 0; c < nv; c++) {
                B.P32[n * nv + c] = c < kn ? (float)B.V[(int64_t)(c0 + c) * B.ld + n] : 0.f;
                B.Q32[n * nv + c] = 0.f;
            }
        }
        return;
    }
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        for (int c = 0; c < nv; c++) {
            B.P[n * nv + c] = c < kn ? B.V[(int64_t)(c0 + c) * B.ld + n] : 0.0;
            B.Q[n * nv + c] = 0.0;
        }
    }
}

__device__ __forceinline__ void tn_dims(int mode, const BState &s, const Bufs &B, const double *&A, int &ma,
                                        const double *&Bm, int &b0, int &kb)
{
    if (mode == TN_GRAM) { A = B.V; ma = s.m; Bm = B.Q; b0 = s.m - s.knew; kb = s.knew; }
    else if (mode == TN_TT) { A = B.T; ma = s.kk; Bm = B.T; b0 = 0; kb = s.kk; }
    else if (mode == TN_VT) { A = B.V; ma = s.base; Bm = B.T; b0 = 0; kb = s.kk; }
    else { A = B.T2; ma = s.k1; Bm = B.T2; b0 = 0; kb = s.k1; }
}

// Per-chunk partial of A[:, :ma]^T B[:, b0:b0+kb] over the chunk's rows.  In
// TN_GRAM mode B is the SpMM output Q (row-major) and the kernel also stores
// it as W's new columns.
// D (8 x 8, FP64) += A (8 x 4) B (4 x 8) on the FP64 tensor cores.
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Per-chunk partial of A[:, :ma]^T B[:, b0:b0+kb] over the chunk's rows, on
// the FP64 tensor cores: the chunk's rows pass through shared memory 32 at a
// time (zero-padded to whole 8 x 8 output tiles) and each of the 8 warps owns
// up to QT 8 x 8 tiles of the ma x kb product, eight m8n8k4 steps per 32 rows.
// In TN_GRAM mode B is the SpMM output Q (row-major) and the kernel also
// stores it as W's new columns.
template <int MODE>
__global__ void __launch_bounds__(256) kb_tn(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const double *A, *Bm;
    int ma, b0, kb;
    tn_dims(MODE, s, B, A, ma, Bm, b0, kb);
    constexpr int MT = BT_MS / 8, NT = (BT_LV + 7) / 8, QT = (MT * NT + 7) / 8;
    static_assert(BT_MS % 8 == 0, "subspace maximum must be a multiple of 8");
    __shared__ double As[BT_TR][MT * 8 + 1];
    __shared__ double Bs[BT_TR][NT * 8 + 1];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int mt = (ma + 7) / 8, nt = (kb + 7) / 8, ntile = mt * nt;
    const int map = mt * 8, kbp = nt * 8;
    double acc[QT][2] = {};
    const int64_t ld = B.ld;
    for (int64_t r0 = ch.row0; r0 < ch.row1; r0 += BT_TR) {
        const int nr = (int)min((int64_t)BT_TR, ch.row1 - r0);
        for (int idx = t; idx < BT_TR * map; idx += blockDim.x) {
            const int r = idx % BT_TR, i = idx / BT_TR;
            As[r][i] = (r < nr && i < ma) ? A[(int64_t)i * ld + r0 + r] : 0.0;
        }
        for (int idx = t; idx < BT_TR * kbp; idx += blockDim.x) {
            const int r = idx % BT_TR, c = idx / BT_TR;
            double v = 0.0;
            if (r < nr && c < kb) {
                if (MODE == TN_GRAM) {
                    v = s.phase == 0 ? (double)B.Q32[(r0 + r) * B.nlv + c] : Bm[(r0 + r) * B.nlv + c];
                    B.W[(int64_t)(b0 + c) * ld + r0 + r] = v;
                } else {
                    v = Bm[(int64_t)(b0 + c) * ld + r0 + r];
                }
            }
            Bs[r][c] = v;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < QT; q++) {
            const int tile = w + 8 * q;
            if (tile < ntile) {
                const int mi = tile / nt, ni = tile - mi * nt;
                const int ka = lane & 3, row = lane >> 2;
#pragma unroll
                for (int k0 = 0; k0 < BT_TR; k0 += 4)
                    dmma884(acc[q], As[k0 + ka][mi * 8 + row], Bs[k0 + ka][ni * 8 + row]);
            }
        }
        __syncthreads();
    }
    double *out = B.part + (int64_t)blockIdx.x * BT_PW;
#pragma unroll
    for (int q = 0; q < QT; q++) {
        const int tile = w + 8 * q;
        if (tile < ntile) {
            const int mi = tile / nt, ni = tile - mi * nt;
            const int i = mi * 8 + (lane >> 2);
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int c = ni * 8 + 2 * (lane & 3) + u;
                if (i < ma && c < kb) out[i * kb + c] = acc[q][u];
            }
        }
    }
}

// Sum of up to BT_LV per-thread values over the thread block into out[0..n).
__device__ void block_sum(double (&v)[BT_LV], int n, double *out)
{
    __shared__ double red[8][BT_LV];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < BT_LV; j++) {
        double x = v[j];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL_MASK, x, o);
        if (lane == 0) red[w][j] = x;
    }
    __syncthreads();
    if (threadIdx.x < n) {
        double x = 0.0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) x += red[ww][threadIdx.x];
        out[threadIdx.x] = x;
    }
}

// R = W E[:, :nlv] - V E[:, :nlv] diag(theta); partial sums of |r_j|^2.
__global__ void __launch_bounds__(256) kb_resid(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const int m = s.m, nlv = B.nlv;
    __shared__ double Ys[BT_MS * BT_LV];
    const double *EV = B.EV + (int64_t)ch.blk * BT_MS * BT_MS;
    for (int e = threadIdx.x; e < m * nlv; e += blockDim.x) {
        const int i = e / nlv, j = e % nlv;
        Ys[e] = EV[j * BT_MS + i];
    }
    double th[BT_LV];
#pragma unroll
    for (int j = 0; j < BT_LV; j++) th[j] = j < nlv ? s.theta[j] : 0.0;
    __syncthreads();
    double ss[BT_LV];
#pragma unroll
    for (int j = 0; j < BT_LV; j++) ss[j] = 0.0;
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        double x[BT_LV], hx[BT_LV];
#pragma unroll
        for (int j = 0; j < BT_LV; j++) x[j] = hx[j] = 0.0;
        for (int i = 0; i < m; i++) {
            const double v = B.V[(int64_t)i * B.ld + n], w = B.W[(int64_t)i * B.ld + n];
#pragma unroll
            for (int j = 0; j < BT_LV; j++) {
                if (j < nlv) {
                    x[j] += v * Ys[i * nlv + j];
                    hx[j] += w * Ys[i * nlv + j];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < BT_LV; j++) {
            if (j < nlv) {
                const double r = hx[j] - th[j] * x[j];
                B.R[(int64_t)j * B.ld + n] = r;
                if (B.Xk) B.Xk[(int64_t)j * B.ld + n] = x[j];
                ss[j] += r * r;
            }
        }
    }
    block_sum(ss, nlv, B.part + (int64_t)blockIdx.x * BT_PW);
}

// Thick restart: V[:, :base] = V[:, :m] E[:, :base], W likewise, row by row
// through shared memory.
__global__ void __launch_bounds__(BT_ROT_THREADS) kb_rotate(const Chunk *__restrict__ chunks,
                                                            const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done || !s.restart) return;
    extern __shared__ double sm[];
    const int m = s.m, kb = s.base;
    double *Es = sm;                         // [m][kb]
    double *rowv = sm + BT_MS * BT_MS;       // [m][BT_ROT_THREADS]
    const double *EV = B.EV + (int64_t)ch.blk * BT_MS * BT_MS;
    for (int e = threadIdx.x; e < m * kb; e += blockDim.x) {
        const int i = e / kb, c = e % kb;
        Es[e] = EV[c * BT_MS + i];
    }
    __syncthreads();
    for (int64_t nb = ch.row0; nb < ch.row1; nb += BT_ROT_THREADS) {
        const int64_t n = nb + threadIdx.x;
        const bool ok = n < ch.row1;
        for (int pass = 0; pass < 2; pass++) {
            double *A = pass ? B.W : B.V;
            if (ok)
                for (int i = 0; i < m; i++) rowv[i * BT_ROT_THREADS + threadIdx.x] = A[(int64_t)i * B.ld + n];
            if (ok)
                for (int c = 0; c < kb; c++) {
                    double acc = 0.0;
                    for (int i = 0; i < m; i++) acc += rowv[i * BT_ROT_THREADS + threadIdx.x] * Es[i * kb + c];
                    A[(int64_t)c * B.ld + n] = acc;
                }
        }
    }
}

// T[:, s] = R[:, jsel[s]] / (theta_j - H_nn).
__global__ void kb_correct(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const int kk = s.kk;
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        const double dn = B.D[n];
        for (int c = 0; c < kk; c++) {
            const int j = s.jsel[c];
            double d = s.theta[j] - dn;
            if (fabs(d) < 1e-8) d = d < 0.0 ? -1e-8 : 1e-8;
            B.T[(int64_t)c * B.ld + n] = B.R[(int64_t)j * B.ld + n] / d;
        }
    }
}

// Learned correction: T[:, c] = MLP(features of row n) for the correction
// slots whose root still uses it (lrn); kb_correct's diagonal correction
// stays in the other slots.  Features of row n for root j: the occupied
// orbitals of its determinant, H_nn - theta_j, s r_jn and s r_jn / (theta_j
// - H_nn) (the diagonal correction, its denominator kept away from zero as in
// kb_correct, clipped to +-1e4), with s = sqrt(nd) / |r_j|.
// One warp evaluates 16 rows of one slot on the tensor cores (mlp_tc.cuh);
// work items are (chunk, 16-row tile, slot) in a grid-stride loop.
__global__ void __launch_bounds__(256, 2) kb_learned(const Chunk *__restrict__ chunks, int nch,
                                                     const BlkCsr *__restrict__ blks, const BState *__restrict__ bst,
                                                     Bufs B, mlptc::Weights W)
{
    extern __shared__ double smw[];
    const mlptc::Smem S = mlptc::load(W, reinterpret_cast<unsigned char *>(smw));
    const int lane = threadIdx.x & 31, g = lane >> 2;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int TILES = BT_CH / 16;
    const int64_t nitems = (int64_t)nch * TILES * BT_LV;
    for (int64_t it = warp; it < nitems; it += nwarps) {
        const int c = (int)(it % BT_LV);
        const int64_t q = it / BT_LV;
        const int sub = (int)(q % TILES);
        const Chunk ch = chunks[q / TILES];
        const BState &s = bst[ch.blk];
        if (s.done || c >= s.kk) continue;
        const int j = s.jsel[c];
        if (!s.lrn[j]) continue;
        const int64_t r0 = ch.row0 + (int64_t)sub * 16;
        if (r0 >= ch.row1) continue;
        const BlkCsr &Bk = blks[ch.blk];
        const double fs = sqrt((double)Bk.nd) / fmax(s.rnorm[j], 1e-300);
        const double th = s.theta[j];
        uint8_t o[2][mlptc::MAXOCC];
        float f[2][mlptc::NSCAL], out[2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int64_t n = r0 + g + 8 * r;
            const bool ok = n < ch.row1;
            const uint8_t *src = Bk.orbs + (ok ? (n - Bk.r0) * mlptc::MAXOCC : 0);
#pragma unroll
            for (int e = 0; e < mlptc::MAXOCC; e++) o[r][e] = ok ? src[e] : (uint8_t)0xff;
            const double dn = ok ? B.D[n] : 0.0, rn = ok ? B.R[(int64_t)j * B.ld + n] * fs : 0.0;
            double den = th - dn;
            if (fabs(den) < 1e-8) den = den < 0.0 ? -1e-8 : 1e-8;
            f[r][0] = ok ? (float)(dn - th) : 0.f;
            f[r][1] = (float)rn;
            f[r][2] = ok ? (float)fmax(-1e4, fmin(1e4, rn / den)) : 0.f;
        }
        mlptc::tile(S, W.nin, o, f, out);
        if ((lane & 3) == 0) {
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const int64_t n = r0 + g + 8 * r;
                if (n < ch.row1) B.T[(int64_t)c * B.ld + n] = (double)out[r];
            }
        }
    }
}

// Samples for training the learned correction: for every sampled row and
// every root still above the criterion of a running block, the Ritz vector
// and residual entries with the Ritz value, residual norm and H_nn.
__global__ void kb_harvest(const int64_t *__restrict__ rows, int64_t nrows, const int32_t *__restrict__ row_blk,
                           const BlkCsr *__restrict__ blks, const BState *__restrict__ bst, Bufs B,
                           pci_batch_sample *out, int64_t cap, unsigned long long *count)
{
    const int nlv = B.nlv;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nrows * nlv;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / nlv;
        const int j = (int)(e - i * nlv);
        const int64_t n = rows[i];
        const int b = row_blk[n];
        const BState &s = bst[b];
        if (s.done || !(s.rnorm[j] > B.tol)) continue;
        const unsigned long long pos = atomicAdd(count, 1ULL);
        if ((int64_t)pos >= cap) continue;
        pci_batch_sample rec;
        rec.blk = b;
        rec.iter = s.iters;
        rec.root = j;
        rec.phase = s.phase;
        rec.row = n - blks[b].r0;
        rec.x = B.Xk[(int64_t)j * B.ld + n];
        rec.r = B.R[(int64_t)j * B.ld + n];
        rec.theta = s.theta[j];
        rec.rnorm = s.rnorm[j];
        rec.diag = B.D[n];
        out[pos] = rec;
    }
}

// Occupied orbitals (0-based) of every determinant: orbs[n][e] = orbital of
// m-state occ[n][e], 0xff past the Ne electrons.
__global__ void kb_row_orbs(const uint16_t *occ, const int16_t *ms_orb, int ne, int64_t nd, uint8_t *orbs)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int e = 0; e < mlptc::MAXOCC; e++)
            orbs[n * mlptc::MAXOCC + e] = e < ne ? (uint8_t)ms_orb[occ[n * ne + e]] : (uint8_t)0xff;
}

// T[:, s] = scale_s T[:, s] - V[:, :base] C[:, s].
__global__ void __launch_bounds__(256) kb_proj(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const int kk = s.kk, base = s.base;
    __shared__ double Cs[BT_PW];
    const double *C = B.coef + (int64_t)ch.blk * BT_PW;
    for (int e = threadIdx.x; e < base * kk; e += blockDim.x) Cs[e] = C[e];
    __syncthreads();
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        double acc[BT_LV];
#pragma unroll
        for (int c = 0; c < BT_LV; c++) acc[c] = c < kk ? s.scale[c] * B.T[(int64_t)c * B.ld + n] : 0.0;
        for (int i = 0; i < base; i++) {
            const double v = B.V[(int64_t)i * B.ld + n];
#pragma unroll
            for (int c = 0; c < BT_LV; c++)
                if (c < kk) acc[c] -= v * Cs[i * kk + c];
        }
#pragma unroll
        for (int c = 0; c < BT_LV; c++)
            if (c < kk) B.T[(int64_t)c * B.ld + n] = acc[c];
    }
}

// out[:, :kout] = in[:, :kin] M (M = coef, kin x kout); pass 1 T -> T2,
// pass 2 T2 -> V[:, base:].
template <int PASS>
__global__ void __launch_bounds__(256) kb_tri(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    if (s.done) return;
    const int kin = PASS == 1 ? s.kk : s.k1, kout = PASS == 1 ? s.k1 : s.k2;
    const double *in = PASS == 1 ? B.T : B.T2;
    double *out = PASS == 1 ? B.T2 : B.V + (int64_t)s.base * B.ld;
    __shared__ double Ms[BT_LV * BT_LV];
    const double *M = B.coef + (int64_t)ch.blk * BT_PW;
    for (int e = threadIdx.x; e < kin * kout; e += blockDim.x) Ms[e] = M[e];
    __syncthreads();
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        double x[BT_LV];
#pragma unroll
        for (int c = 0; c < BT_LV; c++) x[c] = c < kin ? in[(int64_t)c * B.ld + n] : 0.0;
        for (int o = 0; o < kout; o++) {
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < BT_LV; c++)
                if (c < kin) acc += x[c] * Ms[c * kout + o];
            out[(int64_t)o * B.ld + n] = acc;
        }
    }
}

// Final Ritz vectors X[:, j] = V[:, :m] E[:, j] into R.
__global__ void __launch_bounds__(256) kb_ritz(const Chunk *__restrict__ chunks, const BState *__restrict__ bst, Bufs B)
{
    const Chunk ch = chunks[blockIdx.x];
    const BState &s = bst[ch.blk];
    const int m = s.m, nlv = B.nlv;
    __shared__ double Ys[BT_MS * BT_LV];
    const double *EV = B.EV + (int64_t)ch.blk * BT_MS * BT_MS;
    for (int e = threadIdx.x; e < m * nlv; e += blockDim.x) Ys[e] = EV[(e % nlv) * BT_MS + e / nlv];
    __syncthreads();
    for (int64_t n = ch.row0 + threadIdx.x; n < ch.row1; n += blockDim.x) {
        double x[BT_LV];
#pragma unroll
        for (int j = 0; j < BT_LV; j++) x[j] = 0.0;
        for (int i = 0; i < m; i++) {
            const double v = B.V[(int64_t)i * B.ld + n];
#pragma unroll
            for (int j = 0; j < BT_LV; j++)
                if (j < nlv) x[j] += v * Ys[i * nlv + j];
        }
        for (int j = 0; j < nlv; j++) B.R[(int64_t)j * B.ld + n] = x[j];
    }
}

// --------------------------------------------------- per-block steps ---

// Cholesky of the k x k Gram matrix S (row-major) with dependent columns
// (pivot <= thr) dropped; M (k x kept, row-major) maps the k columns to the
// kept orthonormal ones: out = in M.  Returns the number kept.
__device__ int chol_drop(const double *S, int k, double thr, double *M)
{
    double L[BT_LV][BT_LV];
    int kept[BT_LV], nk = 0;
    for (int i = 0; i < BT_LV; i++)
        for (int j = 0; j < BT_LV; j++) L[i][j] = 0.0;
    for (int j = 0; j < k; j++) {
        double d = S[j * k + j];
        for (int a = 0; a < nk; a++) d -= L[j][kept[a]] * L[j][kept[a]];
        if (!(d > thr)) continue;
        const double ljj = sqrt(d);
        L[j][j] = ljj;
        for (int i = j + 1; i < k; i++) {
            double x = S[i * k + j];
            for (int a = 0; a < nk; a++) x -= L[i][kept[a]] * L[j][kept[a]];
            L[i][j] = x / ljj;
        }
        kept[nk++] = j;
    }
    // Li = inverse of L restricted to the kept rows and columns (lower triangular)
    double Li[BT_LV][BT_LV];
    for (int a = 0; a < nk; a++) {
        for (int c = 0; c < nk; c++) Li[a][c] = 0.0;
        Li[a][a] = 1.0 / L[kept[a]][kept[a]];
        for (int c = 0; c < a; c++) {
            double x = 0.0;
            for (int p = c; p < a; p++) x += L[kept[a]][kept[p]] * Li[p][c];
            Li[a][c] = -x * Li[a][a];
        }
    }
    for (int r = 0; r < k; r++)
        for (int c = 0; c < nk; c++) M[r * nk + c] = 0.0;
    for (int a = 0; a < nk; a++)
        for (int c = 0; c < nk; c++) M[kept[a] * nk + c] = Li[c][a];
    return nk;
}

template <int MODE>
__global__ void __launch_bounds__(BT_FIN_THREADS) kb_fin(const int64_t *__restrict__ cb, BState *bst, Bufs B)
{
    const int b = blockIdx.x, t = threadIdx.x;
    BState &s = bst[b];
    if (s.done) return;
    int ma, kb;
    if (MODE == FIN_GRAM) { ma = s.m; kb = s.knew; }
    else if (MODE == FIN_NORM || MODE == FIN_CHOL1) { ma = s.kk; kb = s.kk; }
    else if (MODE == FIN_VT1 || MODE == FIN_VT2) { ma = s.base; kb = s.kk; }
    else if (MODE == FIN_CHOL2) { ma = s.k1; kb = s.k1; }
    else { ma = 1; kb = B.nlv; }
    __shared__ double res[BT_PW];
    const int ne = ma * kb;
    const int64_t c0 = cb[b], c1 = cb[b + 1];
    for (int e = t; e < ne; e += blockDim.x) {
        // four running sums over the chunks (more loads in flight), added in a fixed order
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int64_t c = c0;
        for (; c + 3 < c1; c += 4) {
            a0 += B.part[c * BT_PW + e];
            a1 += B.part[(c + 1) * BT_PW + e];
            a2 += B.part[(c + 2) * BT_PW + e];
            a3 += B.part[(c + 3) * BT_PW + e];
        }
        for (; c < c1; c++) a0 += B.part[c * BT_PW + e];
        res[e] = (a0 + a1) + (a2 + a3);
    }
    __syncthreads();
    double *coef = B.coef + (int64_t)b * BT_PW;
    if (MODE == FIN_GRAM) {
        double *G = B.G + (int64_t)b * BT_MS * BT_MS;
        const int n0 = s.m - s.knew;
        for (int e = t; e < ne; e += blockDim.x) {
            const int i = e / kb, c = e % kb, col = n0 + c;
            double v = res[e];
            if (i >= n0) v = 0.5 * (v + res[col * kb + (i - n0)]);
            G[i * BT_MS + col] = v;
            G[col * BT_MS + i] = v;
        }
    } else if (MODE == FIN_NORM) {
        if (t < kb) {
            const double q = res[t * kb + t];
            s.scale[t] = q > 0.0 ? 1.0 / sqrt(q) : 0.0;
        }
    } else if (MODE == FIN_VT1) {
        for (int e = t; e < ne; e += blockDim.x) coef[e] = res[e] * s.scale[e % kb];
    } else if (MODE == FIN_VT2) {
        for (int e = t; e < ne; e += blockDim.x) coef[e] = res[e];
        __syncthreads();
        if (t < kb) s.scale[t] = 1.0;
    } else if (MODE == FIN_CHOL1) {
        if (t == 0) s.k1 = chol_drop(res, kb, 1e-16, coef);
    } else if (MODE == FIN_CHOL2) {
        if (t == 0) s.k2 = chol_drop(res, kb, 1e-3, coef);
    } else {   // FIN_RESID: convergence, corrections to form, restart
        __shared__ int sh_base, sh_restart;
        if (t == 0) {
            int nconv = 0, nsw = 0;
            double mx = 0.0;
            for (int j = 0; j < B.nlv; j++) {
                const double rn = sqrt(fmax(res[j], 0.0));
                s.prev[j] = s.rnorm[j];
                s.rnorm[j] = rn;
                nconv += rn <= B.tol;
                nsw += rn <= B.swtol;
                mx = fmax(mx, rn);
            }
            s.iters += 1;
            sh_restart = 0;
            sh_base = 0;
            // fallback of the learned correction: a root whose residual did not drop
            // since the previous iteration takes the diagonal correction from now on
            // (not right after the end of the FP32 phase, whose restart recomputes H V)
            if (s.iters >= 2 && s.iters != s.swit + 1)
                for (int j = 0; j < B.nlv; j++)
                    if (s.lrn[j] && s.rnorm[j] >= s.prev[j]) s.lrn[j] = 0;
            const bool p0 = s.phase == 0;
            if (p0) {
                s.it32 += 1;
                if (mx < 0.9 * s.best) {
                    s.best = mx;
                    s.stall = 0;
                } else {
                    s.stall += 1;
                }
            }
            if (!p0 && nconv == B.nlv) {
                s.done = 1;
            } else if (s.iters >= B.max_it) {
                s.done = 2;
            } else if (p0 && (nsw == B.nlv || s.stall >= B.stall_max)) {
                // end of the FP32 phase: restart on the nlv Ritz vectors; the next
                // iteration recomputes their H V with the FP64 SpMM
                s.kk = 0;
                s.sw = 1;
                s.swit = s.iters;
                sh_base = B.nlv;
                sh_restart = 1;
                s.base = sh_base;
                s.restart = sh_restart;
            } else {
                const double thr = p0 ? B.swtol : B.tol;
                int kk = 0;
                for (int j = 0; j < B.nlv; j++)
                    if (!(s.rnorm[j] <= thr)) s.jsel[kk++] = j;
                s.kk = kk;
                if (s.m + kk > B.msub) {
                    sh_base = min(B.keep, s.m);
                    sh_restart = 1;
                } else {
                    sh_base = s.m;
                }
                s.base = sh_base;
                s.restart = sh_restart;
            }
        }
        __syncthreads();
        if (sh_restart) {
            double *G = B.G + (int64_t)b * BT_MS * BT_MS;
            const double *EW = B.EW + (int64_t)b * BT_MS;
            for (int e = t; e < sh_base * sh_base; e += blockDim.x) {
                const int i = e / sh_base, j = e % sh_base;
                G[i * BT_MS + j] = i == j ? EW[i] : 0.0;
            }
        }
    }
}

// Eigenpairs of the m x m projected matrix of every running block by cyclic
// Jacobi rotations in round-robin order (m/2 disjoint rotations per step; the
// rotation angle as in Golub & Van Loan, Matrix Computations, sec. 8.5),
// eigenvalues ascending.
__global__ void __launch_bounds__(256) kb_eig(BState *bst, Bufs B)
{
    const int b = blockIdx.x, t = threadIdx.x;
    BState &s = bst[b];
    if (s.done) return;
    const int m = s.m, mp = m + (m & 1), h = mp / 2;
    extern __shared__ double sm[];
    double *A = sm, *Vm = sm + mp * mp;
    __shared__ int pp[BT_MS / 2], qq[BT_MS / 2];
    __shared__ double cc[BT_MS / 2], sn[BT_MS / 2];
    __shared__ double red[2][8];
    __shared__ int stop;
    __shared__ int order[BT_MS];
    const double *G = B.G + (int64_t)b * BT_MS * BT_MS;
    for (int e = t; e < mp * mp; e += blockDim.x) {
        const int i = e / mp, j = e % mp;
        A[e] = (i < m && j < m) ? G[i * BT_MS + j] : 0.0;
        Vm[e] = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int sweep = 0; sweep < 40; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int e = t; e < mp * mp; e += blockDim.x) {
            const double a = A[e];
            tot += a * a;
            if (e / mp != e % mp) off += a * a;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_down_sync(FULL_MASK, off, o);
            tot += __shfl_down_sync(FULL_MASK, tot, o);
        }
        if ((t & 31) == 0) { red[0][t >> 5] = off; red[1][t >> 5] = tot; }
        __syncthreads();
        if (t == 0) {
            double o2 = 0.0, t2 = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) { o2 += red[0][w]; t2 += red[1][w]; }
            stop = !(o2 > 1e-30 * t2);
        }
        __syncthreads();
        if (stop) break;
        for (int r = 0; r < mp - 1; r++) {
            if (t < h) {
                int p, q;
                if (t == 0) { p = mp - 1; q = r; }
                else { p = (r + t) % (mp - 1); q = (r - t + mp - 1) % (mp - 1); }
                if (p > q) { const int x = p; p = q; q = x; }
                const double apq = A[p * mp + q];
                double c = 1.0, sv = 0.0;
                if (apq != 0.0) {
                    const double th = (A[q * mp + q] - A[p * mp + p]) / (2.0 * apq);
                    const double at = fabs(th);
                    const double tt = at > 1e150 ? 0.5 / th : (th >= 0.0 ? 1.0 : -1.0) / (at + sqrt(th * th + 1.0));
                    c = 1.0 / sqrt(tt * tt + 1.0);
                    sv = tt * c;
                }
                pp[t] = p; qq[t] = q; cc[t] = c; sn[t] = sv;
            }
            __syncthreads();
            for (int w = t; w < mp * h; w += blockDim.x) {   // columns: A <- A J, V <- V J
                const int k = w % mp, i = w / mp;
                const int p = pp[i], q = qq[i];
                const double c = cc[i], sv = sn[i];
                const double ap = A[k * mp + p], aq = A[k * mp + q];
                A[k * mp + p] = c * ap - sv * aq;
                A[k * mp + q] = sv * ap + c * aq;
                const double vp = Vm[k * mp + p], vq = Vm[k * mp + q];
                Vm[k * mp + p] = c * vp - sv * vq;
                Vm[k * mp + q] = sv * vp + c * vq;
            }
            __syncthreads();
            for (int w = t; w < mp * h; w += blockDim.x) {   // rows: A <- J^T A
                const int k = w % mp, i = w / mp;
                const int p = pp[i], q = qq[i];
                const double c = cc[i], sv = sn[i];
                const double ap = A[p * mp + k], aq = A[q * mp + k];
                A[p * mp + k] = c * ap - sv * aq;
                A[q * mp + k] = sv * ap + c * aq;
            }
            __syncthreads();
        }
    }
    if (t == 0) {
        for (int i = 0; i < m; i++) order[i] = i;
        for (int i = 0; i < m; i++) {   // stable selection of the ascending order
            int best = i;
            for (int j = i + 1; j < m; j++) {
                const double dj = A[order[j] * mp + order[j]], db = A[order[best] * mp + order[best]];
                if (dj < db) best = j;
            }
            const int x = order[best];
            for (int j = best; j > i; j--) order[j] = order[j - 1];
            order[i] = x;
        }
        for (int j = 0; j < B.nlv; j++) s.theta[j] = A[order[j] * mp + order[j]];
    }
    __syncthreads();
    double *EW = B.EW + (int64_t)b * BT_MS, *EV = B.EV + (int64_t)b * BT_MS * BT_MS;
    for (int e = t; e < m * m; e += blockDim.x) {
        const int j = e / m, i = e % m;
        EV[j * BT_MS + i] = Vm[i * mp + order[j]];
        if (i == 0) EW[j] = A[order[j] * mp + order[j]];
    }
}

__global__ void kb_commit(BState *bst, int nblk)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    BState &s = bst[b];
    if (s.done) return;
    s.restart = 0;
    if (s.sw) {   // FP64 from now on, every basis vector's H V recomputed
        s.m = s.base;
        s.knew = s.base;
        s.phase = 1;
        s.sw = 0;
        return;
    }
    s.m = s.base + s.k2;
    s.knew = s.k2;
    if (s.k2 == 0) {
        // no direction left: with learned corrections in use, fall back to the
        // diagonal ones for every root and go on; otherwise stop
        bool any = false;
        for (int j = 0; j < BT_LV; j++) {
            any = any || s.lrn[j] != 0;
            s.lrn[j] = 0;
        }
        if (!any) s.done = 3;
    }
}

__global__ void kb_count(const BState *bst, int nblk, int *ndone)
{
    __shared__ int c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        if (bst[b].done) atomicAdd(&c, 1);
    __syncthreads();
    if (threadIdx.x == 0) *ndone = c;
}

}  // namespace

// ------------------------------------------------------------- host ---

struct BlockRec {
    Csr H;            // lower triangle (freed once a full copy exists)
    Csr F;            // both triangles, or empty
    int64_t r0 = 0, nd = 0, nnz = 0;   // rows and stored lower-triangle elements
    int split = 0;    // H.val holds {hi, lo} float pairs (value precision 48)
    uint8_t *orbs = nullptr;   // [nd][8] occupied orbitals of each row (from the handle's basis), or null
    int nsu = 0;               // orbitals of the block's basis (0 without a basis)
    double *D = nullptr;       // diagonal H_nn
};

struct pci_batch {
    pci_gpu core;   // device, stream, error text and scratch
    int nsm = 148;
    std::string devname;
    std::vector<BlockRec> blocks;
    int64_t rows = 0, nnz = 0;
    bool dirty = true;
    BlkCsr *d_blk = nullptr;
    int32_t *d_row_blk = nullptr;
    double *d_D = nullptr;
    Chunk *d_chunks = nullptr;
    int64_t *d_cb = nullptr;
    int nch = 0;
    // solve buffers
    int64_t cap_rows = 0;
    int cap_nlv = 0;
    double *d_V = nullptr, *d_W = nullptr, *d_R = nullptr, *d_T = nullptr, *d_T2 = nullptr, *d_P = nullptr,
           *d_Q = nullptr, *d_G = nullptr, *d_EV = nullptr, *d_EW = nullptr, *d_part = nullptr, *d_coef = nullptr;
    float *d_P32 = nullptr, *d_Q32 = nullptr;
    BState *d_st = nullptr;
    int *d_ndone = nullptr;
    int last_nlv = 0;
    int storage = 0;          // 1: full copies where memory allows, 0: lower triangles only
    int value_prec = 32;      // 32: blocks rounded to FP32 when added; 64: kept as built; 48: hi/lo split
    bool storage_done = false;
    int64_t full_nnz = 0;     // lower-triangle elements of the blocks held as full copies
    int tuned_variant = -1, tuned_nv = 0;
    pci_mlp *model = nullptr;                 // learned correction (not owned)
    // samples for the learned correction
    int hv_per_block = 0, hv_seed = 0;
    int64_t hv_cap = 0, hv_n = 0, hv_last = 0;
    int64_t *d_hv_rows = nullptr;
    pci_batch_sample *d_hv = nullptr;
    unsigned long long *d_hv_count = nullptr;
    double *d_Xk = nullptr;
    double tuned_ms = 0.0;
    double st_total = 0, st_iters = 0, st_spmm = 0, st_variant = 0, st_setup = 0, st_launches = 0;
    double st_spmm32 = 0, st_it32 = 0, st_switched = 0;
};

static void free_solve(pci_batch *b)
{
    double **bufs[] = {&b->d_V, &b->d_W, &b->d_R, &b->d_T, &b->d_T2, &b->d_P, &b->d_Q,
                       &b->d_G, &b->d_EV, &b->d_EW, &b->d_part, &b->d_coef};
    for (double **p : bufs) { dev_free(*p); *p = nullptr; }
    dev_free(b->d_P32);
    dev_free(b->d_Q32);
    b->d_P32 = b->d_Q32 = nullptr;
    dev_free(b->d_st);
    b->d_st = nullptr;
    dev_free(b->d_ndone);
    b->d_ndone = nullptr;
    b->cap_rows = 0;
    b->cap_nlv = 0;
}

static void free_tables(pci_batch *b)
{
    dev_free(b->d_blk);
    dev_free(b->d_row_blk);
    dev_free(b->d_D);
    dev_free(b->d_chunks);
    dev_free(b->d_cb);
    b->d_blk = nullptr;
    b->d_row_blk = nullptr;
    b->d_D = nullptr;
    b->d_chunks = nullptr;
    b->d_cb = nullptr;
    b->nch = 0;
}

// Block table, row -> block map, diagonal and the chunk table.
static int build_tables(pci_batch *b)
{
    if (!b->dirty) return PCI_OK;
    pci_gpu *h = &b->core;
    free_tables(b);
    const int nblk = (int)b->blocks.size();
    std::vector<BlkCsr> tab(nblk);
    std::vector<int32_t> rb(b->rows);
    std::vector<Chunk> ch;
    std::vector<int64_t> cb(nblk + 1, 0);
    for (int i = 0; i < nblk; i++) {
        const BlockRec &r = b->blocks[i];
        const Csr &M = r.F.rowptr ? r.F : r.H;
        tab[i] = BlkCsr{M.rowptr, M.col, M.val, r.r0, r.nd, r.F.rowptr ? 1 : 0,
                        (M.val_f32 || r.split) ? 0 : 1, r.split ? 1 : 0, 0, r.orbs};
        std::fill(rb.begin() + r.r0, rb.begin() + r.r0 + r.nd, i);
        cb[i] = (int64_t)ch.size();
        for (int64_t s = 0; s < r.nd; s += BT_CH)
            ch.push_back(Chunk{i, 0, r.r0 + s, r.r0 + std::min<int64_t>(s + BT_CH, r.nd)});
    }
    cb[nblk] = (int64_t)ch.size();
    int rc = 0;
    b->d_blk = (BlkCsr *)dev_alloc(h, sizeof(BlkCsr) * nblk, &rc);
    if (rc) return rc;
    b->d_row_blk = (int32_t *)dev_alloc(h, 4 * b->rows, &rc);
    if (rc) return rc;
    b->d_D = (double *)dev_alloc(h, 8 * b->rows, &rc);
    if (rc) return rc;
    b->d_chunks = (Chunk *)dev_alloc(h, sizeof(Chunk) * ch.size(), &rc);
    if (rc) return rc;
    b->d_cb = (int64_t *)dev_alloc(h, 8 * cb.size(), &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpy(b->d_blk, tab.data(), sizeof(BlkCsr) * nblk, cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemcpy(b->d_row_blk, rb.data(), 4 * b->rows, cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemcpy(b->d_chunks, ch.data(), sizeof(Chunk) * ch.size(), cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemcpy(b->d_cb, cb.data(), 8 * cb.size(), cudaMemcpyHostToDevice));
    b->nch = (int)ch.size();
    for (int i = 0; i < nblk; i++) {
        const BlockRec &r = b->blocks[i];
        PCI_CUDA(h, cudaMemcpyAsync(b->d_D + r.r0, r.D, 8 * r.nd, cudaMemcpyDeviceToDevice, h->st));
    }
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    b->dirty = false;
    return PCI_OK;
}

static int ensure_solve(pci_batch *b, int nlv)
{
    if (b->cap_rows == b->rows && b->cap_nlv == nlv) return PCI_OK;
    free_solve(b);
    pci_gpu *h = &b->core;
    const int64_t R = b->rows, nblk = (int64_t)b->blocks.size();
    int rc = 0;
    auto al = [&](double **p, int64_t words) {
        if (!rc) *p = (double *)dev_alloc(h, 8 * std::max<int64_t>(words, 1), &rc);
    };
    al(&b->d_V, R * BT_MS);
    al(&b->d_W, R * BT_MS);
    al(&b->d_R, R * nlv);
    al(&b->d_T, R * nlv);
    al(&b->d_T2, R * nlv);
    al(&b->d_P, R * nlv);
    al(&b->d_Q, R * nlv);
    if (!rc) b->d_P32 = (float *)dev_alloc(h, 4 * std::max<int64_t>(R * nlv, 1), &rc);
    if (!rc) b->d_Q32 = (float *)dev_alloc(h, 4 * std::max<int64_t>(R * nlv, 1), &rc);
    al(&b->d_G, nblk * BT_MS * BT_MS);
    al(&b->d_EV, nblk * BT_MS * BT_MS);
    al(&b->d_EW, nblk * BT_MS);
    al(&b->d_part, (int64_t)b->nch * BT_PW);
    al(&b->d_coef, nblk * BT_PW);
    if (rc) return rc;
    b->d_st = (BState *)dev_alloc(h, sizeof(BState) * nblk, &rc);
    if (rc) return rc;
    b->d_ndone = (int *)dev_alloc(h, 16, &rc);
    if (rc) return rc;
    b->cap_rows = R;
    b->cap_nlv = nlv;
    return PCI_OK;
}

static Bufs make_bufs(pci_batch *b, const pci_batch_params *p)
{
    Bufs B;
    B.V = b->d_V; B.W = b->d_W; B.R = b->d_R; B.T = b->d_T; B.T2 = b->d_T2; B.P = b->d_P; B.Q = b->d_Q;
    B.G = b->d_G; B.EV = b->d_EV; B.EW = b->d_EW; B.part = b->d_part; B.coef = b->d_coef; B.D = b->d_D;
    B.P32 = b->d_P32; B.Q32 = b->d_Q32;
    B.Xk = nullptr;
    B.ld = b->rows;
    B.msub = p ? p->max_sub : BT_MS;
    B.nlv = p ? p->nlv : b->cap_nlv;
    B.keep = p ? p->keep : 0;
    B.max_it = p ? p->max_it : 0;
    B.tol = p ? p->tol : 0.0;
    B.swtol = p ? p->switch_tol : 0.0;
    B.stall_max = p ? (p->stall_max > 0 ? p->stall_max : 8) : 8;
    return B;
}

static int set_attrs(pci_batch *b)
{
    pci_gpu *h = &b->core;
    PCI_CUDA(h, cudaFuncSetAttribute(kb_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * BT_MS * BT_MS * 8));
    PCI_CUDA(h, cudaFuncSetAttribute(kb_rotate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (BT_MS * BT_MS + BT_MS * BT_ROT_THREADS) * 8));
    if (b->model)
        PCI_CUDA(h, cudaFuncSetAttribute(kb_learned, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mlptc::smem_bytes(mlp_num_inputs(b->model))));
    return PCI_OK;
}

// One SpMM of every running block in `phase`.
template <typename XT>
static cudaError_t spmm_all(pci_batch *b, int nv, int variant, cudaStream_t st, int phase, const XT *X, XT *Y)
{
    launch_spmm<XT>(nv, variant, b->nsm, st, b->d_blk, b->d_row_blk, b->d_st, b->rows, phase, X, Y);
    return cudaGetLastError();
}

// One iteration of every running block (25 launches, one more for the FP32
// SpMM of the mixed-precision form, one more for the learned correction and
// one more while harvesting samples; no host synchronisation).
static int enqueue_iteration(pci_batch *b, const Bufs &B, int variant, int nv, bool mixed, bool learned)
{
    pci_gpu *h = &b->core;
    cudaStream_t st = h->st;
    const int nch = b->nch, nblk = (int)b->blocks.size();
    kb_pack<<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    if (mixed) PCI_CUDA(h, spmm_all<float>(b, nv, variant, st, 0, B.P32, B.Q32));
    PCI_CUDA(h, spmm_all<double>(b, nv, variant, st, 1, B.P, B.Q));
    kb_tn<TN_GRAM><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_GRAM><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_eig<<<nblk, 256, 2 * BT_MS * BT_MS * 8, st>>>(b->d_st, B);
    kb_resid<<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_RESID><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    if (B.Xk)
        kb_harvest<<<b->nsm * 4, 256, 0, st>>>(b->d_hv_rows, b->hv_n, b->d_row_blk, b->d_blk, b->d_st, B, b->d_hv,
                                               b->hv_cap, b->d_hv_count);
    kb_rotate<<<nch, BT_ROT_THREADS, (BT_MS * BT_MS + BT_MS * BT_ROT_THREADS) * 8, st>>>(b->d_chunks, b->d_st, B);
    kb_correct<<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    if (learned)
        kb_learned<<<b->nsm * 2, 256, mlptc::smem_bytes(mlp_num_inputs(b->model)), st>>>(
            b->d_chunks, nch, b->d_blk, b->d_st, B, mlp_tc_weights(b->model));
    kb_tn<TN_TT><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_NORM><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_tn<TN_VT><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_VT1><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_proj<<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_tn<TN_VT><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_VT2><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_proj<<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_tn<TN_TT><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_CHOL1><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_tri<1><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_tn<TN_T2><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_fin<FIN_CHOL2><<<nblk, BT_FIN_THREADS, 0, st>>>(b->d_cb, b->d_st, B);
    kb_tri<2><<<nch, 256, 0, st>>>(b->d_chunks, b->d_st, B);
    kb_commit<<<(nblk + 127) / 128, 128, 0, st>>>(b->d_st, nblk);
    kb_count<<<1, 256, 0, st>>>(b->d_st, nblk, b->d_ndone);
    PCI_CUDA(h, cudaGetLastError());
    return PCI_OK;
}

static const int ITER_LAUNCHES = 25;
static const int LEARNED_LAUNCHES = 1;

static int prepare_harvest(pci_batch *b, Bufs &B, int nlv);

// The learned correction needs a model whose inputs cover every block's
// orbitals, and every block's determinant basis.
static int learned_ready(pci_batch *b)
{
    pci_gpu *h = &b->core;
    if (!b->model) return set_err(h, PCI_E_STATE, "learned correction requested without a model");
    const int nin = mlp_num_inputs(b->model);
    for (const BlockRec &r : b->blocks) {
        if (!r.orbs) return set_err(h, PCI_E_INPUT, "a block has no determinant basis (added from a CSR)");
        if (r.nsu > nin - mlptc::NSCAL) return set_err(h, PCI_E_INPUT, "a block has more orbitals than the model's inputs");
    }
    return PCI_OK;
}

// CUDA events released when the scope ends, on every return path.
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EventPair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    cudaError_t create()
    {
        cudaError_t e = cudaEventCreate(&a);
        return e != cudaSuccess ? e : cudaEventCreate(&b);
    }
};

// Device memory released when the scope ends.
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { dev_free(p); }
};

// Every block running and in SpMM phase `phase` (the state of a solve is
// overwritten: used before a solve, for timing).
__global__ void kb_set_phase(BState *bst, int nblk, int phase)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nblk) {
        bst[b].done = 0;
        bst[b].phase = phase;
    }
}

// One SpMM of every block with the given variant on P (FP64 vectors, phase 1)
// or P32 (FP32 vectors, phase 0), timed with events; average ms over `reps`.
static int time_spmm(pci_batch *b, int nv, int variant, int reps, int phase, double *ms)
{
    pci_gpu *h = &b->core;
    const int nblk = (int)b->blocks.size();
    EventPair ev;
    PCI_CUDA(h, ev.create());
    kb_set_phase<<<(nblk + 127) / 128, 128, 0, h->st>>>(b->d_st, nblk, phase);
    auto one = [&]() {
        return phase ? spmm_all<double>(b, nv, variant, h->st, 1, b->d_P, b->d_Q)
                     : spmm_all<float>(b, nv, variant, h->st, 0, b->d_P32, b->d_Q32);
    };
    PCI_CUDA(h, one());
    PCI_CUDA(h, cudaEventRecord(ev.a, h->st));
    for (int r = 0; r < reps; r++) {
        if (phase) PCI_CUDA(h, cudaMemsetAsync(b->d_Q, 0, 8 * b->rows * nv, h->st));
        else PCI_CUDA(h, cudaMemsetAsync(b->d_Q32, 0, 4 * b->rows * nv, h->st));
        PCI_CUDA(h, one());
    }
    PCI_CUDA(h, cudaEventRecord(ev.b, h->st));
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaEventSynchronize(ev.b));
    float f = 0.f;
    PCI_CUDA(h, cudaEventElapsedTime(&f, ev.a, ev.b));
    *ms = f / reps;
    return PCI_OK;
}

// Full symmetric copy of one block (lower triangle freed afterwards).
static int make_full(pci_batch *b, BlockRec &r)
{
    pci_gpu tmp;
    tmp.device = b->core.device;
    tmp.st = b->core.st;
    tmp.H = r.H;
    int rc = sp_build_full(&tmp);
    dev_free(tmp.d_tmp);
    tmp.d_tmp = nullptr;
    if (rc) {
        csr_free(tmp.Hfull);
        b->core.err = tmp.err;
        return rc;
    }
    r.F = tmp.Hfull;
    csr_free(r.H);
    return PCI_OK;
}

// With storage mode 1, blocks (largest first) get a full symmetric copy while
// the copy fits in the free device memory beside the solve buffers with a
// 4 GiB margin; the others stay lower triangles.
static int choose_storage(pci_batch *b)
{
    if (b->storage_done) return PCI_OK;
    b->storage_done = true;
    if (b->storage != 1) return PCI_OK;
    std::vector<int> order(b->blocks.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->blocks[x].nnz > b->blocks[y].nnz; });
    const size_t margin = (size_t)4 << 30;
    for (int i : order) {
        BlockRec &r = b->blocks[i];
        if (r.F.rowptr || r.split) continue;
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        // the copy (both triangles, FP32 + int32) and its build scratch
        const size_t need = (size_t)(2 * r.nnz) * 8 + (size_t)(r.nd + 1) * 24;
        if (need + margin > fr) continue;
        int rc = make_full(b, r);
        if (rc) return rc;
        b->full_nnz += r.nnz;
        b->dirty = true;
    }
    return PCI_OK;
}

static int prepare(pci_batch *b, int nlv)
{
    pci_gpu *h = &b->core;
    cudaSetDevice(h->device);
    if (b->blocks.empty()) return set_err(h, PCI_E_STATE, "batch has no blocks");
    int rc = build_tables(b);
    if (rc) return rc;
    if ((rc = ensure_solve(b, nlv))) return rc;
    if ((rc = choose_storage(b))) return rc;
    if ((rc = build_tables(b))) return rc;
    return set_attrs(b);
}

// Revision of the SpMM kernels, part of the cache key: cached picks of an
// older kernel are not reused.
static const int SPMM_REV = 8;

static std::string tune_key(pci_batch *b, int nv)
{
    std::ostringstream k;
    std::string dn = b->devname;
    for (char &c : dn)
        if (c == ' ') c = '_';
    int f64 = 0, split = 0;
    for (const BlockRec &r : b->blocks) {
        f64 += (r.F.rowptr ? !r.F.val_f32 : !r.H.val_f32) && !r.split;
        split += r.split;
    }
    k << dn << "|rev=" << SPMM_REV << "|storage=" << b->storage << "|full=" << b->full_nnz << "|f64=" << f64
      << "|split=" << split
      << "|blocks=" << b->blocks.size() << "|rows=" << b->rows << "|nnz=" << b->nnz << "|nv=" << nv;
    return k.str();
}

extern "C" {

int pci_batch_create(int32_t device, pci_batch_t **out)
{
    if (!out) return PCI_E_INPUT;
    pci_batch *b = new pci_batch();
    *out = b;
    b->core.device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_err(&b->core, e, "cudaSetDevice");
    e = cudaStreamCreateWithFlags(&b->core.st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_err(&b->core, e, "cudaStreamCreate");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
        b->nsm = prop.multiProcessorCount;
        b->devname = prop.name;
    }
    return PCI_OK;
}

int pci_batch_add_block(pci_batch_t *b, pci_gpu_t *h, int32_t *index)
{
    if (!b || !h) return PCI_E_INPUT;
    pci_gpu *c = &b->core;
    if (h->device != c->device) return set_err(c, PCI_E_INPUT, "block handle is on another device");
    if (!h->H.rowptr) return set_err(c, PCI_E_STATE, "the handle holds no Hamiltonian");
    if (h->h_pt_nd1 >= 0) return set_err(c, PCI_E_STATE, "the handle holds conf_pt's PT block, not a Hamiltonian");
    if (b->blocks.size() >= (size_t)INT32_MAX) return set_err(c, PCI_E_INPUT, "too many blocks");
    if (b->rows + h->H.nrows >= (int64_t)1 << 40) return set_err(c, PCI_E_INPUT, "too many rows");
    cudaSetDevice(c->device);
    BlockRec r;
    r.H = h->H;
    h->H = Csr();   // the batch owns the matrix from here on, error paths included
    r.r0 = b->rows;
    r.nd = r.H.nrows;
    r.nnz = r.H.nnz;
    // on an error return the block's device buffers are released
    struct Release {
        BlockRec *r;
        bool armed = true;
        ~Release()
        {
            if (!armed) return;
            csr_free(r->H);
            dev_free(r->orbs);
            dev_free(r->D);
        }
    } release{&r};
    if (h->have_basis && h->d_occ && h->d_ms_orb && h->nd == r.nd && h->nsu <= 254 && h->ne <= mlptc::MAXOCC) {
        // the occupied orbitals of every row: inputs of the learned correction
        int rc = 0;
        r.orbs = (uint8_t *)dev_alloc(c, (size_t)std::max<int64_t>(r.nd, 1) * mlptc::MAXOCC, &rc);
        if (rc) return rc;
        kb_row_orbs<<<b->nsm * 4, 256, 0, c->st>>>(h->d_occ, h->d_ms_orb, h->ne, r.nd, r.orbs);
        PCI_CUDA(c, cudaGetLastError());
        PCI_CUDA(c, cudaStreamSynchronize(c->st));
        r.nsu = h->nsu;
    }
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    if (r.H.cap > r.H.nnz && (size_t)r.H.nnz * 8 + ((size_t)1 << 30) < fr) {
        // a padded build leaves its candidate slots allocated: keep nnz of them
        // (when a copy of the values fits beside them)
        int rc = 0;
        const int64_t n = std::max<int64_t>(r.H.nnz, 1);
        int32_t *col = (int32_t *)dev_alloc(c, n * 4, &rc);
        if (rc) return rc;
        PCI_CUDA(c, cudaMemcpyAsync(col, r.H.col, r.H.nnz * 4, cudaMemcpyDeviceToDevice, c->st));
        PCI_CUDA(c, cudaStreamSynchronize(c->st));
        dev_free(r.H.col);
        r.H.col = col;
        if (r.H.val_f32 || b->value_prec != 32) {
            const size_t vb = r.H.val_f32 ? 4 : 8;
            void *val = dev_alloc(c, n * vb, &rc);
            if (rc) return rc;
            PCI_CUDA(c, cudaMemcpyAsync(val, r.H.val, r.H.nnz * vb, cudaMemcpyDeviceToDevice, c->st));
            PCI_CUDA(c, cudaStreamSynchronize(c->st));
            dev_free(r.H.val);
            r.H.val = val;
        }
        r.H.cap = 0;
    }
    if (!r.H.val_f32 && b->value_prec == 48) {
        // in place: each FP64 value becomes {hi, lo} = {(float)v, (float)(v - hi)}
        k_split<<<b->nsm * 8, 256, 0, c->st>>>((double *)r.H.val, r.H.nnz);
        PCI_CUDA(c, cudaGetLastError());
        PCI_CUDA(c, cudaStreamSynchronize(c->st));
        r.split = 1;
    }
    if (!r.H.val_f32 && b->value_prec == 32) {
        int rc = 0;
        float *v = (float *)dev_alloc(c, std::max<int64_t>(r.H.nnz, 1) * 4, &rc);
        if (rc) return rc;
        k_to_f32<<<b->nsm * 8, 256, 0, c->st>>>((const double *)r.H.val, v, r.H.nnz);
        PCI_CUDA(c, cudaGetLastError());
        PCI_CUDA(c, cudaStreamSynchronize(c->st));
        dev_free(r.H.val);
        r.H.val = v;
        r.H.val_f32 = 1;
    }
    {   // the block's diagonal, while its CSR columns are there
        int rc = 0;
        r.D = (double *)dev_alloc(c, 8 * (size_t)std::max<int64_t>(r.nd, 1), &rc);
        if (rc) return rc;
        kb_diag_blk<<<b->nsm * 8, 256, 0, c->st>>>(r.H.rowptr, r.H.col, r.H.val, (r.H.val_f32 || r.split) ? 0 : 1,
                                                   r.split, r.nd, r.D);
        PCI_CUDA(c, cudaGetLastError());
        PCI_CUDA(c, cudaStreamSynchronize(c->st));
    }
    release.armed = false;
    csr_free(h->Hfull);
    h->h_from_tiles = false;
    b->blocks.push_back(r);
    b->rows += r.H.nrows;
    b->nnz += r.H.nnz;
    b->dirty = true;
    b->storage_done = false;
    b->tuned_variant = -1;
    free_solve(b);
    if (index) *index = (int32_t)(b->blocks.size() - 1);
    return PCI_OK;
}

int pci_batch_set_value_prec(pci_batch_t *b, int32_t value_prec)
{
    if (!b) return PCI_E_INPUT;
    if (value_prec != 32 && value_prec != 64 && value_prec != 48)
        return set_err(&b->core, PCI_E_INPUT, "value_prec must be 32, 48 (FP32 hi + lo) or 64");
    b->value_prec = value_prec;
    return PCI_OK;
}

int pci_batch_set_storage(pci_batch_t *b, int32_t mode)
{
    if (!b) return PCI_E_INPUT;
    if (mode != 0 && mode != 1) return set_err(&b->core, PCI_E_INPUT, "storage mode must be 0 or 1");
    if (b->storage_done && mode != b->storage && b->full_nnz)
        return set_err(&b->core, PCI_E_STATE, "full copies already made; set the storage before the first solve");
    b->storage = mode;
    b->storage_done = false;
    b->tuned_variant = -1;
    return PCI_OK;
}

int pci_batch_info(pci_batch_t *b, int32_t *nblocks, int64_t *rows, int64_t *nnz)
{
    if (!b) return PCI_E_INPUT;
    if (nblocks) *nblocks = (int32_t)b->blocks.size();
    if (rows) *rows = b->rows;
    if (nnz) *nnz = b->nnz;
    return PCI_OK;
}

int pci_batch_variant(int32_t variant, int32_t *lanes_per_row, int32_t *blocks_per_sm)
{
    if (variant < 0 || variant >= N_VARIANTS) return N_VARIANTS;
    if (lanes_per_row) *lanes_per_row = SUBS[variant / N_CTAS];
    if (blocks_per_sm) *blocks_per_sm = CTAS[variant % N_CTAS];
    return PCI_OK;
}

int pci_batch_tune(pci_batch_t *b, int32_t nv, const char *cache_path, int32_t *variant, double *ms,
                   int32_t *from_cache)
{
    if (!b) return PCI_E_INPUT;
    pci_gpu *h = &b->core;
    if (nv < 1 || nv > BT_LV) return set_err(h, PCI_E_INPUT, "nv must be 1..12");
    int rc = prepare(b, nv);
    if (rc) return rc;
    const std::string key = tune_key(b, nv);
    int best = -1;
    double best_ms = 0.0;
    int cached = 0;
    if (cache_path) {
        std::ifstream f(cache_path);
        std::string tag, k;
        int v;
        double t;
        while (f >> tag >> k >> v >> t)
            if (tag == "pci_batch_spmm" && k == key && variant_ok(nv, v)) { best = v; best_ms = t; cached = 1; }
    }
    if (best < 0) {
        // every block running, P = 1
        PCI_CUDA(h, cudaMemsetAsync(b->d_st, 0, sizeof(BState) * b->blocks.size(), h->st));
        std::vector<double> ones(std::min<int64_t>(b->rows * nv, (int64_t)1 << 20), 1.0);
        for (int64_t o = 0; o < b->rows * nv; o += (int64_t)ones.size()) {
            const int64_t n = std::min<int64_t>((int64_t)ones.size(), b->rows * nv - o);
            PCI_CUDA(h, cudaMemcpyAsync(b->d_P + o, ones.data(), 8 * n, cudaMemcpyHostToDevice, h->st));
            PCI_CUDA(h, cudaStreamSynchronize(h->st));
        }
        for (int v = 0; v < N_VARIANTS; v++) {
            if (!variant_ok(nv, v)) continue;
            double t = 0.0;
            if ((rc = time_spmm(b, nv, v, 3, 1, &t))) return rc;
            if (best < 0 || t < best_ms) { best = v; best_ms = t; }
        }
        if (cache_path) {
            std::ofstream f(cache_path, std::ios::app);
            if (f) f << std::setprecision(9) << "pci_batch_spmm " << key << " " << best << " " << best_ms << "\n";
        }
    }
    b->tuned_variant = best;
    b->tuned_nv = nv;
    b->tuned_ms = best_ms;
    if (variant) *variant = best;
    if (ms) *ms = best_ms;
    if (from_cache) *from_cache = cached;
    return PCI_OK;
}

int pci_batch_davidson(pci_batch_t *b, const pci_batch_params *p, double *E, double *rnorm, int32_t *iters,
                       int32_t *status, int32_t *graph_launches)
{
    if (!b || !p) return PCI_E_INPUT;
    pci_gpu *h = &b->core;
    const int nlv = p->nlv;
    if (nlv < 1 || nlv > BT_LV) return set_err(h, PCI_E_INPUT, "nlv must be 1..12");
    if (p->max_sub < 2 * nlv || p->max_sub > BT_MS) return set_err(h, PCI_E_INPUT, "max_sub must be 2*nlv..PCI_BATCH_MAX_SUB");
    if (p->keep < nlv || p->keep > p->max_sub - nlv) return set_err(h, PCI_E_INPUT, "keep must be nlv..max_sub-nlv");
    if (p->max_it < 1 || p->it_per_graph < 1 || !(p->tol > 0.0)) return set_err(h, PCI_E_INPUT, "bad max_it/it_per_graph/tol");
    if (p->precision != PCI_BATCH_FP64 && p->precision != PCI_BATCH_MIXED)
        return set_err(h, PCI_E_INPUT, "precision must be PCI_BATCH_FP64 or PCI_BATCH_MIXED");
    const bool mixed = p->precision == PCI_BATCH_MIXED;
    if (mixed && !(p->switch_tol >= p->tol)) return set_err(h, PCI_E_INPUT, "switch_tol must be >= tol");
    if (p->correction != PCI_BATCH_CORR_DIAG && p->correction != PCI_BATCH_CORR_LEARNED)
        return set_err(h, PCI_E_INPUT, "correction must be PCI_BATCH_CORR_DIAG or PCI_BATCH_CORR_LEARNED");
    if (p->spmm_variant >= 0 && !variant_ok(nlv, p->spmm_variant))
        return set_err(h, PCI_E_INPUT, "unknown SpMM variant, or fewer lanes per row than vectors");
    for (const BlockRec &r : b->blocks)
        if (r.nd < nlv) return set_err(h, PCI_E_INPUT, "a block has fewer rows than nlv");
    auto t0 = std::chrono::steady_clock::now();
    int rc = prepare(b, nlv);
    if (rc) return rc;
    const bool learned = p->correction == PCI_BATCH_CORR_LEARNED;
    if (learned && (rc = learned_ready(b))) return rc;
    const int nblk = (int)b->blocks.size();
    const int variant = p->spmm_variant >= 0 ? p->spmm_variant
                        : (b->tuned_variant >= 0 && b->tuned_nv == nlv ? b->tuned_variant : DEFAULT_VARIANT);
    Bufs B = make_bufs(b, p);
    b->last_nlv = nlv;
    if ((rc = prepare_harvest(b, B, nlv))) return rc;

    // SpMM time per call (FP64 vectors, and FP32 vectors for the mixed form), outside the solve
    PCI_CUDA(h, cudaMemsetAsync(b->d_P, 0, 8 * b->rows * nlv, h->st));
    PCI_CUDA(h, cudaMemsetAsync(b->d_P32, 0, 4 * b->rows * nlv, h->st));
    double spmm_ms = 0.0, spmm32_ms = 0.0;
    if ((rc = time_spmm(b, nlv, variant, 2, 1, &spmm_ms))) return rc;
    if (mixed && (rc = time_spmm(b, nlv, variant, 2, 0, &spmm32_ms))) return rc;

    EventPair ev;
    PCI_CUDA(h, ev.create());
    // initial basis: unit vectors at the nlv lowest diagonal elements of each block
    std::vector<double> D(b->rows);
    PCI_CUDA(h, cudaMemcpy(D.data(), b->d_D, 8 * b->rows, cudaMemcpyDeviceToHost));
    std::vector<int64_t> pos;
    std::vector<BState> st0(nblk);
    for (int i = 0; i < nblk; i++) {
        const BlockRec &r = b->blocks[i];
        std::vector<int64_t> idx(r.nd);
        for (int64_t n = 0; n < r.nd; n++) idx[n] = n;
        std::partial_sort(idx.begin(), idx.begin() + nlv, idx.end(), [&](int64_t a, int64_t c) {
            const double da = D[r.r0 + a], dc = D[r.r0 + c];
            return da < dc || (da == dc && a < c);
        });
        for (int s = 0; s < nlv; s++) pos.push_back((int64_t)s * b->rows + r.r0 + idx[s]);
        BState s{};
        s.m = nlv;
        s.knew = nlv;
        s.phase = mixed ? 0 : 1;
        s.best = 1e300;
        for (int j = 0; j < BT_LV; j++) s.lrn[j] = learned ? 1 : 0;
        st0[i] = s;
    }
    DevBuf d_pos;
    d_pos.p = dev_alloc(h, 8 * pos.size(), &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaEventRecord(ev.a, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(d_pos.p, pos.data(), 8 * pos.size(), cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemcpyAsync(b->d_st, st0.data(), sizeof(BState) * nblk, cudaMemcpyHostToDevice, h->st));
    PCI_CUDA(h, cudaMemsetAsync(b->d_V, 0, 8 * b->rows * BT_MS, h->st));
    PCI_CUDA(h, cudaMemsetAsync(b->d_G, 0, 8 * (int64_t)nblk * BT_MS * BT_MS, h->st));
    kb_set_units<<<((int)pos.size() + 255) / 256, 256, 0, h->st>>>(b->d_V, b->rows, (const int64_t *)d_pos.p,
                                                                   (int)pos.size());
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    auto t1 = std::chrono::steady_clock::now();

    // capture it_per_graph iterations once, replay until every block is done
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    PCI_CUDA(h, cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < p->it_per_graph && !rc; i++) rc = enqueue_iteration(b, B, variant, nlv, mixed, learned);
    cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (ce != cudaSuccess) return cuda_err(h, ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) { cudaGraphDestroy(graph); return cuda_err(h, ce, "cudaGraphInstantiate"); }
    int replays = 0, ndone = 0;
    const int max_replays = (p->max_it + p->it_per_graph - 1) / p->it_per_graph + 1;
    while (replays < max_replays) {
        ce = cudaGraphLaunch(exec, h->st);
        if (ce != cudaSuccess) break;
        replays++;
        ce = cudaMemcpyAsync(&ndone, b->d_ndone, 4, cudaMemcpyDeviceToHost, h->st);
        if (ce != cudaSuccess) break;
        ce = cudaStreamSynchronize(h->st);
        if (ce != cudaSuccess || ndone == nblk) break;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_err(h, ce, "graph replay");
    kb_ritz<<<b->nch, 256, 0, h->st>>>(b->d_chunks, b->d_st, B);
    PCI_CUDA(h, cudaGetLastError());
    PCI_CUDA(h, cudaEventRecord(ev.b, h->st));
    std::vector<BState> sf(nblk);
    PCI_CUDA(h, cudaMemcpyAsync(sf.data(), b->d_st, sizeof(BState) * nblk, cudaMemcpyDeviceToHost, h->st));
    PCI_CUDA(h, cudaStreamSynchronize(h->st));
    float total = 0.f;
    PCI_CUDA(h, cudaEventElapsedTime(&total, ev.a, ev.b));
    if (B.Xk) {
        unsigned long long cnt = 0;
        PCI_CUDA(h, cudaMemcpy(&cnt, b->d_hv_count, 8, cudaMemcpyDeviceToHost));
        b->hv_last = (int64_t)cnt;
    }
    int maxit = 0, maxit32 = 0, switched = 0;
    for (int i = 0; i < nblk; i++) {
        for (int j = 0; j < nlv; j++) {
            if (E) E[(int64_t)i * nlv + j] = sf[i].theta[j];
            if (rnorm) rnorm[(int64_t)i * nlv + j] = sf[i].rnorm[j];
        }
        if (iters) iters[i] = sf[i].iters;
        if (status) status[i] = sf[i].done;
        maxit = std::max(maxit, sf[i].iters);
        maxit32 = std::max(maxit32, sf[i].it32);
        switched += sf[i].phase == 1 && mixed;
    }
    if (graph_launches) *graph_launches = replays;
    b->st_total = total;
    b->st_iters = maxit;
    b->st_spmm = spmm_ms;
    b->st_spmm32 = spmm32_ms;
    b->st_it32 = maxit32;
    b->st_switched = switched;
    b->st_variant = variant;
    b->st_setup = std::chrono::duration<double, std::milli>(t1 - t0).count();
    b->st_launches = ITER_LAUNCHES + (mixed ? 1 : 0) + (learned ? LEARNED_LAUNCHES : 0);
    return ndone == nblk ? PCI_OK : set_err(h, PCI_E_NOT_CONVERGED, "graph replays ended before every block stopped");
}

int pci_batch_set_correction_model(pci_batch_t *b, pci_mlp_t *m)
{
    if (!b) return PCI_E_INPUT;
    if (m && mlp_num_inputs(m) < mlptc::NSCAL + 1)
        return set_err(&b->core, PCI_E_INPUT, "the model needs at least 4 inputs");
    b->model = m;
    return PCI_OK;
}

int pci_batch_set_harvest(pci_batch_t *b, int32_t rows_per_block, int64_t capacity, int32_t seed)
{
    if (!b) return PCI_E_INPUT;
    if (rows_per_block < 0 || capacity < 0) return set_err(&b->core, PCI_E_INPUT, "negative harvest size");
    b->hv_per_block = rows_per_block;
    b->hv_cap = rows_per_block ? capacity : 0;
    b->hv_seed = seed;
    return PCI_OK;
}

int pci_batch_harvest(pci_batch_t *b, pci_batch_sample *out, int64_t cap, int64_t *count)
{
    if (!b) return PCI_E_INPUT;
    pci_gpu *h = &b->core;
    if (count) *count = b->hv_last;
    if (!out || cap <= 0 || !b->d_hv) return PCI_OK;
    const int64_t n = std::min<int64_t>(std::min<int64_t>(cap, b->hv_last), b->hv_cap);
    if (n > 0) PCI_CUDA(h, cudaMemcpy(out, b->d_hv, (size_t)n * sizeof(pci_batch_sample), cudaMemcpyDeviceToHost));
    return PCI_OK;
}

}  // extern "C"

// Sampled rows of every block (seeded, ascending) and the sample buffers for
// a solve that harvests; B.Xk set so kb_resid keeps the Ritz vectors.
static int prepare_harvest(pci_batch *b, Bufs &B, int nlv)
{
    pci_gpu *h = &b->core;
    B.Xk = nullptr;
    b->hv_last = 0;
    if (!b->hv_per_block || !b->hv_cap) return PCI_OK;
    std::vector<int64_t> rows;
    uint64_t st = 0x853C49E6748FEA9BULL ^ (uint64_t)(uint32_t)b->hv_seed;
    for (const BlockRec &r : b->blocks) {
        const int64_t k = std::min<int64_t>(b->hv_per_block, r.nd);
        std::vector<int64_t> pick;
        if (k == r.nd) {
            for (int64_t n = 0; n < r.nd; n++) pick.push_back(n);
        } else {   // Floyd's sampling of k distinct rows
            std::vector<int64_t> chosen;
            for (int64_t j = r.nd - k; j < r.nd; j++) {
                st ^= st << 13; st ^= st >> 7; st ^= st << 17;
                const int64_t t = (int64_t)(st % (uint64_t)(j + 1));
                if (std::find(chosen.begin(), chosen.end(), t) == chosen.end()) chosen.push_back(t);
                else chosen.push_back(j);
            }
            pick = chosen;
            std::sort(pick.begin(), pick.end());
        }
        for (int64_t n : pick) rows.push_back(r.r0 + n);
    }
    int rc = 0;
    dev_free(b->d_hv_rows);
    dev_free(b->d_Xk);
    b->d_hv_rows = (int64_t *)dev_alloc(h, 8 * std::max<size_t>(rows.size(), 1), &rc);
    if (rc) return rc;
    b->d_Xk = (double *)dev_alloc(h, 8 * (size_t)std::max<int64_t>(b->rows * nlv, 1), &rc);
    if (rc) return rc;
    if (!b->d_hv_count) {
        b->d_hv_count = (unsigned long long *)dev_alloc(h, 16, &rc);
        if (rc) return rc;
    }
    dev_free(b->d_hv);
    b->d_hv = (pci_batch_sample *)dev_alloc(h, sizeof(pci_batch_sample) * (size_t)b->hv_cap, &rc);
    if (rc) return rc;
    PCI_CUDA(h, cudaMemcpy(b->d_hv_rows, rows.data(), 8 * rows.size(), cudaMemcpyHostToDevice));
    PCI_CUDA(h, cudaMemset(b->d_hv_count, 0, 16));
    b->hv_n = (int64_t)rows.size();
    B.Xk = b->d_Xk;
    return PCI_OK;
}

extern "C" {

}  // extern "C"

namespace {
// Random FP64 reductions in teams of nv lanes onto nv consecutive words of a
// rows x nv array: the access pattern of the SpMM's transpose part.
__global__ void kb_red_probe(double *Y, uint32_t rows, int nv, int iters)
{
    const int lane = threadIdx.x & 31;
    const int teams = 32 / nv, team = lane / nv, v = lane - team * nv;
    if (team >= teams) return;
    uint32_t x = (uint32_t)((blockIdx.x * blockDim.x + threadIdx.x) / 32 * teams + team) * 2654435761u + 12345u;
    for (int i = 0; i < iters; i++) {
        x ^= x << 13; x ^= x >> 17; x ^= x << 5;
        atomicAdd(&Y[(size_t)(x % rows) * nv + v], 1.0);
    }
}
}  // namespace

extern "C" {

int pci_batch_probe_reduction(int32_t device, int64_t rows, int32_t nv, double *gbs)
{
    if (!gbs || rows < 1 || nv < 1 || nv > 32) return PCI_E_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return PCI_E_CUDA;
    double *Y = nullptr;
    if (cudaMalloc(&Y, (size_t)rows * nv * 8) != cudaSuccess) return PCI_E_OOM;
    cudaMemset(Y, 0, (size_t)rows * nv * 8);
    cudaDeviceProp prop;
    int nsm = 148;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) nsm = prop.multiProcessorCount;
    const int grid = nsm * 8, block = 256, iters = 400;
    EventPair ev;
    int rc = PCI_OK;
    if (ev.create() != cudaSuccess) rc = PCI_E_CUDA;
    if (!rc) {
        kb_red_probe<<<grid, block>>>(Y, (uint32_t)std::min<int64_t>(rows, UINT32_MAX), nv, 20);
        cudaEventRecord(ev.a);
        kb_red_probe<<<grid, block>>>(Y, (uint32_t)std::min<int64_t>(rows, UINT32_MAX), nv, iters);
        cudaEventRecord(ev.b);
        float ms = 0.f;
        if (cudaEventSynchronize(ev.b) != cudaSuccess || cudaEventElapsedTime(&ms, ev.a, ev.b) != cudaSuccess) rc = PCI_E_CUDA;
        const double reds = (double)grid * (block / 32) * (32 / nv) * nv * iters;
        if (!rc) *gbs = reds * 8.0 / (ms * 1e-3) / 1e9;
    }
    cudaFree(Y);
    return rc;
}

int pci_batch_vectors(pci_batch_t *b, int32_t blk, double *X)
{
    if (!b || !X) return PCI_E_INPUT;
    pci_gpu *h = &b->core;
    if (blk < 0 || blk >= (int)b->blocks.size()) return set_err(h, PCI_E_INPUT, "block index out of range");
    if (!b->d_R || !b->last_nlv) return set_err(h, PCI_E_STATE, "no solve yet");
    const BlockRec &r = b->blocks[blk];
    for (int j = 0; j < b->last_nlv; j++)
        PCI_CUDA(h, cudaMemcpy(X + (int64_t)j * r.nd, b->d_R + (int64_t)j * b->rows + r.r0, 8 * r.nd,
                               cudaMemcpyDeviceToHost));
    return PCI_OK;
}

int pci_batch_stats(pci_batch_t *b, double *out, int32_t n)
{
    if (!b || !out || n < 0) return PCI_E_INPUT;
    const double v[10] = {b->st_total, b->st_iters, b->st_spmm, b->st_variant, b->st_setup, b->st_launches,
                          b->nnz ? (double)b->full_nnz / (double)b->nnz : 0.0, b->st_spmm32, b->st_it32,
                          b->st_switched};
    for (int i = 0; i < n && i < 10; i++) out[i] = v[i];
    return PCI_OK;
}

const char *pci_batch_last_error(pci_batch_t *b)
{
    return b ? b->core.err.c_str() : "null batch";
}

void pci_batch_destroy(pci_batch_t *b)
{
    if (!b) return;
    cudaSetDevice(b->core.device);
    if (b->core.st) cudaStreamSynchronize(b->core.st);
    for (BlockRec &r : b->blocks) {
        csr_free(r.H);
        csr_free(r.F);
        dev_free(r.orbs);
        dev_free(r.D);
    }
    dev_free(b->d_hv_rows);
    dev_free(b->d_hv);
    dev_free(b->d_hv_count);
    dev_free(b->d_Xk);
    free_solve(b);
    free_tables(b);
    dev_free(b->core.d_tmp);
    if (b->core.st) cudaStreamDestroy(b->core.st);
    delete b;
}

}  // extern "C"
