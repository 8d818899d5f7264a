// Davidson eigensolver for the lowest Nlv levels (Diag4, src/pconf.F90:1993-2264,
// and the davidson module, src/davidson.f90), plain FP64 form.
//
// The iteration is the reference's, step for step: Ortn on the Nlv probe
// vectors, Mxmpy(1) + FormP(1), Dvdsn + Ortn for the corrections, Mxmpy(2) +
// FormP(2), the 2Nlv x 2Nlv projected eigenproblem, admixture test and FormB.
// Vectors stay on the device in one row-major block ArrB[Nd][3*Nlv] (column
// c of the reference's ArrB is element c of each row), so the SpMM gathers
// one contiguous Nlv-wide row of X per stored element.  The small decisions
// (convergence flags, the projected eigensolve) are taken on the host from a
// few scalars copied back per iteration; the orthogonalisation's pass logic
// runs in a one-thread kernel so an Ortn call needs no host round trip.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pci_internal.h"

#define FULL_MASK 0xffffffffu

namespace {

// ---------------------------------------------------------- host eigensolver

// Cyclic Jacobi for a symmetric n x n matrix (column-major a, overwritten).
// Returns eigenvalues ascending in w and eigenvectors as columns of v.
void jacobi_eig(int n, std::vector<double> &a, std::vector<double> &w, std::vector<double> &v)
{
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) v[i + (size_t)i * n] = 1.0;
    auto A = [&](int i, int j) -> double & { return a[i + (size_t)j * n]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double x = A(i, j) * A(i, j);
                tot += x;
                if (i != j) off += x;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++) {
            for (int q = p + 1; q < n; q++) {
                double apq = A(p, q);
                if (apq == 0.0) continue;
                double app = A(p, p), aqq = A(q, q);
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {
                    double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = v[k + (size_t)p * n], vkq = v[k + (size_t)q * n];
                    v[k + (size_t)p * n] = c * vkp - s * vkq;
                    v[k + (size_t)q * n] = s * vkp + c * vkq;
                }
            }
        }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int x, int y) { return A(x, x) < A(y, y); });
    w.resize(n);
    std::vector<double> vs((size_t)n * n);
    for (int j = 0; j < n; j++) {
        w[j] = A(idx[j], idx[j]);
        // sign convention: largest-magnitude component positive
        int im = 0;
        for (int k = 1; k < n; k++)
            if (fabs(v[k + (size_t)idx[j] * n]) > fabs(v[im + (size_t)idx[j] * n])) im = k;
        double sg = v[im + (size_t)idx[j] * n] < 0 ? -1.0 : 1.0;
        for (int k = 0; k < n; k++) vs[k + (size_t)j * n] = sg * v[k + (size_t)idx[j] * n];
    }
    v.swap(vs);
}

// ------------------------------------------------------------ kernels ---

constexpr int GRAM_ROWS = 32;
constexpr int GRAM_BLOCKS = 148 * 4;
// offsets into the device scratch of small vectors (doubles)
constexpr int SM_GRAM = 0;     // gram output / eigenvectors for FormB, <= 512
constexpr int SM_ORTN = 512;   // Ortn overlaps, <= 32
constexpr int SM_NORM = 576;   // Ortn norm
constexpr int SM_THETA = 640;  // Rayleigh quotients
constexpr int SM_TSEL = 672;   // quotients of unconverged levels
constexpr int SM_N2 = 704;     // squared correction norms
constexpr int SM_TOTAL = 768;

// partial[b][i*p + k] = sum over rows of this block of A[n][a0+i] * A[n][b0+k]
// (m*p <= 512: each thread owns the pairs t and t+256)
__global__ void __launch_bounds__(256) k_gram(const double *__restrict__ A, int ld, int64_t nd, int a0, int m,
                                               int b0, int p, double *__restrict__ partial)
{
    __shared__ double rows[GRAM_ROWS][64];
    const int t = threadIdx.x;
    const int mp = m * p;
    const int t2 = t + 256;
    const int i1 = t / p, k1 = t - i1 * p, i2 = t2 / p, k2 = t2 - i2 * p;
    double acc1 = 0.0, acc2 = 0.0;
    const int ncols = ld;
    for (int64_t r0 = blockIdx.x * (int64_t)GRAM_ROWS; r0 < nd; r0 += (int64_t)gridDim.x * GRAM_ROWS) {
        int nr = (int)min((int64_t)GRAM_ROWS, nd - r0);
        __syncthreads();
        for (int e = t; e < nr * ncols; e += blockDim.x) {
            int rr = e / ncols, cc = e - rr * ncols;
            rows[rr][cc] = A[(r0 + rr) * ld + cc];
        }
        __syncthreads();
        if (t < mp)
            for (int rr = 0; rr < nr; rr++) acc1 += rows[rr][a0 + i1] * rows[rr][b0 + k1];
        if (t2 < mp)
            for (int rr = 0; rr < nr; rr++) acc2 += rows[rr][a0 + i2] * rows[rr][b0 + k2];
    }
    if (t < mp) partial[(size_t)blockIdx.x * mp + t] = acc1;
    if (t2 < mp) partial[(size_t)blockIdx.x * mp + t2] = acc2;
}

__global__ void k_gram_reduce(const double *partial, int nblk, int mp, double *out)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= mp) return;
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += partial[(size_t)b * mp + t];
    out[t] = s;
}

// Ortn pass state: state 0 running, 1 done, 2 failed; sub = subtract in this
// pass; fail_* are sticky across calls and hold the 1-based vector index.
struct OrtnState {
    int state, sub, fail_ortho, fail_norm, j, pad;
    double smax2;
};

__global__ void k_ortn_begin(OrtnState *st, int j)
{
    st->state = 0;
    st->sub = 0;
    st->j = j;
    st->smax2 = 1e10;
}

// masks converged-level overlaps, decides the pass (src/davidson.f90:699-724)
__global__ void k_ortn_logic(OrtnState *st, double *s, int jm, int nlv, const int *iconv, int pass)
{
    if (st->state != 0) { st->sub = 0; return; }
    double smax1 = 0.0;
    for (int l = 1; l <= jm; l++) {
        if (l > nlv && iconv[l - nlv - 1] == 1) s[l - 1] = 0.0;
        else if (fabs(s[l - 1]) > smax1) smax1 = fabs(s[l - 1]);
    }
    st->sub = jm > 0;
    if (smax1 < 1e-6) st->state = 1;
    else if (smax1 > st->smax2 || pass > 3) { st->state = 2; if (!st->fail_ortho) st->fail_ortho = st->j; }
    st->smax2 = smax1;
}

__global__ void k_ortn_sub(double *A, int ld, int64_t nd, int j, int jm, const double *s, const OrtnState *st)
{
    if (!st->sub) return;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        const double *row = A + n * ld;
        for (int l = 0; l < jm; l++) acc += row[l] * s[l];
        A[n * ld + j] = row[j] - acc;
    }
}

__global__ void k_scale_col(double *A, int ld, int64_t nd, int j, const double *ss, OrtnState *st)
{
    double s = ss[0];
    if (blockIdx.x == 0 && threadIdx.x == 0 && s < 1e-9 && !st->fail_norm) st->fail_norm = st->j;
    double f = 1.0 / sqrt(s);
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        A[n * ld + j] *= f;
}

// Z1 = (H - Hmin)[0:nd0, 0:nd0] from the lower CSR (Init4, src/davidson.f90:45-63)
template <typename VT>
__global__ void k_extract_z1(const int64_t *rowptr, const int32_t *col, const VT *val, double hmin, int nd0, double *Z)
{
    int lane = threadIdx.x & 31;
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t n = warp; n < nd0; n += nwarps) {
        for (int64_t l = rowptr[n] + lane; l < rowptr[n + 1]; l += 32) {
            int k = col[l];
            double t = (double)val[l];
            if (k == n) t = t - hmin;
            if (k < nd0) {
                Z[n + (int64_t)k * nd0] = t;
                Z[k + (int64_t)n * nd0] = t;
            }
        }
    }
}

// Diag(n) = H_nn - Hmin (filled by the first Mxmpy in the reference)
template <typename VT>
__global__ void k_diag(const int64_t *rowptr, const int32_t *col, const VT *val, double hmin, int64_t nd, double *D)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        double d = 0.0;
        int64_t r1 = rowptr[n + 1];
        if (r1 > rowptr[n] && col[r1 - 1] == n) d = (double)val[r1 - 1] - hmin;  // diagonal is last in the row
        D[n] = d;
    }
}

// Residuals of all levels at once (Dvdsn, src/davidson.f90:477-486):
// t = HX_j - theta_j X_j; C[j*nd0 + n] = t for n < nd0; rows >= nd0 get the
// diagonal preconditioner t/(theta - Diag) written in place into column Nlv+j;
// per-block partial sums of t^2 go to part[b*nlv + j].
__global__ void __launch_bounds__(256) k_resid(double *A, int ld, int64_t nd, int nlv, int nd0, const double *theta,
                                               const double *D, double *C, double *part, int raw)
{
    __shared__ double red[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double acc[16];
    for (int j = 0; j < 16; j++) acc[j] = 0.0;
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        double *row = A + n * ld;
        for (int j = 0; j < nlv; j++) {
            double t = row[nlv + j] - theta[j] * row[j];
            acc[j] += t * t;
            if (n < nd0) C[(int64_t)j * nd0 + n] = t;
            else row[nlv + j] = raw ? t : t / (theta[j] - D[n]);
        }
    }
    for (int j = 0; j < nlv; j++) {
        double v = acc[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL_MASK, v, o);
        if (lane == 0) red[w][j & 31] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q][j & 31];
            part[(size_t)blockIdx.x * nlv + j] = s;
        }
        __syncthreads();
    }
}

// D[m + n ldd] += sum_k A(m, k) B(k, n) for m < M, n < N (N <= 16), k < K,
// with A(m, k) = A[m am + k ak] and B(k, n) = B[k + n ldb]: the two products
// of the Z1 projector (src/davidson.f90:526-544, DGEMV per level in the
// reference, here batched over the levels).  FP64 tensor cores (mma m8n8k4):
// one warp per 8 rows of D, K cut into gridDim.y slices added into D (zeroed
// by the caller) with atomics.
__global__ void __launch_bounds__(256) k_gemm_dmma(int M, int N, int K, const double *__restrict__ A, int64_t am,
                                                   int64_t ak, const double *__restrict__ B, int64_t ldb, double *D,
                                                   int64_t ldd)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int m0 = (int)(warp * 8);
    if (m0 >= M) return;
    const int kc = (K + gridDim.y - 1) / gridDim.y;
    const int kb = blockIdx.y * kc, ke = min(K, kb + kc);
    const int rw = lane >> 2, kq = lane & 3;
    const int m = m0 + rw;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
    for (int k0 = kb; k0 < ke; k0 += 4) {
        const int k = k0 + kq;
        const bool kin = k < ke;
        const double a = (m < M && kin) ? A[(int64_t)m * am + (int64_t)k * ak] : 0.0;
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
            const int n = nt * 8 + rw;
            const double b = (n < N && kin) ? B[k + (int64_t)n * ldb] : 0.0;
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(acc[nt][0]), "+d"(acc[nt][1])
                         : "d"(a), "d"(b));
        }
    }
#pragma unroll
    for (int nt = 0; nt < 2; nt++)
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int n = nt * 8 + 2 * kq + u;
            if (m < M && n < N) atomicAdd(&D[m + (int64_t)n * ldd], acc[nt][u]);
        }
}

// D (M x N, column-major, leading dimension ldd) = A B in slices of 16 columns.
static cudaError_t gemm_dmma(cudaStream_t st, int M, int N, int K, const double *A, int64_t am, int64_t ak,
                             const double *B, int64_t ldb, double *D, int64_t ldd)
{
    for (int n = 0; n < N; n++) {
        cudaError_t e = cudaMemsetAsync(D + (int64_t)n * ldd, 0, (size_t)M * 8, st);
        if (e != cudaSuccess) return e;
    }
    const int warps = (M + 7) / 8;
    const dim3 grid((warps + 7) / 8, (unsigned)std::max(1, std::min(32, K / 256)));
    for (int n0 = 0; n0 < N; n0 += 16)
        k_gemm_dmma<<<grid, 256, 0, st>>>(M, std::min(16, N - n0), K, A, am, ak, B + (int64_t)n0 * ldb, ldb,
                                          D + (int64_t)n0 * ldd, ldd);
    return cudaGetLastError();
}

// ------------------------------------------- eigenpairs of the initial block ---
// The reference diagonalises the Nd0 x Nd0 initial block with LAPACK DSYEVD
// (src/pconf.F90:1874-1889).  Here: one-sided cyclic Jacobi (Hestenes) on the
// block shifted to be positive definite (the shift is the Gershgorin bound
// max_i sum_j |a_ij|), whose right singular vectors are the eigenvectors and
// whose column norms, minus the shift, the eigenvalues.  Every round rotates
// n/2 disjoint column pairs (round-robin tournament order), one thread block
// per pair; a sweep is n - 1 rounds, replayed from a CUDA graph until no pair
// is rotated.

// Gershgorin bound of the column-major n x n block: bound = max over columns
// (the block is symmetric) of the absolute column sums.
__global__ void kj_gersh(const double *A, int n, double *colsum)
{
    const int j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += fabs(A[i + (int64_t)j * n]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        colsum[j] = t;
    }
}

// A += shift I; V = I.
__global__ void kj_init(double *A, double *V, int n, double shift)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        if (i == j) A[e] += shift;
        V[e] = i == j ? 1.0 : 0.0;
    }
}

__device__ __forceinline__ double block_sum256(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < 8; w++) t += red[w];
    __syncthreads();
    return t;
}

// Round r of a sweep over np (n rounded up to even) indices: pair t of the
// tournament; the index n (odd n) is a dummy.  Rotates columns p, q of U and V
// when their cosine |u_p . u_q| / (|u_p| |u_q|) exceeds tol; flag records it.
__global__ void __launch_bounds__(256) kj_round(double *U, double *V, int n, int np, int r, double tol, int *flag)
{
    __shared__ double red[8];
    const int t = blockIdx.x;
    int p, q;
    if (t == 0) { p = np - 1; q = r; }
    else { p = (r + t) % (np - 1); q = (r - t + np - 1) % (np - 1); }
    if (p > q) { const int x = p; p = q; q = x; }
    if (q >= n) return;
    double *up = U + (int64_t)p * n, *uq = U + (int64_t)q * n;
    double a = 0.0, b = 0.0, g = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = up[i], y = uq[i];
        a += x * x;
        b += y * y;
        g += x * y;
    }
    a = block_sum256(a, red);
    b = block_sum256(b, red);
    g = block_sum256(g, red);
    if (!(fabs(g) > tol * sqrt(a * b))) return;
    if (threadIdx.x == 0) *flag = 1;
    const double zeta = (b - a) / (2.0 * g);
    const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
    const double c = 1.0 / sqrt(1.0 + tt * tt), sn = c * tt;
    double *vp = V + (int64_t)p * n, *vq = V + (int64_t)q * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = up[i], y = uq[i];
        up[i] = c * x - sn * y;
        uq[i] = sn * x + c * y;
        const double xv = vp[i], yv = vq[i];
        vp[i] = c * xv - sn * yv;
        vq[i] = sn * xv + c * yv;
    }
}

// Column norms of U.
__global__ void kj_norms(const double *U, int n, double *out)
{
    __shared__ double red[8];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = U[i + (int64_t)j * n];
        s += x * x;
    }
    s = block_sum256(s, red);
    if (threadIdx.x == 0) out[j] = sqrt(s);
}

// Z[:, k] = V[:, perm[k]].
__global__ void kj_gather(const double *V, int n, const int *perm, double *Z)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, k = e / n;
        Z[e] = V[i + (int64_t)perm[k] * n];
    }
}

// s_vec(i) /= (theta - E1(i)), zero for |den| < 1e-6 (src/davidson.f90:531-538)
__global__ void k_zscale(double *S, int nz, int nj, const double *E1s, const double *theta_sel)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nz * nj) return;
    int i = t % nz, j = t / nz;
    double den = theta_sel[j] - E1s[i];
    S[t] = fabs(den) < 1e-6 ? 0.0 : S[t] / den;
}

// squared norm of the correction: B (nd0 part, column-major nd0 x nj) plus
// rows >= nd0 of column Nlv+jsel[j]; partial sums per block
__global__ void __launch_bounds__(256) k_corr_norm(const double *A, int ld, int64_t nd, int nlv, int nd0, const double *B,
                                                   const int *jsel, int nj, double *part)
{
    const int lane = threadIdx.x & 31;
    for (int j = 0; j < nj; j++) {
        double acc = 0.0;
        int col = nlv + jsel[j];
        for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
            double x = n < nd0 ? B[(int64_t)j * nd0 + n] : A[n * ld + col];
            acc += x * x;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(FULL_MASK, acc, o);
        __shared__ double red[8];
        if (lane == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += red[q];
            part[(size_t)blockIdx.x * nj + j] = s;
        }
        __syncthreads();
    }
}

__global__ void k_corr_write(double *A, int ld, int64_t nd, int nlv, int nd0, const double *B, const int *jsel, int nj,
                             const double *norm2)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        for (int j = 0; j < nj; j++) {
            double s = 1.0 / sqrt(norm2[j]);
            int col = nlv + jsel[j];
            if (n < nd0) A[n * ld + col] = B[(int64_t)j * nd0 + n] * s;
            else A[n * ld + col] = A[n * ld + col] * s;
        }
    }
}

__global__ void k_zero_col(double *A, int ld, int64_t nd, int col)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        A[n * ld + col] = 0.0;
}

// X <- [X|D] * P(:, 0:nlv)   (FormB / FormBskip, src/davidson.f90:195-267)
__global__ void k_formb(double *A, int ld, int64_t nd, int nlv, const double *Pv)
{
    __shared__ double sp[32 * 16];
    for (int e = threadIdx.x; e < 2 * nlv * nlv; e += blockDim.x) sp[e] = Pv[e];
    __syncthreads();
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x) {
        double *row = A + n * ld;
        double in[32];
        for (int c = 0; c < 2 * nlv; c++) in[c] = row[c];
        for (int k = 0; k < nlv; k++) {
            double acc = 0.0;
            for (int c = 0; c < 2 * nlv; c++) acc += in[c] * sp[c + k * 2 * nlv];
            row[k] = acc;
        }
    }
}

// place initial vectors: column j of ArrB from column-major src (nrow x ncol, ld_src)
__global__ void k_put_cols(double *A, int ld, int64_t nd, const double *src, int64_t nrow, int64_t ldsrc, int c0, int ncol)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncol; c++) A[n * ld + c0 + c] = n < nrow ? src[n + (int64_t)c * ldsrc] : 0.0;
}

__global__ void k_get_cols(const double *A, int ld, int64_t nd, double *dst, int ncol)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int c = 0; c < ncol; c++) dst[n + (int64_t)c * nd] = A[n * ld + c];
}

// ----------------------------------------------------------- Kv = 3 ---

// AvgDiag (src/davidson.f90:371-434): each configuration's diagonal entries
// replaced by their average (sequential sum, as the reference).
__global__ void k_avg_diag(double *D, const int64_t *conf_start, int nc)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const int64_t a = conf_start[c], b = conf_start[c + 1];
        if (b > a) {
            double s = 0.0;
            for (int64_t i = a; i < b; i++) s += D[i];
            const double v = s / (double)(b - a);
            for (int64_t i = a; i < b; i++) D[i] = v;
        }
    }
}

// J^2 (lower-triangle CSR, 0-based columns) applied to the probe vectors of
// unconverged levels, columns cin.. -> cout.. (zeroed before), with the
// symmetric scatter of Prj_J (src/davidson.f90:811-826).
__global__ void k_jsq_apply(const int64_t *rowptr, const int32_t *col, const double *val, int64_t nd, double *A,
                            int ld, int cin, int cout, int nv, const int *iconv)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int64_t l = rowptr[n]; l < rowptr[n + 1]; l++) {
            const int64_t k = col[l];
            const double t = val[l];
            for (int v = 0; v < nv; v++) {
                if (iconv[v]) continue;
                atomicAdd(&A[n * ld + cout + v], t * A[k * ld + cin + v]);
                if (k != n) atomicAdd(&A[k * ld + cout + v], t * A[n * ld + cin + v]);
            }
        }
}

// Prj_J filter step a = x - f * J^2 x on unconverged levels
__global__ void k_prj_update(double *A, int ld, int64_t nd, int cin, int cout, int nv, double f, const int *iconv)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int v = 0; v < nv; v++)
            if (!iconv[v]) A[n * ld + cin + v] = A[n * ld + cin + v] - f * A[n * ld + cout + v];
}

__global__ void k_prj_scale(double *A, int ld, int64_t nd, int cin, int nv, const double *inv, const int *iconv)
{
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nd; n += (int64_t)gridDim.x * blockDim.x)
        for (int v = 0; v < nv; v++)
            if (!iconv[v]) A[n * ld + cin + v] *= inv[v];
}

// ------------------------------------------------ learned correction ---

// Features of rows n0 .. n0+cnt of level j for the correction model:
// occupation count of each orbital (Nsu values), D_n - theta_j, and the
// residual entry (raw, column col) times fscale = sqrt(Nd) / |r_j|.
__global__ void k_features(DevSys S, const double *A, int ld, const double *D, int64_t n0, int64_t cnt, int col,
                           double theta, float fscale, int nin, float *F)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = n0 + i;
        float *f = F + i * nin;
        for (int q = 0; q < nin - 2; q++) f[q] = 0.0f;
        for (int e = 0; e < S.ne; e++) {
            const int o = S.ms_orb[S.occ[n * S.ne + e]];
            if (o < nin - 2) f[o] += 1.0f;
        }
        f[nin - 2] = (float)(D[n] - theta);
        f[nin - 1] = (float)A[n * ld + col] * fscale;
    }
}

// rows n0 .. n0+cnt of column col <- y * scale (the model's correction)
__global__ void k_apply_net(double *A, int ld, int64_t n0, int64_t cnt, int col, const float *y, double scale)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        A[(n0 + i) * ld + col] = (double)y[i] * scale;
}

// rows n0 .. n0+cnt of column col: raw residual -> r / (theta - D) (Dvdsn's correction)
__global__ void k_apply_diag(double *A, int ld, const double *D, int64_t n0, int64_t cnt, int col, double theta)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = n0 + i;
        A[n * ld + col] = A[n * ld + col] / (theta - D[n]);
    }
}

__global__ void k_get_col(const double *A, int ld, int64_t n0, int64_t cnt, int col, double *out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = A[(n0 + i) * ld + col];
}

// sum of squares of x[0..n) into out (atomic)
template <typename T>
__global__ void k_sumsq(const T *x, int64_t n, int64_t stride, double *out)
{
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)x[i * stride];
        s += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(FULL_MASK, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

struct HarvestRec {
    int it = 0, j = 0;
    int64_t n0 = 0, cnt = 0;
    std::vector<float> feat;
    std::vector<double> xk;
};

// -------------------------------------------------- SpMM block packing ---

// The probe block goes to the SpMM as a contiguous Nd x nv array (the basis
// rows hold 3 Nlv columns), so the column gathers of the SpMM touch nv
// values per determinant instead of whole basis rows; in the FP32 form the
// packed block is float.
template <typename T>
__global__ void k_pack(const double *A, int ld, int64_t nd, int c0, int nv, T *P)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nd * nv; i += (int64_t)gridDim.x * blockDim.x)
        P[i] = (T)A[(i / nv) * ld + c0 + (i % nv)];
}

template <typename T>
__global__ void k_unpack(const T *P, int64_t nd, int nv, double *A, int ld, int c0)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nd * nv; i += (int64_t)gridDim.x * blockDim.x)
        A[(i / nv) * ld + c0 + (i % nv)] = (double)P[i];
}

// ------------------------------------------------------------ driver ---

struct Dvd {
    pci_gpu *h;
    cudaStream_t st;
    int64_t nd;
    int nlv, ld, nd0;
    double *A = nullptr, *D = nullptr, *Z1 = nullptr, *E1 = nullptr, *C = nullptr, *Bz = nullptr, *Sz = nullptr;
    double *part = nullptr, *small = nullptr;  // small: scratch scalars
    void *xp = nullptr, *yp = nullptr;         // packed SpMM input / output blocks
    bool learned = false;                      // learned correction on rows >= Nd0
    int nin = 0;
    int64_t chunk = 0;
    float *feat = nullptr, *yout = nullptr;    // features / model output of one chunk of rows
    double *ycol = nullptr;
    bool fp32 = false;                         // FP32 form: float blocks, FP32 SpMM
    OrtnState *ost = nullptr;
    int *iconv_d = nullptr, *jsel_d = nullptr;
    std::vector<int> iconv;
    int blocks = 148 * 4;
    float spmm_ms = 0;
    int spmm_calls = 0;
    cudaEvent_t ea = nullptr, eb = nullptr;
};

int gram(Dvd &d, int a0, int m, int b0, int p, double *out_dev)
{
    k_gram<<<GRAM_BLOCKS, 256, 0, d.st>>>(d.A, d.ld, d.nd, a0, m, b0, p, d.part);
    k_gram_reduce<<<(m * p + 255) / 256, 256, 0, d.st>>>(d.part, GRAM_BLOCKS, m * p, out_dev);
    return cudaGetLastError() == cudaSuccess ? PCI_OK : set_err(d.h, PCI_E_CUDA, "gram kernel failed");
}

// Ortn(j) for 1-based column j (src/davidson.f90:649-741)
int ortn(Dvd &d, int j)
{
    int jc = j - 1, jm = j - 1;
    double *s = d.small + SM_ORTN;
    double *ss = d.small + SM_NORM;
    k_ortn_begin<<<1, 1, 0, d.st>>>(d.ost, j);
    for (int pass = 1; pass <= 4; pass++) {
        if (jm > 0) {
            int rc = gram(d, 0, jm, jc, 1, s);
            if (rc) return rc;
        }
        k_ortn_logic<<<1, 1, 0, d.st>>>(d.ost, s, jm, d.nlv, d.iconv_d, pass);
        if (jm > 0) k_ortn_sub<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, d.nd, jc, jm, s, d.ost);
    }
    int rc = gram(d, jc, 1, jc, 1, ss);
    if (rc) return rc;
    k_scale_col<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, d.nd, jc, ss, d.ost);
    return cudaGetLastError() == cudaSuccess ? PCI_OK : set_err(d.h, PCI_E_CUDA, "ortn kernel failed");
}

int check_ortn(Dvd &d)
{
    OrtnState s;
    cudaMemcpyAsync(&s, d.ost, sizeof(s), cudaMemcpyDeviceToHost, d.st);
    cudaStreamSynchronize(d.st);
    if (s.fail_ortho) return set_err(d.h, PCI_E_ORTHO_FAIL, "Fail of orthogonalization of vector " + std::to_string(s.fail_ortho));
    if (s.fail_norm) return set_err(d.h, PCI_E_ORTHO_FAIL, "Fail of normalization of vector " + std::to_string(s.fail_norm));
    return PCI_OK;
}

int mxmpy(Dvd &d, int ip)
{
    int i2 = ip * d.nlv, i1 = i2 - d.nlv;
    cudaEventRecord(d.ea, d.st);
    int rc;
    if (d.fp32) {
        k_pack<float><<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, d.nd, i1, d.nlv, (float *)d.xp);
        rc = sp_spmm_f32(d.h, (const float *)d.xp, d.nlv, (float *)d.yp, d.nlv, d.nlv, d.st);
        if (!rc) k_unpack<float><<<d.blocks, 256, 0, d.st>>>((const float *)d.yp, d.nd, d.nlv, d.A, d.ld, i2);
    } else {
        k_pack<double><<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, d.nd, i1, d.nlv, (double *)d.xp);
        rc = sp_spmm(d.h, (const double *)d.xp, d.nlv, (double *)d.yp, d.nlv, d.nlv, d.st);
        if (!rc) k_unpack<double><<<d.blocks, 256, 0, d.st>>>((const double *)d.yp, d.nd, d.nlv, d.A, d.ld, i2);
    }
    cudaEventRecord(d.eb, d.st);
    cudaEventSynchronize(d.eb);
    float ms = 0;
    cudaEventElapsedTime(&ms, d.ea, d.eb);
    d.spmm_ms += ms;
    d.spmm_calls++;
    return rc;
}

void free_dvd(Dvd &d)
{
    dev_free(d.A); dev_free(d.D); dev_free(d.Z1); dev_free(d.E1); dev_free(d.C); dev_free(d.Bz); dev_free(d.Sz);
    dev_free(d.part); dev_free(d.small); dev_free(d.ost); dev_free(d.iconv_d); dev_free(d.jsel_d);
    dev_free(d.xp); dev_free(d.yp); dev_free(d.feat); dev_free(d.yout); dev_free(d.ycol);
    if (d.ea) cudaEventDestroy(d.ea);
    if (d.eb) cudaEventDestroy(d.eb);
}

}  // namespace

// Device memory released when the scope ends (allocation skipped once rc is set).
struct DevBlock {
    void *p = nullptr;
    DevBlock(pci_gpu *h, size_t bytes, int &rc)
    {
        if (!rc) p = dev_alloc(h, bytes, &rc);
    }
    ~DevBlock() { dev_free(p); }
};

// All eigenpairs of the symmetric n x n block A (column-major, device):
// on return A holds the eigenvectors as columns and E1 (host and E1_dev)
// the eigenvalues, ascending -- what DSYEVD returns (src/pconf.F90:1874-1889).
static int block_eigen(pci_gpu *h, cudaStream_t st, double *A, int n, double *E1_dev, std::vector<double> &E1)
{
    if (n <= 0) return PCI_OK;
    int rc = 0;
    DevBlock V(h, (size_t)n * n * 8, rc), tmp(h, (size_t)n * 8, rc), flag(h, 16, rc), perm(h, (size_t)n * 4, rc);
    if (rc) return rc;
    kj_gersh<<<n, 256, 0, st>>>(A, n, (double *)tmp.p);
    std::vector<double> cs(n);
    PCI_CUDA(h, cudaMemcpyAsync(cs.data(), tmp.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    PCI_CUDA(h, cudaStreamSynchronize(st));
    double shift = 0.0;
    for (double x : cs) shift = std::max(shift, x);
    shift = shift > 0.0 ? 1.01 * shift : 1.0;
    kj_init<<<148 * 4, 256, 0, st>>>(A, (double *)V.p, n, shift);
    PCI_CUDA(h, cudaGetLastError());
    const int np = n + (n & 1);
    const double tol = std::max(1e-15, std::sqrt((double)n) * 2.3e-16);
    bool converged = n == 1;
    if (!converged) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        PCI_CUDA(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int r = 0; r < np - 1; r++)
            kj_round<<<np / 2, 256, 0, st>>>(A, (double *)V.p, n, np, r, tol, (int *)flag.p);
        cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (ce != cudaSuccess) return cuda_err(h, ce, "Jacobi sweep capture");
        ce = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return cuda_err(h, ce, "Jacobi sweep instantiate");
        for (int sweep = 0; sweep < 60 && ce == cudaSuccess; sweep++) {
            int f = 0;
            ce = cudaMemsetAsync(flag.p, 0, 4, st);
            if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(&f, flag.p, 4, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            if (ce == cudaSuccess && !f) converged = true;
            if (converged) break;
        }
        cudaGraphExecDestroy(exec);
        if (ce != cudaSuccess) return cuda_err(h, ce, "Jacobi sweeps");
    }
    if (!converged) return set_err(h, PCI_E_CUDA, "eigenpairs of the initial block: Jacobi did not converge in 60 sweeps");
    kj_norms<<<n, 256, 0, st>>>(A, n, (double *)tmp.p);
    PCI_CUDA(h, cudaMemcpyAsync(cs.data(), tmp.p, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
    PCI_CUDA(h, cudaStreamSynchronize(st));
    std::vector<int> order(n);
    for (int j = 0; j < n; j++) order[j] = j;
    for (int j = 0; j < n; j++) cs[j] -= shift;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cs[x] < cs[y]; });
    for (int j = 0; j < n; j++) E1[j] = cs[order[j]];
    PCI_CUDA(h, cudaMemcpyAsync(perm.p, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
    kj_gather<<<148 * 4, 256, 0, st>>>((const double *)V.p, n, (const int *)perm.p, A);
    PCI_CUDA(h, cudaMemcpyAsync(E1_dev, E1.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
    PCI_CUDA(h, cudaStreamSynchronize(st));
    return PCI_OK;
}

int dv_run(pci_gpu *h, const pci_dvd_params *p, const double *X0, double *Tk_out, double *Tj_out,
           int32_t *Iconverge_out, double *X_out, int32_t *iters_out, double *resid_out, DvdHarvest *hv)
{
    if (!h->H.rowptr) return set_err(h, PCI_E_STATE, "davidson before form_h");
    if (!h->J.rowptr) return set_err(h, PCI_E_STATE, "davidson before form_j");
    if (p->Nlv < 1 || p->Nlv > 16) return set_err(h, PCI_E_INPUT, "Nlv must be 1..16");
    if (p->mode != PCI_DVD_FP64 && p->mode != PCI_DVD_FP32 && p->mode != PCI_DVD_LEARNED)
        return set_err(h, PCI_E_INPUT, "mode must be FP64, FP32 or LEARNED");
    if (p->mode == PCI_DVD_LEARNED && (!h->corr_model || mlp_num_inputs(h->corr_model) != h->nsu + 2))
        return set_err(h, PCI_E_INPUT, "the learned form needs a correction model with Nsu + 2 inputs");
    if (p->mode == PCI_DVD_FP32 && !h->H.val_f32)
        return set_err(h, PCI_E_INPUT, "the FP32 form needs H stored in FP32 (form_h with value_prec 32)");
    if (p->Kv != 3 && p->Kv != 4) return set_err(h, PCI_E_INPUT, "Kv must be 4 or 3");
    const int jav = (int)(2 * p->XJ_av + 0.1);
    if (p->Kv == 3 && jav != 0 && std::find(h->h_jterms.begin(), h->h_jterms.end(), 0) != h->h_jterms.end())
        // the filter factor 1/(jx(jx+2)) of Prj_J (src/davidson.f90:808) is 1/0 for a J = 0 term
        return set_err(h, PCI_E_INPUT, "Prj_J: a J = 0 term with XJ_av /= 0 divides by zero");
    Dvd d;
    d.h = h;
    d.st = h->st;
    d.nd = h->nd;
    int Nlv = p->Nlv;
    d.nlv = Nlv;
    d.ld = 3 * Nlv;
    const int64_t nd = h->nd;
    cudaEvent_t t0, t1, t2;
    cudaEventCreate(&t0); cudaEventCreate(&t1); cudaEventCreate(&t2);
    cudaEventCreate(&d.ea); cudaEventCreate(&d.eb);
    cudaEventRecord(t0, d.st);
    int rc = 0;
    // calcNd0 (src/determinants.f90:22-45)
    {
        int nc4 = p->Nc4 > 0 ? std::min(p->Nc4, h->nc) : h->nc;
        int64_t n1 = 0, n2 = 0, n0 = (int64_t)p->MaxNd0 + 1;
        for (int ic = 0; ic < nc4; ic++) {
            n1 += h->h_ndc[ic];
            if (n1 < n0) n2 = n1;
        }
        d.nd0 = (int)n2;
    }
    const int nd0 = d.nd0;
    if (nd0 < Nlv && p->Kl4 != 2) { free_dvd(d); return set_err(h, PCI_E_INPUT, "initial block Nd0 smaller than Nlv"); }
#define ALLOC(ptr, T, n)                                            \
    do {                                                            \
        ptr = (T *)dev_alloc(h, (size_t)(n) * sizeof(T), &rc);      \
        if (rc) { free_dvd(d); return rc; }                         \
    } while (0)
    ALLOC(d.A, double, nd * d.ld);
    ALLOC(d.D, double, nd);
    ALLOC(d.Z1, double, std::max<int64_t>((int64_t)nd0 * nd0, 1));
    ALLOC(d.E1, double, std::max(nd0, 1));
    ALLOC(d.C, double, std::max<int64_t>((int64_t)nd0 * Nlv, 1));
    ALLOC(d.Bz, double, std::max<int64_t>((int64_t)nd0 * Nlv, 1));
    ALLOC(d.Sz, double, std::max<int64_t>((int64_t)nd0 * Nlv, 1));
    ALLOC(d.part, double, (size_t)GRAM_BLOCKS * 512);
    ALLOC(d.small, double, SM_TOTAL);
    ALLOC(d.ost, OrtnState, 1);
    ALLOC(d.iconv_d, int, 16);
    ALLOC(d.jsel_d, int, 16);
    d.fp32 = p->mode == PCI_DVD_FP32;
    d.learned = p->mode == PCI_DVD_LEARNED;
    if (d.learned || hv) {
        d.nin = h->nsu + 2;
        d.chunk = std::max<int64_t>(1, std::min<int64_t>(nd - nd0, (int64_t)1 << 18));
        ALLOC(d.feat, float, d.chunk * d.nin);
        ALLOC(d.yout, float, std::max<int64_t>(1, nd - nd0));
        ALLOC(d.ycol, double, d.chunk);
    }
    ALLOC(d.xp, double, nd * Nlv);
    ALLOC(d.yp, double, nd * Nlv);
#undef ALLOC
    // the SpMM picks the full symmetric copy or the lower-triangle kernel by free memory
    PCI_CUDA(h, cudaMemsetAsync(d.A, 0, (size_t)nd * d.ld * 8, d.st));
    PCI_CUDA(h, cudaMemsetAsync(d.iconv_d, 0, 16 * 4, d.st));
    PCI_CUDA(h, cudaMemsetAsync(d.ost, 0, sizeof(OrtnState), d.st));
    const Csr &H = h->H;
    // Diag
    if (H.val_f32) k_diag<float><<<d.blocks, 256, 0, d.st>>>(H.rowptr, H.col, (const float *)H.val, h->hmin, nd, d.D);
    else k_diag<double><<<d.blocks, 256, 0, d.st>>>(H.rowptr, H.col, (const double *)H.val, h->hmin, nd, d.D);
    std::vector<double> E1(std::max(nd0, 1));
    // Init4 + DiagInitApprox
    if (nd0 > 0) {
        PCI_CUDA(h, cudaMemsetAsync(d.Z1, 0, (size_t)nd0 * nd0 * 8, d.st));
        if (H.val_f32) k_extract_z1<float><<<d.blocks, 256, 0, d.st>>>(H.rowptr, H.col, (const float *)H.val, h->hmin, nd0, d.Z1);
        else k_extract_z1<double><<<d.blocks, 256, 0, d.st>>>(H.rowptr, H.col, (const double *)H.val, h->hmin, nd0, d.Z1);
        if ((rc = block_eigen(h, d.st, d.Z1, nd0, d.E1, E1))) { free_dvd(d); return rc; }
    }
    cudaEventRecord(t1, d.st);
    // FormB0 (src/davidson.f90:75-193): initial vectors from the Nd0 block;
    // with Kv = 3 only eigenvectors with |J - XJ_av| <= 0.1 (J from J_av on
    // the first Nd0 rows) are taken, and Nlv becomes the number taken
    std::vector<int> acc;
    if (p->Kl4 != 2) {
        if (p->Kv == 3) {
            for (int j0 = 0; j0 < nd0 && (int)acc.size() < Nlv; j0 += 64) {
                const int nv = std::min(64, nd0 - j0);
                std::vector<double> xj(nv);
                if ((rc = sp_jav_strided(h, d.Z1 + (size_t)j0 * nd0, 1, nd0, nv, nd0, xj.data()))) { free_dvd(d); return rc; }
                for (int q = 0; q < nv && (int)acc.size() < Nlv; q++)
                    if (!(fabs(xj[q] - p->XJ_av) > 1e-1)) acc.push_back(j0 + q);
            }
            if (acc.empty()) { free_dvd(d); return set_err(h, PCI_E_INPUT, "FormB0: no initial vector has J = XJ_av"); }
        } else {
            for (int j = 0; j < Nlv; j++) acc.push_back(j);
        }
        Nlv = (int)acc.size();
        d.nlv = Nlv;
        d.ld = 3 * Nlv;
    }
    std::vector<double> E(2 * Nlv, 0.0), Tj(Nlv, 0.0), Tk(Nlv, 0.0);
    if (p->Kl4 == 2) {
        if (!X0) { free_dvd(d); return set_err(h, PCI_E_INPUT, "Kl4 = 2 needs X0"); }
        double *tmp = (double *)dev_alloc(h, (size_t)nd * Nlv * 8, &rc);
        if (rc) { free_dvd(d); return rc; }
        PCI_CUDA(h, cudaMemcpyAsync(tmp, X0, (size_t)nd * Nlv * 8, cudaMemcpyHostToDevice, d.st));
        k_put_cols<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, tmp, nd, nd, 0, Nlv);
        PCI_CUDA(h, cudaStreamSynchronize(d.st));
        dev_free(tmp);
    } else {
        for (int q = 0; q < Nlv; q++) {
            k_put_cols<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, d.Z1 + (size_t)acc[q] * nd0, nd0, nd0, q, 1);
            E[q] = -(E1[acc[q]] + h->hmin);
        }
    }
    // Davidson loop
    const DevSys S = make_devsys(h);
    std::vector<int> learned_on(Nlv, 1);
    std::vector<double> prev_cn(Nlv, 0.0);
    std::vector<HarvestRec> harvest;
    std::vector<double> P((size_t)4 * Nlv * Nlv, 0.0), Pt((size_t)2 * Nlv * Nlv), cn(Nlv, 0.0);
    std::vector<double> part_h((size_t)d.blocks * Nlv);
    d.iconv.assign(Nlv, 0);
    const double crit = p->admix_crit > 0 ? p->admix_crit : -1.0;
    double ax = 1.0, vmax = 0.0, cnx = 1.0;
    int it_done = 0, n1 = 2 * Nlv;
    const int n01 = (p->Kl4 == 2 || p->Kl4 == -2) ? 1 : Nlv + 1;
    const int nz = nd0 - n01 + 1;
    for (int it = 1; it <= p->N_it; it++) {
        if (!(ax > crit)) continue;
        it_done = it;
        for (int i = 1; i <= Nlv; i++) {
            if ((rc = ortn(d, i))) { free_dvd(d); return rc; }
        }
        if ((rc = check_ortn(d))) { free_dvd(d); return rc; }
        if ((rc = mxmpy(d, 1))) { free_dvd(d); return rc; }
        // FormP(1)
        if ((rc = gram(d, 0, Nlv, Nlv, Nlv, d.small + SM_GRAM))) { free_dvd(d); return rc; }
        PCI_CUDA(h, cudaMemcpyAsync(Pt.data(), d.small + SM_GRAM, (size_t)Nlv * Nlv * 8, cudaMemcpyDeviceToHost, d.st));
        PCI_CUDA(h, cudaStreamSynchronize(d.st));
        for (int i = 0; i < Nlv; i++)
            for (int k = 0; k <= i; k++) {
                double v = Pt[(size_t)i * Nlv + k];
                P[i + (size_t)k * n1] = v;
                P[k + (size_t)i * n1] = v;
            }
        if (it == 1 && p->Kv == 3)
            k_avg_diag<<<(h->nc + 255) / 256, 256, 0, d.st>>>(d.D, h->d_conf_start, h->nc);
        // Dvdsn for all levels: residual norms first
        std::vector<double> theta(Nlv);
        for (int j = 0; j < Nlv; j++) theta[j] = P[j + (size_t)j * n1];
        PCI_CUDA(h, cudaMemcpyAsync(d.small + SM_THETA, theta.data(), Nlv * 8, cudaMemcpyHostToDevice, d.st));
        const bool raw_rows = d.learned || hv;   // rows >= Nd0 keep the raw residual for the features
        k_resid<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, nd0, d.small + SM_THETA, d.D, d.C, d.part, raw_rows);
        PCI_CUDA(h, cudaGetLastError());
        PCI_CUDA(h, cudaMemcpyAsync(part_h.data(), d.part, (size_t)d.blocks * Nlv * 8, cudaMemcpyDeviceToHost, d.st));
        PCI_CUDA(h, cudaStreamSynchronize(d.st));
        cnx = 0.0;
        std::vector<int> jsel;
        for (int j = 0; j < Nlv; j++) {
            double s = 0.0;
            for (int b = 0; b < d.blocks; b++) s += part_h[(size_t)b * Nlv + j];
            cn[j] = sqrt(fabs(s));
            d.iconv[j] = cn[j] < p->Crt4 ? 1 : 0;
            if (cn[j] > cnx) cnx = cn[j];
            if (!d.iconv[j]) jsel.push_back(j);
        }
        PCI_CUDA(h, cudaMemcpyAsync(d.iconv_d, d.iconv.data(), Nlv * 4, cudaMemcpyHostToDevice, d.st));
        for (int j = 0; j < Nlv; j++)
            if (d.iconv[j]) k_zero_col<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv + j);
        if (raw_rows && nd > nd0) {
            // rows >= Nd0: the learned correction (with the diagonal one as the fallback of
            // each level whose residual stopped decreasing), or the diagonal one while harvesting
            const int64_t nrest = nd - nd0;
            const double rs = sqrt((double)nd);
            for (int j : jsel) {
                if (d.learned && it > 1 && learned_on[j] && cn[j] >= prev_cn[j]) learned_on[j] = 0;
                const bool use_net = d.learned && learned_on[j];
                const float fscale = (float)(rs / cn[j]);
                for (int64_t c0 = 0; c0 < nrest; c0 += d.chunk) {
                    const int64_t cnt = std::min<int64_t>(d.chunk, nrest - c0);
                    if (!use_net && !hv) break;
                    k_features<<<d.blocks, 256, 0, d.st>>>(S, d.A, d.ld, d.D, nd0 + c0, cnt, Nlv + j, theta[j], fscale,
                                                           d.nin, d.feat);
                    PCI_CUDA(h, cudaGetLastError());
                    if (hv) {
                        // features now; the current vector's rows to form the target after the solve
                        HarvestRec rec;
                        rec.it = it;
                        rec.j = j;
                        rec.n0 = nd0 + c0;
                        rec.cnt = cnt;
                        rec.feat.resize((size_t)cnt * d.nin);
                        rec.xk.resize((size_t)cnt);
                        PCI_CUDA(h, cudaMemcpyAsync(rec.feat.data(), d.feat, rec.feat.size() * 4, cudaMemcpyDeviceToHost, d.st));
                        k_get_col<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd0 + c0, cnt, j, d.ycol);
                        PCI_CUDA(h, cudaMemcpyAsync(rec.xk.data(), d.ycol, (size_t)cnt * 8, cudaMemcpyDeviceToHost, d.st));
                        PCI_CUDA(h, cudaStreamSynchronize(d.st));
                        harvest.push_back(std::move(rec));
                    }
                    if (use_net && (rc = mlp_forward_device(h->corr_model, d.feat, cnt, d.yout + c0, d.st))) {
                        free_dvd(d);
                        return set_err(h, rc, "learned correction: model forward failed");
                    }
                }
                // Dvdsn's correction r / (theta - D) on rows >= Nd0
                k_apply_diag<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, d.D, nd0, nrest, Nlv + j, theta[j]);
                if (use_net) {
                    // the model gives the direction on rows >= Nd0, the diagonal correction its length
                    PCI_CUDA(h, cudaMemsetAsync(d.small + SM_N2, 0, 16, d.st));
                    k_sumsq<double><<<d.blocks, 256, 0, d.st>>>(d.A + (size_t)nd0 * d.ld + Nlv + j, nrest, d.ld,
                                                                d.small + SM_N2);
                    k_sumsq<float><<<d.blocks, 256, 0, d.st>>>(d.yout, nrest, 1, d.small + SM_N2 + 1);
                    double n2[2];
                    PCI_CUDA(h, cudaMemcpyAsync(n2, d.small + SM_N2, 16, cudaMemcpyDeviceToHost, d.st));
                    PCI_CUDA(h, cudaStreamSynchronize(d.st));
                    if (n2[1] > 0.0 && std::isfinite(n2[1]))
                        k_apply_net<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd0, nrest, Nlv + j, d.yout, sqrt(n2[0] / n2[1]));
                }
                PCI_CUDA(h, cudaGetLastError());
            }
        }
        for (int j = 0; j < Nlv; j++) prev_cn[j] = cn[j];
        const int nj = (int)jsel.size();
        if (nj > 0) {
            // Z1 projection preconditioner on rows < nd0, batched over levels
            std::vector<double> tsel(nj);
            for (int q = 0; q < nj; q++) tsel[q] = theta[jsel[q]];
            PCI_CUDA(h, cudaMemcpyAsync(d.jsel_d, jsel.data(), nj * 4, cudaMemcpyHostToDevice, d.st));
            PCI_CUDA(h, cudaMemcpyAsync(d.small + SM_TSEL, tsel.data(), nj * 8, cudaMemcpyHostToDevice, d.st));
            // C columns of the selected levels -> contiguous Cs (reuse Bz)
            for (int q = 0; q < nj; q++)
                PCI_CUDA(h, cudaMemcpyAsync(d.Bz + (size_t)q * nd0, d.C + (size_t)jsel[q] * nd0, (size_t)nd0 * 8,
                                            cudaMemcpyDeviceToDevice, d.st));
            if (nz > 0 && nd0 > 0) {
                const double *Z1s = d.Z1 + (size_t)(n01 - 1) * nd0;
                // Sz = Z1s^T Bz, scaled by 1 / (theta - E1), then Bz = Z1s Sz
                PCI_CUDA(h, gemm_dmma(d.st, nz, nj, nd0, Z1s, nd0, 1, d.Bz, nd0, d.Sz, nz));
                k_zscale<<<(nz * nj + 255) / 256, 256, 0, d.st>>>(d.Sz, nz, nj, d.E1 + (n01 - 1), d.small + SM_TSEL);
                PCI_CUDA(h, gemm_dmma(d.st, nd0, nj, nz, Z1s, 1, nd0, d.Sz, nz, d.Bz, nd0));
            } else if (nd0 > 0) {
                PCI_CUDA(h, cudaMemsetAsync(d.Bz, 0, (size_t)nd0 * nj * 8, d.st));
            }
            k_corr_norm<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, nd0, d.Bz, d.jsel_d, nj, d.part);
            std::vector<double> np((size_t)d.blocks * nj), n2(nj, 0.0);
            PCI_CUDA(h, cudaMemcpyAsync(np.data(), d.part, np.size() * 8, cudaMemcpyDeviceToHost, d.st));
            PCI_CUDA(h, cudaStreamSynchronize(d.st));
            for (int q = 0; q < nj; q++)
                for (int b = 0; b < d.blocks; b++) n2[q] += np[(size_t)b * nj + q];
            PCI_CUDA(h, cudaMemcpyAsync(d.small + SM_N2, n2.data(), nj * 8, cudaMemcpyHostToDevice, d.st));
            k_corr_write<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, nd0, d.Bz, d.jsel_d, nj, d.small + SM_N2);
            for (int q = 0; q < nj; q++) {
                if ((rc = ortn(d, Nlv + jsel[q] + 1))) { free_dvd(d); return rc; }
            }
            if ((rc = check_ortn(d))) { free_dvd(d); return rc; }
        }
        if (p->Kv == 3) {
            // Prj_J(Nlv+1, Nlv, 2Nlv+1, 1e-5) (src/davidson.f90:743-884), then Ortn of the new vectors
            const std::vector<int32_t> &jt = h->h_jterms;
            const int njd = (int)jt.size();
            int jx = 0;
            double f = 0.0;
            std::vector<double> G((size_t)Nlv * Nlv), inv(Nlv, 1.0);
            const Csr &J = h->J;
            for (int iter = 1; iter <= njd + 1; iter++) {
                const int itj = njd + 1 - iter;
                if (itj != 0) {
                    jx = jt[itj - 1];
                    f = jx != 0 ? 1.0 / (double)(jx * (jx + 2)) : 0.0;   // jx = 0 is used only when J = 0 is the target
                }
                if (!(jx != jav || itj == 0)) continue;
                for (int v = 0; v < Nlv; v++) k_zero_col<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, 2 * Nlv + v);
                k_jsq_apply<<<d.blocks, 256, 0, d.st>>>(J.rowptr, J.col, (const double *)J.val, nd, d.A, d.ld, Nlv,
                                                        2 * Nlv, Nlv, d.iconv_d);
                PCI_CUDA(h, cudaGetLastError());
                if ((rc = gram(d, Nlv, Nlv, 2 * Nlv, Nlv, d.small + SM_GRAM))) { free_dvd(d); return rc; }
                PCI_CUDA(h, cudaMemcpyAsync(G.data(), d.small + SM_GRAM, G.size() * 8, cudaMemcpyDeviceToHost, d.st));
                PCI_CUDA(h, cudaStreamSynchronize(d.st));
                double err1 = 0.0;
                for (int v = 0; v < Nlv; v++)
                    if (!d.iconv[v]) err1 = std::max(err1, fabs(sqrt(1.0 + G[(size_t)v * Nlv + v]) - 1.0 - jav));
                if (err1 < 1e-5) break;
                if (itj != 0) {
                    k_prj_update<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, 2 * Nlv, Nlv, f, d.iconv_d);
                    if ((rc = gram(d, Nlv, Nlv, Nlv, Nlv, d.small + SM_GRAM))) { free_dvd(d); return rc; }
                    PCI_CUDA(h, cudaMemcpyAsync(G.data(), d.small + SM_GRAM, G.size() * 8, cudaMemcpyDeviceToHost, d.st));
                    PCI_CUDA(h, cudaStreamSynchronize(d.st));
                    for (int v = 0; v < Nlv; v++) inv[v] = d.iconv[v] ? 1.0 : 1.0 / sqrt(G[(size_t)v * Nlv + v]);
                    PCI_CUDA(h, cudaMemcpyAsync(d.small + SM_TSEL, inv.data(), Nlv * 8, cudaMemcpyHostToDevice, d.st));
                    k_prj_scale<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, Nlv, d.small + SM_TSEL, d.iconv_d);
                    PCI_CUDA(h, cudaGetLastError());
                }
            }
            for (int i = Nlv + 1; i <= 2 * Nlv; i++)
                if (!d.iconv[i - Nlv - 1] && (rc = ortn(d, i))) { free_dvd(d); return rc; }
            if ((rc = check_ortn(d))) { free_dvd(d); return rc; }
        }
        if (cnx > p->Crt4) {
            if ((rc = mxmpy(d, 2))) { free_dvd(d); return rc; }
            double pmax = P[0];
            for (int i = 1; i < Nlv; i++) pmax = std::max(pmax, P[i + (size_t)i * n1]);
            if (pmax > vmax) vmax = pmax;
            // FormP(2)
            if ((rc = gram(d, 0, 2 * Nlv, 2 * Nlv, Nlv, d.small + SM_GRAM))) { free_dvd(d); return rc; }
            PCI_CUDA(h, cudaMemcpyAsync(Pt.data(), d.small + SM_GRAM, (size_t)2 * Nlv * Nlv * 8, cudaMemcpyDeviceToHost, d.st));
            PCI_CUDA(h, cudaStreamSynchronize(d.st));
            auto PT = [&](int i, int k) { return Pt[(size_t)i * Nlv + k]; };  // Ptmp(i, k), i < 2Nlv, k < Nlv
            for (int i = 0; i < Nlv; i++)
                for (int k = Nlv; k < 2 * Nlv; k++) {
                    P[i + (size_t)k * n1] = PT(i, k - Nlv);
                    P[k + (size_t)i * n1] = PT(i, k - Nlv);
                }
            for (int i = Nlv; i < 2 * Nlv; i++)
                for (int k = Nlv; k <= i; k++) {
                    P[i + (size_t)k * n1] = PT(i, k - Nlv);
                    P[k + (size_t)i * n1] = PT(i, k - Nlv);
                }
            for (int i = 0; i < Nlv; i++)
                if (d.iconv[i] == 1) {
                    int i1 = i + Nlv;
                    for (int c = 0; c < n1; c++) { P[i1 + (size_t)c * n1] = 0.0; P[c + (size_t)i1 * n1] = 0.0; }
                    P[i1 + (size_t)i1 * n1] = 2 * vmax - P[i + (size_t)i * n1] + 1.0;
                }
            std::vector<double> w, V;
            jacobi_eig(n1, P, w, V);
            P = V;
            for (int i = 0; i < n1; i++) E[i] = w[i];
            ax = 0.0;
            vmax = -1e10;
            for (int i = 0; i < Nlv; i++) {
                double xx = 0.0;
                for (int k = 0; k < Nlv; k++) xx = std::max(xx, fabs(P[(k + Nlv) + (size_t)i * n1]));
                ax = std::max(ax, xx);
                vmax = std::max(vmax, E[i]);
            }
            PCI_CUDA(h, cudaMemcpyAsync(d.small + SM_GRAM, P.data(), (size_t)n1 * Nlv * 8, cudaMemcpyHostToDevice, d.st));
            k_formb<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, Nlv, d.small + SM_GRAM);
            PCI_CUDA(h, cudaGetLastError());
            for (int k = 0; k < Nlv; k++) Tk[k] = -(E[k] + h->hmin);
        } else {
            if (it == 1)
                for (int k = 0; k < Nlv; k++) Tk[k] = E[k];
            break;
        }
    }
    if (hv) {
        // targets of the recorded samples: the converged vector minus the vector of
        // that iteration (signs aligned), in units of the residual scale
        hv->count = 0;
        // targets per (iteration, level): the difference scaled to unit RMS over rows >= Nd0
        std::vector<std::vector<double>> dif(harvest.size());
        for (size_t r = 0; r < harvest.size(); r++) {
            const HarvestRec &rec = harvest[r];
            std::vector<double> xs((size_t)rec.cnt);
            if (hv->xref) {
                memcpy(xs.data(), hv->xref + (size_t)rec.j * nd + rec.n0, (size_t)rec.cnt * 8);
            } else {
                k_get_col<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, rec.n0, rec.cnt, rec.j, d.ycol);
                PCI_CUDA(h, cudaMemcpyAsync(xs.data(), d.ycol, (size_t)rec.cnt * 8, cudaMemcpyDeviceToHost, d.st));
                PCI_CUDA(h, cudaStreamSynchronize(d.st));
            }
            dif[r] = xs;
        }
        for (size_t g0 = 0; g0 < harvest.size();) {
            size_t g1 = g0;
            double dot = 0.0;
            int64_t rows = 0;
            while (g1 < harvest.size() && harvest[g1].it == harvest[g0].it && harvest[g1].j == harvest[g0].j) {
                for (int64_t i = 0; i < harvest[g1].cnt; i++) dot += dif[g1][i] * harvest[g1].xk[i];
                rows += harvest[g1].cnt;
                g1++;
            }
            const double sg = dot < 0.0 ? -1.0 : 1.0;
            double ss = 0.0;
            for (size_t r = g0; r < g1; r++)
                for (int64_t i = 0; i < harvest[r].cnt; i++) {
                    dif[r][i] = sg * dif[r][i] - harvest[r].xk[i];
                    ss += dif[r][i] * dif[r][i];
                }
            const double inv = ss > 0.0 ? sqrt((double)rows / ss) : 0.0;
            for (size_t r = g0; r < g1; r++)
                for (int64_t i = 0; i < harvest[r].cnt; i++, hv->count++) {
                    if (hv->count >= hv->cap) continue;
                    if (hv->feat)
                        memcpy(hv->feat + hv->count * d.nin, harvest[r].feat.data() + i * d.nin, (size_t)d.nin * 4);
                    if (hv->target) hv->target[hv->count] = (float)(dif[r][i] * inv);
                }
            g0 = g1;
        }
    }
    // WriteFinalXIJ: J of each level
    if ((rc = sp_jav(h, d.A, d.ld, Nlv, nd, Tj.data()))) { free_dvd(d); return rc; }
    if (X_out) {
        double *tmp = (double *)dev_alloc(h, (size_t)nd * Nlv * 8, &rc);
        if (rc) { free_dvd(d); return rc; }
        k_get_cols<<<d.blocks, 256, 0, d.st>>>(d.A, d.ld, nd, tmp, Nlv);
        PCI_CUDA(h, cudaMemcpyAsync(X_out, tmp, (size_t)nd * Nlv * 8, cudaMemcpyDeviceToHost, d.st));
        PCI_CUDA(h, cudaStreamSynchronize(d.st));
        dev_free(tmp);
    }
    cudaEventRecord(t2, d.st);
    cudaEventSynchronize(t2);
    float ms01 = 0, ms02 = 0;
    cudaEventElapsedTime(&ms01, t0, t1);
    cudaEventElapsedTime(&ms02, t0, t2);
    cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(t2);
    h->st_init = ms01;
    h->st_dvd = ms02;
    h->st_spmm = d.spmm_ms;
    h->st_spmm_calls = d.spmm_calls;
    for (int k = 0; k < Nlv; k++) {
        if (Tk_out) Tk_out[k] = Tk[k];
        if (Tj_out) Tj_out[k] = Tj[k];
        if (Iconverge_out) Iconverge_out[k] = d.iconv[k];
        if (resid_out) resid_out[k] = cn[k];
    }
    // levels FormB0 could not seed (Kv = 3: fewer initial vectors with J = XJ_av)
    for (int k = Nlv; k < p->Nlv; k++) {
        if (Tk_out) Tk_out[k] = 0.0;
        if (Tj_out) Tj_out[k] = 0.0;
        if (Iconverge_out) Iconverge_out[k] = -1;
        if (resid_out) resid_out[k] = 0.0;
        if (X_out) memset(X_out + (size_t)k * nd, 0, (size_t)nd * 8);
    }
    if (iters_out) *iters_out = it_done;
    free_dvd(d);
    return PCI_OK;
}
