// Learned Davidson correction: a small MLP (nin -> 128 -> 128 -> 128 -> 1,
// ReLU) with BF16 weights used by the forward and backward kernels and FP32
// master weights, activations, gradients and Adam moments.  Trained on the
// GPU by the kernels of this file, whose products run on the tensor cores
// (split-BF16 mma.sync with FP32 accumulation); evaluated per determinant by
// the Davidson's learned mode (mlp_tc.cuh).
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "pci_internal.h"
#include "mlp_tc.cuh"

namespace {

constexpr int HID = 128;
constexpr int NLAYER = 4;   // three hidden layers and the output layer
constexpr int TB = 64;      // GEMM tile (rows and columns)

// C[i][j] = sum_p A(i,p) B(p,j) on the tensor cores (mma.sync m16n8k16, BF16
// in, FP32 accumulate), A(i,p) = A[i*ars + p*acs], B(p,j) = B[p*brs + j*bcs].
// An FP32 operand is split into hi = bf16(x) and lo = bf16(x - hi) and the
// products hi*hi + hi*lo + lo*hi are summed (split-BF16: about 16 bits of
// each FP32 operand kept); a BF16 operand (the weights) is exact.  A 64 x 64
// tile per block of 4 warps (32 x 32 each), 16-deep steps through shared
// memory; the reduction is split over gridDim.z with atomic adds when split.
template <typename AT, typename BT>
__global__ void __launch_bounds__(128) k_gemm_tc(int M, int N, int K, const AT *A, int64_t ars, int64_t acs,
                                                 const BT *B, int64_t brs, int64_t bcs, float *C, int64_t ldc)
{
    __shared__ float As[16][TB + 4];
    __shared__ float Bs[16][TB + 4];
    constexpr bool ASPLIT = sizeof(AT) == 4, BSPLIT = sizeof(BT) == 4;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int wm = (w >> 1) * 32, wn = (w & 1) * 32;
    const int i0 = blockIdx.y * TB, j0 = blockIdx.x * TB;
    const int kchunk = (K + gridDim.z - 1) / gridDim.z;
    const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
    float acc[2][4][4] = {};
    for (int p0 = kbeg; p0 < kend; p0 += 16) {
        for (int e = t; e < 16 * TB; e += 128) {
            const int pp = e / TB, ii = e % TB;
            const int p = p0 + pp;
            As[pp][ii] = (i0 + ii < M && p < kend) ? (float)A[(int64_t)(i0 + ii) * ars + (int64_t)p * acs] : 0.0f;
            Bs[pp][ii] = (j0 + ii < N && p < kend) ? (float)B[(int64_t)p * brs + (int64_t)(j0 + ii) * bcs] : 0.0f;
        }
        __syncthreads();
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int r0 = wm + mt * 16 + g;
            const float v[8] = {As[2 * q][r0],     As[2 * q + 1][r0],     As[2 * q][r0 + 8],     As[2 * q + 1][r0 + 8],
                                As[2 * q + 8][r0], As[2 * q + 9][r0],     As[2 * q + 8][r0 + 8], As[2 * q + 9][r0 + 8]};
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float x0 = v[2 * u], x1 = v[2 * u + 1];
                ah[mt][u] = mlptc::pack2(x0, x1);
                if (ASPLIT) {
                    const __nv_bfloat162 hh = *reinterpret_cast<const __nv_bfloat162 *>(&ah[mt][u]);
                    al[mt][u] = mlptc::pack2(x0 - __low2float(hh), x1 - __high2float(hh));
                }
            }
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const int c0 = wn + nt * 8 + g;
            const float v[4] = {Bs[2 * q][c0], Bs[2 * q + 1][c0], Bs[2 * q + 8][c0], Bs[2 * q + 9][c0]};
            const uint32_t bh0 = mlptc::pack2(v[0], v[1]), bh1 = mlptc::pack2(v[2], v[3]);
            uint32_t bl0 = 0, bl1 = 0;
            if (BSPLIT) {
                const __nv_bfloat162 h0 = *reinterpret_cast<const __nv_bfloat162 *>(&bh0);
                const __nv_bfloat162 h1 = *reinterpret_cast<const __nv_bfloat162 *>(&bh1);
                bl0 = mlptc::pack2(v[0] - __low2float(h0), v[1] - __high2float(h0));
                bl1 = mlptc::pack2(v[2] - __low2float(h1), v[3] - __high2float(h1));
            }
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                mlptc::mma16816(acc[mt][nt], ah[mt], bh0, bh1);
                if (BSPLIT) mlptc::mma16816(acc[mt][nt], ah[mt], bl0, bl1);
                if (ASPLIT) mlptc::mma16816(acc[mt][nt], al[mt], bh0, bh1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = i0 + wm + mt * 16 + g + (u >= 2 ? 8 : 0);
                const int j = j0 + wn + nt * 8 + 2 * q + (u & 1);
                if (i < M && j < N) {
                    float *c = &C[(int64_t)i * ldc + j];
                    if (gridDim.z > 1) atomicAdd(c, acc[mt][nt][u]);
                    else *c = acc[mt][nt][u];
                }
            }
}

// Z += bias (per column), A = relu(Z) when relu
__global__ void k_bias_act(float *Z, float *A, const float *bias, int64_t n, int m, int relu)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * m; t += (int64_t)gridDim.x * blockDim.x) {
        const float z = Z[t] + bias[t % m];
        Z[t] = z;
        if (A) A[t] = relu ? fmaxf(z, 0.0f) : z;
    }
}

// dY = 2 (y - t) / n and the summed squared error
__global__ void k_mse(const float *y, const float *tgt, int64_t n, float *dy, float *loss)
{
    float s = 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = y[i] - tgt[i];
        dy[i] = 2.0f * d / (float)n;
        s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s);
}

// dZ = dA * (Z > 0)
__global__ void k_relu_back(float *dA, const float *Z, int64_t n)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        if (Z[t] <= 0.0f) dA[t] = 0.0f;
}

// db[j] = sum_i dZ[i][j]
__global__ void k_colsum(const float *dZ, int64_t n, int m, float *db)
{
    for (int j = blockIdx.x; j < m; j += gridDim.x) {
        float s = 0.0f;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += dZ[i * m + j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        __shared__ float part[32];
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = 0.0f;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
            db[j] = t;
        }
        __syncthreads();
    }
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr, float b1, float b2,
                       float c1, float c2, __nv_bfloat16 *pb)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float q = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
        p[i] = q;
        pb[i] = __float2bfloat16(q);
    }
}

// rows idx[0..b) of (X, T) into (x, t)
__global__ void k_gather(const float *X, const float *T, const int64_t *idx, int64_t b, int nin, float *x, float *t)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < b * nin; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / nin, c = e - r * nin;
        x[e] = X[idx[r] * nin + c];
        if (c == 0) t[r] = T[idx[r]];
    }
}

__global__ void k_to_bf16(const float *p, __nv_bfloat16 *pb, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16(p[i]);
}

// Tensor-core forward pass over n rows given in compact form: orbs[i][8]
// (occupied orbitals, 0xff = empty), f[i][NSCAL] (the last NSCAL inputs).
__global__ void __launch_bounds__(256) k_forward_tc(mlptc::Weights W, const uint8_t *orbs, const float *f, int64_t n,
                                                    float *y)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const mlptc::Smem S = mlptc::load(W, sm);
    const int lane = threadIdx.x & 31, g = lane >> 2;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r0 = warp * 16; r0 < n; r0 += nwarps * 16) {
        uint8_t o[2][mlptc::MAXOCC];
        float fs[2][mlptc::NSCAL], out[2];
        for (int r = 0; r < 2; r++) {
            const int64_t i = r0 + g + 8 * r;
            const bool ok = i < n;
            for (int e = 0; e < mlptc::MAXOCC; e++) o[r][e] = ok ? orbs[i * mlptc::MAXOCC + e] : 0xff;
            for (int j = 0; j < mlptc::NSCAL; j++) fs[r][j] = ok ? f[i * mlptc::NSCAL + j] : 0.f;
        }
        mlptc::tile(S, W.nin, o, fs, out);
        if ((lane & 3) == 0)
            for (int r = 0; r < 2; r++) {
                const int64_t i = r0 + g + 8 * r;
                if (i < n) y[i] = out[r];
            }
    }
}

}  // namespace

struct pci_mlp {
    int device = 0, nin = 0;
    cudaStream_t st = nullptr;
    std::string err;
    int64_t nparam = 0;
    int64_t woff[NLAYER], boff[NLAYER];
    int din[NLAYER], dout[NLAYER];
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // FP32 masters, gradients, moments
    __nv_bfloat16 *pb = nullptr;                                    // BF16 weights of the kernels
    int64_t step = 0;
    // activations of the last batch
    int64_t cap = 0;
    float *Z[NLAYER] = {}, *A[NLAYER] = {}, *dA = nullptr, *dB = nullptr, *x = nullptr, *t = nullptr, *loss = nullptr;
};

static int mlp_fail(pci_mlp *m, int code, const std::string &msg)
{
    if (m) m->err = msg;
    return code;
}

#define MLP_CUDA(m, call)                                                                       \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess) return mlp_fail((m), PCI_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

static void mlp_free_batch(pci_mlp *m)
{
    for (int l = 0; l < NLAYER; l++) { cudaFree(m->Z[l]); cudaFree(m->A[l]); m->Z[l] = m->A[l] = nullptr; }
    cudaFree(m->dA); cudaFree(m->dB); cudaFree(m->x); cudaFree(m->t); cudaFree(m->loss);
    m->dA = m->dB = m->x = m->t = m->loss = nullptr;
    m->cap = 0;
}

static int mlp_reserve(pci_mlp *m, int64_t n)
{
    if (n <= m->cap) return PCI_OK;
    mlp_free_batch(m);
    for (int l = 0; l < NLAYER; l++) {
        MLP_CUDA(m, cudaMalloc(&m->Z[l], (size_t)n * m->dout[l] * 4));
        MLP_CUDA(m, cudaMalloc(&m->A[l], (size_t)n * m->dout[l] * 4));
    }
    MLP_CUDA(m, cudaMalloc(&m->dA, (size_t)n * HID * 4));
    MLP_CUDA(m, cudaMalloc(&m->dB, (size_t)n * HID * 4));
    MLP_CUDA(m, cudaMalloc(&m->x, (size_t)n * m->nin * 4));
    MLP_CUDA(m, cudaMalloc(&m->t, (size_t)n * 4));
    MLP_CUDA(m, cudaMalloc(&m->loss, 16));
    m->cap = n;
    return PCI_OK;
}

// Activations x BF16 weights (forward, and the backward's dA = dZ W^T).
static void gemm(cudaStream_t st, int M, int N, int K, const float *A, int64_t ars, int64_t acs, const __nv_bfloat16 *B,
                 int64_t brs, int64_t bcs, float *C, int64_t ldc, int split)
{
    dim3 grid((N + TB - 1) / TB, (M + TB - 1) / TB, split);
    k_gemm_tc<float, __nv_bfloat16><<<grid, 128, 0, st>>>(M, N, K, A, ars, acs, B, brs, bcs, C, ldc);
}

// FP32 x FP32 (the weight gradients in^T dZ), both operands split.
static void gemm_f(cudaStream_t st, int M, int N, int K, const float *A, int64_t ars, int64_t acs, const float *B,
                   int64_t brs, int64_t bcs, float *C, int64_t ldc, int split)
{
    dim3 grid((N + TB - 1) / TB, (M + TB - 1) / TB, split);
    k_gemm_tc<float, float><<<grid, 128, 0, st>>>(M, N, K, A, ars, acs, B, brs, bcs, C, ldc);
}

// Forward pass over n rows of m->x; output (pre-activation of the last
// layer) in m->Z[NLAYER-1].
static int mlp_forward_dev(pci_mlp *m, int64_t n)
{
    const float *in = m->x;
    int64_t ldin = m->nin;
    for (int l = 0; l < NLAYER; l++) {
        const int K = m->din[l], N = m->dout[l];
        gemm(m->st, (int)n, N, K, in, ldin, 1, m->pb + m->woff[l], N, 1, m->Z[l], N, 1);
        k_bias_act<<<148 * 4, 256, 0, m->st>>>(m->Z[l], m->A[l], m->p + m->boff[l], n, N, l < NLAYER - 1);
        in = m->A[l];
        ldin = N;
    }
    MLP_CUDA(m, cudaGetLastError());
    return PCI_OK;
}

// Loss and gradients (into m->g) of the batch in m->x, m->t.
static int mlp_backward_dev(pci_mlp *m, int64_t n, float *loss_host)
{
    MLP_CUDA(m, cudaMemsetAsync(m->loss, 0, 4, m->st));
    MLP_CUDA(m, cudaMemsetAsync(m->g, 0, (size_t)m->nparam * 4, m->st));
    k_mse<<<148 * 4, 256, 0, m->st>>>(m->A[NLAYER - 1], m->t, n, m->dA, m->loss);
    float *dZ = m->dA, *dnext = m->dB;
    const int split = (int)std::min<int64_t>(148, std::max<int64_t>(1, n / 256));
    for (int l = NLAYER - 1; l >= 0; l--) {
        const int K = m->din[l], N = m->dout[l];
        const float *in = l ? m->A[l - 1] : m->x;
        // dW = in^T dZ   (K x N), reduction over the batch
        gemm_f(m->st, K, N, (int)n, in, 1, K, dZ, N, 1, m->g + m->woff[l], N, split);
        k_colsum<<<std::min(N, 148 * 4), 256, 0, m->st>>>(dZ, n, N, m->g + m->boff[l]);
        if (l > 0) {
            // dA_prev = dZ W^T (n x K), then through the ReLU
            gemm(m->st, (int)n, K, N, dZ, N, 1, m->pb + m->woff[l], 1, N, dnext, K, 1);
            k_relu_back<<<148 * 4, 256, 0, m->st>>>(dnext, m->Z[l - 1], n * K);
            std::swap(dZ, dnext);
        }
    }
    MLP_CUDA(m, cudaGetLastError());
    if (loss_host) {
        float s = 0.0f;
        MLP_CUDA(m, cudaMemcpyAsync(&s, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
        MLP_CUDA(m, cudaStreamSynchronize(m->st));
        *loss_host = s / (float)n;
    }
    return PCI_OK;
}

extern "C" {

int pci_mlp_create(int32_t device, int32_t nin, int32_t seed, pci_mlp_t **out)
{
    if (!out) return PCI_E_INPUT;
    *out = nullptr;
    if (nin < 1 || nin > 1024) return PCI_E_INPUT;
    if (cudaSetDevice(device) != cudaSuccess) return PCI_E_CUDA;
    pci_mlp *m = new pci_mlp();
    m->device = device;
    m->nin = nin;
    const int dims[NLAYER + 1] = {nin, HID, HID, HID, 1};
    int64_t off = 0;
    for (int l = 0; l < NLAYER; l++) {
        m->din[l] = dims[l];
        m->dout[l] = dims[l + 1];
        m->woff[l] = off;
        off += (int64_t)dims[l] * dims[l + 1];
        m->boff[l] = off;
        off += dims[l + 1];
    }
    m->nparam = off;
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&m->p, off * 4) != cudaSuccess || cudaMalloc(&m->g, off * 4) != cudaSuccess ||
        cudaMalloc(&m->m, off * 4) != cudaSuccess || cudaMalloc(&m->v, off * 4) != cudaSuccess ||
        cudaMalloc(&m->pb, off * 2) != cudaSuccess) {
        pci_mlp_destroy(m);
        return PCI_E_OOM;
    }
    // He-style initial weights from a seeded generator, zero biases
    std::vector<float> h(off, 0.0f);
    uint64_t s = 0x9E3779B97F4A7C15ULL ^ (uint64_t)seed;
    for (int l = 0; l < NLAYER; l++) {
        const float sc = sqrtf(2.0f / (float)m->din[l]) * (l == NLAYER - 1 ? 0.1f : 1.0f);
        for (int64_t i = 0; i < (int64_t)m->din[l] * m->dout[l]; i++) {
            float u = 0.0f;
            for (int r = 0; r < 4; r++) {   // sum of uniforms, variance 1/3 each
                s ^= s << 13; s ^= s >> 7; s ^= s << 17;
                u += (float)((s >> 11) * (1.0 / 9007199254740992.0)) - 0.5f;
            }
            h[m->woff[l] + i] = u * sc * sqrtf(3.0f);
        }
    }
    if (pci_mlp_set_params(m, h.data(), off) != PCI_OK) {
        pci_mlp_destroy(m);
        return PCI_E_CUDA;
    }
    *out = m;
    return PCI_OK;
}

int64_t pci_mlp_num_params(pci_mlp_t *m)
{
    return m ? m->nparam : -1;
}

int pci_mlp_set_params(pci_mlp_t *m, const float *p, int64_t n)
{
    if (!m || !p || n != m->nparam) return mlp_fail(m, PCI_E_INPUT, "set_params: wrong parameter count");
    cudaSetDevice(m->device);
    MLP_CUDA(m, cudaMemcpyAsync(m->p, p, n * 4, cudaMemcpyHostToDevice, m->st));
    MLP_CUDA(m, cudaMemsetAsync(m->m, 0, n * 4, m->st));
    MLP_CUDA(m, cudaMemsetAsync(m->v, 0, n * 4, m->st));
    k_to_bf16<<<148 * 4, 256, 0, m->st>>>(m->p, m->pb, n);
    MLP_CUDA(m, cudaStreamSynchronize(m->st));
    m->step = 0;
    return PCI_OK;
}

int pci_mlp_get_params(pci_mlp_t *m, float *p, int64_t n)
{
    if (!m || !p || n != m->nparam) return mlp_fail(m, PCI_E_INPUT, "get_params: wrong parameter count");
    cudaSetDevice(m->device);
    MLP_CUDA(m, cudaMemcpyAsync(p, m->p, n * 4, cudaMemcpyDeviceToHost, m->st));
    MLP_CUDA(m, cudaStreamSynchronize(m->st));
    return PCI_OK;
}

int pci_mlp_forward(pci_mlp_t *m, const float *X, int64_t n, float *y)
{
    if (!m || !X || !y || n < 1) return mlp_fail(m, PCI_E_INPUT, "forward: bad arguments");
    cudaSetDevice(m->device);
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    MLP_CUDA(m, cudaMemcpyAsync(m->x, X, (size_t)n * m->nin * 4, cudaMemcpyHostToDevice, m->st));
    if ((rc = mlp_forward_dev(m, n))) return rc;
    MLP_CUDA(m, cudaMemcpyAsync(y, m->A[NLAYER - 1], (size_t)n * 4, cudaMemcpyDeviceToHost, m->st));
    MLP_CUDA(m, cudaStreamSynchronize(m->st));
    return PCI_OK;
}

int pci_mlp_loss_grad(pci_mlp_t *m, const float *X, const float *T, int64_t n, float *loss, float *grad)
{
    if (!m || !X || !T || n < 1) return mlp_fail(m, PCI_E_INPUT, "loss_grad: bad arguments");
    cudaSetDevice(m->device);
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    MLP_CUDA(m, cudaMemcpyAsync(m->x, X, (size_t)n * m->nin * 4, cudaMemcpyHostToDevice, m->st));
    MLP_CUDA(m, cudaMemcpyAsync(m->t, T, (size_t)n * 4, cudaMemcpyHostToDevice, m->st));
    if ((rc = mlp_forward_dev(m, n))) return rc;
    if ((rc = mlp_backward_dev(m, n, loss))) return rc;
    if (grad) {
        MLP_CUDA(m, cudaMemcpyAsync(grad, m->g, m->nparam * 4, cudaMemcpyDeviceToHost, m->st));
        MLP_CUDA(m, cudaStreamSynchronize(m->st));
    }
    return PCI_OK;
}

int pci_mlp_train(pci_mlp_t *m, const float *X, const float *T, int64_t n, int32_t epochs, int32_t batch, float lr,
                  int32_t seed, float *loss_out)
{
    if (!m || !X || !T || n < 1 || epochs < 1 || batch < 1) return mlp_fail(m, PCI_E_INPUT, "train: bad arguments");
    cudaSetDevice(m->device);
    const int64_t b = std::min<int64_t>(batch, n);
    int rc = mlp_reserve(m, b);
    if (rc) return rc;
    // whole set on the device, batches gathered by a host-side shuffle
    float *dX = nullptr, *dT = nullptr;
    int64_t *dOrd = nullptr;
    MLP_CUDA(m, cudaMalloc(&dX, (size_t)n * m->nin * 4));
    MLP_CUDA(m, cudaMalloc(&dT, (size_t)n * 4));
    MLP_CUDA(m, cudaMalloc(&dOrd, (size_t)n * 8));
    MLP_CUDA(m, cudaMemcpyAsync(dX, X, (size_t)n * m->nin * 4, cudaMemcpyHostToDevice, m->st));
    MLP_CUDA(m, cudaMemcpyAsync(dT, T, (size_t)n * 4, cudaMemcpyHostToDevice, m->st));
    std::vector<int64_t> order(n);
    for (int64_t i = 0; i < n; i++) order[i] = i;
    uint64_t s = 0xD1B54A32D192ED03ULL ^ (uint64_t)seed;
    float last = 0.0f;
    for (int e = 0; e < epochs; e++) {
        for (int64_t i = n - 1; i > 0; i--) {
            s ^= s << 13; s ^= s >> 7; s ^= s << 17;
            std::swap(order[i], order[s % (uint64_t)(i + 1)]);
        }
        MLP_CUDA(m, cudaMemcpyAsync(dOrd, order.data(), (size_t)n * 8, cudaMemcpyHostToDevice, m->st));
        double esum = 0.0;
        int64_t eb = 0;
        for (int64_t b0 = 0; b0 + b <= n; b0 += b) {
            k_gather<<<148 * 4, 256, 0, m->st>>>(dX, dT, dOrd + b0, b, m->nin, m->x, m->t);
            if ((rc = mlp_forward_dev(m, b))) break;
            float l = 0.0f;
            if ((rc = mlp_backward_dev(m, b, &l))) break;
            m->step++;
            const float b1 = 0.9f, b2 = 0.999f;
            k_adam<<<148 * 4, 256, 0, m->st>>>(m->p, m->g, m->m, m->v, m->nparam, lr, b1, b2,
                                               1.0f - powf(b1, (float)m->step), 1.0f - powf(b2, (float)m->step), m->pb);
            esum += l;
            eb++;
        }
        if (rc) break;
        last = eb ? (float)(esum / eb) : 0.0f;
    }
    cudaStreamSynchronize(m->st);
    cudaFree(dX);
    cudaFree(dT);
    cudaFree(dOrd);
    if (rc) return rc;
    MLP_CUDA(m, cudaStreamSynchronize(m->st));
    if (loss_out) *loss_out = last;
    return PCI_OK;
}

const char *pci_mlp_last_error(pci_mlp_t *m)
{
    return m ? m->err.c_str() : "null model";
}

void pci_mlp_destroy(pci_mlp_t *m)
{
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->st) cudaStreamSynchronize(m->st);
    mlp_free_batch(m);
    cudaFree(m->p); cudaFree(m->g); cudaFree(m->m); cudaFree(m->v); cudaFree(m->pb);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
}

}  // extern "C"

// Forward pass for the Davidson (device features in, device output); the
// batch buffers of the model are reused.
int mlp_forward_device(pci_mlp *m, const float *dX, int64_t n, float *dy, cudaStream_t st)
{
    cudaSetDevice(m->device);
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    MLP_CUDA(m, cudaStreamSynchronize(st));
    MLP_CUDA(m, cudaMemcpyAsync(m->x, dX, (size_t)n * m->nin * 4, cudaMemcpyDeviceToDevice, m->st));
    if ((rc = mlp_forward_dev(m, n))) return rc;
    MLP_CUDA(m, cudaMemcpyAsync(dy, m->A[NLAYER - 1], (size_t)n * 4, cudaMemcpyDeviceToDevice, m->st));
    MLP_CUDA(m, cudaStreamSynchronize(m->st));
    return PCI_OK;
}

int mlp_num_inputs(const pci_mlp *m)
{
    return m->nin;
}

mlptc::Weights mlp_tc_weights(const pci_mlp *m)
{
    mlptc::Weights W;
    W.pb = m->pb;
    W.p = m->p;
    W.nin = m->nin;
    for (int l = 0; l < NLAYER; l++) {
        W.woff[l] = m->woff[l];
        W.boff[l] = m->boff[l];
    }
    return W;
}

extern "C" int pci_mlp_forward_occ(pci_mlp_t *m, const uint8_t *orbs, const float *f, int64_t n, float *y)
{
    if (!m || !orbs || !f || !y || n < 1) return mlp_fail(m, PCI_E_INPUT, "forward_occ: bad arguments");
    if (m->nin < mlptc::NSCAL + 1) return mlp_fail(m, PCI_E_INPUT, "forward_occ: the model needs nin >= 4");
    cudaSetDevice(m->device);
    uint8_t *d_o = nullptr;
    float *d_f = nullptr, *d_y = nullptr;
    int rc = PCI_OK;
    const size_t sb = mlptc::smem_bytes(m->nin);
    if (cudaMalloc(&d_o, (size_t)n * mlptc::MAXOCC) != cudaSuccess ||
        cudaMalloc(&d_f, (size_t)n * mlptc::NSCAL * 4) != cudaSuccess || cudaMalloc(&d_y, (size_t)n * 4) != cudaSuccess) {
        rc = mlp_fail(m, PCI_E_OOM, "forward_occ: device allocation failed");
    } else if (cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb) != cudaSuccess) {
        rc = mlp_fail(m, PCI_E_CUDA, "forward_occ: shared memory attribute");
    } else {
        cudaMemcpyAsync(d_o, orbs, (size_t)n * mlptc::MAXOCC, cudaMemcpyHostToDevice, m->st);
        cudaMemcpyAsync(d_f, f, (size_t)n * mlptc::NSCAL * 4, cudaMemcpyHostToDevice, m->st);
        k_forward_tc<<<148, 256, sb, m->st>>>(mlp_tc_weights(m), d_o, d_f, n, d_y);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(y, d_y, (size_t)n * 4, cudaMemcpyDeviceToHost, m->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(m->st);
        if (e != cudaSuccess) rc = mlp_fail(m, PCI_E_CUDA, std::string("forward_occ: ") + cudaGetErrorString(e));
    }
    cudaFree(d_o);
    cudaFree(d_f);
    cudaFree(d_y);
    return rc;
}
