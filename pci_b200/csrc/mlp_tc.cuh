// Tensor-core evaluation of the correction MLP (nin -> 128 -> 128 -> 128 -> 1,
// ReLU) for 16 rows per warp.
//
// The first layer's input is sparse: the occupation counts of the orbitals
// (at most PCI_NE_MAX non-zero entries per determinant) and NSCAL scalars, so it
// is evaluated as a sum of rows of W1 on the CUDA cores.  The two 128 x 128
// hidden layers run as mma.sync m16n8k16 BF16 products with FP32 accumulation:
// a layer's accumulator fragments are, after bias and ReLU, exactly the next
// layer's A fragments, so activations never leave registers.  The output
// layer is a dot product reduced across the four lanes of a row group.
//
// Weights are the model's BF16 copies (the ones its training forward pass
// reads); biases are its FP32 masters.  The hidden activations are rounded to
// BF16 for the tensor-core products (the training forward keeps them in
// FP32), so outputs agree with pci_mlp_forward to about 1e-2 relative.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace mlptc {

constexpr int HID = 128;
constexpr int WPAD = HID + 8;   // row stride (bf16) of the transposed hidden weights in shared memory
constexpr int MAXOCC = 8;       // orbital slots per determinant (PCI_NE_MAX)
constexpr int NSCAL = 3;        // scalar inputs after the occupation counts

// Where the parameters live (device pointers into the model, layer by layer:
// W (din x dout, row-major) then b (dout)).
struct Weights {
    const __nv_bfloat16 *pb;
    const float *p;
    int nin;
    int64_t woff[4], boff[4];
};

struct Smem {
    const __nv_bfloat16 *w1;    // [nin][HID]
    const __nv_bfloat16 *w2t;   // [HID][WPAD]: w2t[n][k] = W2[k][n]
    const __nv_bfloat16 *w3t;
    const float *b1, *b2, *b3, *w4;
    float b4;
};

__host__ __device__ inline size_t smem_bytes(int nin)
{
    return (size_t)nin * HID * 2 + 2 * (size_t)HID * WPAD * 2 + 4 * HID * 4 + 16;
}

// Copy the parameters into shared memory (every thread of the block takes
// part; ends with a barrier).
__device__ inline Smem load(const Weights &W, unsigned char *raw)
{
    __nv_bfloat16 *w1 = (__nv_bfloat16 *)raw;
    __nv_bfloat16 *w2t = w1 + (size_t)W.nin * HID;
    __nv_bfloat16 *w3t = w2t + (size_t)HID * WPAD;
    float *b1 = (float *)(w3t + (size_t)HID * WPAD);
    float *b2 = b1 + HID, *b3 = b2 + HID, *w4 = b3 + HID;
    for (int i = threadIdx.x; i < W.nin * HID; i += blockDim.x) w1[i] = W.pb[W.woff[0] + i];
    for (int i = threadIdx.x; i < HID * HID; i += blockDim.x) {
        const int k = i / HID, n = i % HID;
        w2t[n * WPAD + k] = W.pb[W.woff[1] + i];
        w3t[n * WPAD + k] = W.pb[W.woff[2] + i];
    }
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        b1[i] = W.p[W.boff[0] + i];
        b2[i] = W.p[W.boff[1] + i];
        b3[i] = W.p[W.boff[2] + i];
        w4[i] = __bfloat162float(W.pb[W.woff[3] + i]);
    }
    __syncthreads();
    Smem S;
    S.w1 = w1;
    S.w2t = w2t;
    S.w3t = w3t;
    S.b1 = b1;
    S.b2 = b2;
    S.b3 = b3;
    S.w4 = w4;
    S.b4 = W.p[W.boff[3]];
    return S;
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Accumulator fragments C[16 n-tiles] (after bias and ReLU) -> A fragments of
// the next layer's 8 k-tiles.
__device__ __forceinline__ void c_to_a(const float (&C)[16][4], uint32_t (&A)[8][4])
{
#pragma unroll
    for (int kk = 0; kk < 8; kk++) {
        A[kk][0] = pack2(C[2 * kk][0], C[2 * kk][1]);
        A[kk][1] = pack2(C[2 * kk][2], C[2 * kk][3]);
        A[kk][2] = pack2(C[2 * kk + 1][0], C[2 * kk + 1][1]);
        A[kk][3] = pack2(C[2 * kk + 1][2], C[2 * kk + 1][3]);
    }
}

// One hidden layer: C = relu(A Wt^T + b).
__device__ __forceinline__ void hidden(const uint32_t (&A)[8][4], const __nv_bfloat16 *wt, const float *b,
                                       float (&C)[16][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        C[j][0] = C[j][1] = C[j][2] = C[j][3] = 0.f;
        const __nv_bfloat16 *row = wt + (size_t)(8 * j + g) * WPAD + 2 * t;
#pragma unroll
        for (int kk = 0; kk < 8; kk++) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t *>(row + 16 * kk);
            const uint32_t b1 = *reinterpret_cast<const uint32_t *>(row + 16 * kk + 8);
            mma16816(C[j], A[kk], b0, b1);
        }
        const float bb0 = b[8 * j + 2 * t], bb1 = b[8 * j + 2 * t + 1];
        C[j][0] = fmaxf(C[j][0] + bb0, 0.f);
        C[j][1] = fmaxf(C[j][1] + bb1, 0.f);
        C[j][2] = fmaxf(C[j][2] + bb0, 0.f);
        C[j][3] = fmaxf(C[j][3] + bb1, 0.f);
    }
}

// MLP output for the 16 rows of a warp.  Lane (g = lane / 4, t = lane % 4)
// supplies rows g (index 0) and g + 8 (index 1): up to MAXOCC orbital indices
// each (entries >= nin - NSCAL ignored, so 0xff marks an empty slot; an
// orbital listed twice counts twice) and the scalar inputs f[r][j] (input
// nin - NSCAL + j).  All 32 lanes must call it; out[i] receives row i's
// output (replicated over the four lanes of the group).
__device__ inline void tile(const Smem &S, int nin, const uint8_t (&orb)[2][MAXOCC], const float (&f)[2][NSCAL],
                            float (&out)[2])
{
    const int lane = threadIdx.x & 31, t = lane & 3;
    float C[16][4];
    // layer 1: bias + the W1 rows of the occupied orbitals + the scalar inputs
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const int col = 8 * j + 2 * t;
        C[j][0] = C[j][2] = S.b1[col];
        C[j][1] = C[j][3] = S.b1[col + 1];
    }
#pragma unroll
    for (int r = 0; r < 2; r++) {
        for (int e = 0; e < MAXOCC + NSCAL; e++) {
            int wrow;
            float fe;
            if (e < MAXOCC) {
                wrow = orb[r][e];
                fe = 1.f;
                if (wrow >= nin - NSCAL) continue;
            } else {
                wrow = nin - NSCAL + (e - MAXOCC);
                fe = f[r][e - MAXOCC];
            }
            const __nv_bfloat16 *w = S.w1 + (size_t)wrow * HID + 2 * t;
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(w + 8 * j);
                C[j][2 * r] += fe * __low2float(v);
                C[j][2 * r + 1] += fe * __high2float(v);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 16; j++)
#pragma unroll
        for (int q = 0; q < 4; q++) C[j][q] = fmaxf(C[j][q], 0.f);
    uint32_t A[8][4];
    c_to_a(C, A);
    hidden(A, S.w2t, S.b2, C);
    c_to_a(C, A);
    hidden(A, S.w3t, S.b3, C);
    float o0 = 0.f, o1 = 0.f;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const float w0 = S.w4[8 * j + 2 * t], w1 = S.w4[8 * j + 2 * t + 1];
        o0 += w0 * C[j][0] + w1 * C[j][1];
        o1 += w0 * C[j][2] + w1 * C[j][3];
    }
    o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
    o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
    out[0] = o0 + S.b4;
    out[1] = o1 + S.b4;
}

}  // namespace mlptc
