// gemm_bf16.cuh -- batched matrix product on the BF16 tensor cores with FP32
// accumulation, for the Fourier neural operator (csrc/fno.cu).
//
// C[m][n] = alpha * sum_k A[m][k] B[k][n] (+ beta C) (+ bias[n]), optionally
// with a second output gelu(C), over a batch of independent products.  Every
// index of every operand goes through a two-level map i -> (i / g) s1 +
// (i % g) s0, so one interface serves transposed operands and the layouts of
// the FNO's truncated transforms, whose real/imaginary index sits above the
// transformed axis.  A and B are read as FP32 or BF16 and rounded to BF16;
// products accumulate in FP32 (mma.sync m16n8k16).  gemm() picks one of three
// kernels by the product's shape (gemm_bf16.cu).  With ksplit > 1 the K range
// is split over blocks that add into C atomically (beta must then be 1, no
// bias, no second output).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace ehd {
namespace fno {

// GELU (erf form) and its derivative, shared by the products' epilogues and
// the FNO's elementwise kernels
__device__ __forceinline__ float gelu(float v) {
    return 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float phi = 0.3989422804014327f * expf(-0.5f * z * z);
    const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
    return cdf + z * phi;
}

struct Map {
    long long s0 = 1, s1 = 0;
    int g = 1 << 30;
};
__host__ __device__ __forceinline__ long long at(const Map &d, long long i) {
    if (d.g == (1 << 30)) return i * d.s0;  // one level: no division
    return (i / d.g) * d.s1 + (i % d.g) * d.s0;
}
// the same for a non-negative int index, in the offset type Off (int where
// every offset of the product fits, else long long); 32-bit division
template <typename Off>
__host__ __device__ __forceinline__ Off at_off(const Map &d, int i) {
    if (d.g == (1 << 30)) return (Off)i * (Off)d.s0;
    const unsigned q = (unsigned)i / (unsigned)d.g, r = (unsigned)i - q * (unsigned)d.g;
    return (Off)q * (Off)d.s1 + (Off)r * (Off)d.s0;
}
inline Map lin(long long s0) { return Map{s0, 0, 1 << 30}; }
inline Map two(long long s0, int g, long long s1) { return Map{s0, s1, g}; }

struct GemmArgs {
    int M = 0, N = 0, K = 0, batch = 1, ksplit = 1;
    const void *A = nullptr;
    Map am, ak, abat;
    int a_bf16 = 0;
    const void *B = nullptr;
    Map bk, bn, bbat;
    int b_bf16 = 0;
    float *C = nullptr;
    Map cm, cn, cbat;
    float alpha = 1.f, beta = 0.f;
    const float *bias = nullptr;  // per column n
    float *C2 = nullptr;          // gelu(C), same indexing
    // elements in the A, B and C (and C2) buffers: gemm() rejects a product
    // whose largest offset falls outside them
    long long a_n = 0, b_n = 0, c_n = 0;
    // set by gemm(): which index of A (m) and B (n) the lanes of a warp run
    // along when staging a tile (the one with unit stride)
    int a_rows_fast = 0, b_rows_fast = 0;
};

cudaError_t gemm(const GemmArgs &a, cudaStream_t s);

// G[m][n] += sum_r X[r][m] D[r][n] (BF16 products, FP32 sums) and, unless gb
// is null, gb[n] += sum_r D[r][n] (FP32), over r < rows: the weight and bias
// gradients of a pointwise layer in one pass.  M <= 128; X rows ldx apart,
// D rows ldd apart, G rows ldg apart.
cudaError_t weight_bias_grad(long long rows, int M, int N, const float *X, int ldx, const float *D,
                             int ldd, float *G, int ldg, float *gb, cudaStream_t s);

}  // namespace fno
}  // namespace ehd
