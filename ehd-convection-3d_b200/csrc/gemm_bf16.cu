// gemm_bf16.cu -- the batched BF16 tensor-core product of gemm_bf16.cuh.
//
// 64 x 64 output tiles, K in steps of 32, 128 threads: each warp owns a
// 32 x 32 quarter as 2 x 4 tiles of mma.sync.m16n8k16 (BF16 in, FP32 out).
// Operands are staged in shared memory as BF16, A as [m][k] and B as [n][k],
// so that every fragment register is one aligned 32-bit load of two
// consecutive k.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "gemm_bf16.cuh"

namespace ehd {
namespace fno {

namespace {

constexpr int BM = 64, BN = 64, BK = 32, PK = BK + 8;

__device__ __forceinline__ __nv_bfloat16 load_bf16(const void *p, long long off, int is_bf16) {
    return is_bf16 ? reinterpret_cast<const __nv_bfloat16 *>(p)[off]
                   : __float2bfloat16_rn(reinterpret_cast<const float *>(p)[off]);
}

__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float gelu(float v) {
    return 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
}

__global__ void __launch_bounds__(128) gemm_kernel(const GemmArgs a) {
    __shared__ __align__(16) __nv_bfloat16 As[BM][PK];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][PK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int gq = lane >> 2, tq = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int bidx = blockIdx.z / a.ksplit, split = blockIdx.z % a.ksplit;
    const long long aoff = at(a.abat, bidx), boff = at(a.bbat, bidx), coff = at(a.cbat, bidx);
    const int kper = ((a.K + a.ksplit - 1) / a.ksplit + BK - 1) / BK * BK;
    const int kbeg = split * kper;
    const int kend = min(a.K, kbeg + kper);

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    for (int k0 = kbeg; k0 < kend; k0 += BK) {
#pragma unroll 4
        for (int r = 0; r < (BM * BK) / 128; ++r) {
            const int i = tid + 128 * r;
            const int mm = i / BK, kk = i % BK;
            const int m = m0 + mm, k = k0 + kk;
            As[mm][kk] = (m < a.M && k < kend)
                             ? load_bf16(a.A, aoff + at(a.am, m) + at(a.ak, k), a.a_bf16)
                             : __float2bfloat16_rn(0.f);
        }
#pragma unroll 4
        for (int r = 0; r < (BN * BK) / 128; ++r) {
            const int i = tid + 128 * r;
            const int nn = i / BK, kk = i % BK;
            const int n = n0 + nn, k = k0 + kk;
            Bs[nn][kk] = (n < a.N && k < kend)
                             ? load_bf16(a.B, boff + at(a.bk, k) + at(a.bn, n), a.b_bf16)
                             : __float2bfloat16_rn(0.f);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm * 32 + i * 16 + gq;
                af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][kk + tq * 2]);
                af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + tq * 2]);
                af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][kk + tq * 2 + 8]);
                af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + tq * 2 + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn * 32 + j * 8 + gq;
                bf[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + tq * 2]);
                bf[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + tq * 2 + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mma16816(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bf[j][0],
                             bf[j][1]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int m = m0 + wm * 32 + i * 16 + gq + (e >> 1) * 8;
                const int n = n0 + wn * 32 + j * 8 + tq * 2 + (e & 1);
                if (m >= a.M || n >= a.N) continue;
                const long long off = coff + at(a.cm, m) + at(a.cn, n);
                float v = a.alpha * acc[i][j][e];
                if (a.ksplit > 1) {
                    atomicAdd(a.C + off, v);
                    continue;
                }
                if (a.beta != 0.f) v += a.beta * a.C[off];
                if (a.bias) v += a.bias[n];
                a.C[off] = v;
                if (a.C2) a.C2[off] = gelu(v);
            }
}

}  // namespace

namespace {

// largest offset of the map over i = 0 .. n-1 (strides >= 0)
long long max_at(const Map &d, long long n) {
    if (n <= 0) return 0;
    const long long q = (n - 1) / d.g, r = (n - 1) % d.g;
    long long m = q * d.s1 + r * d.s0;
    if (q >= 1) m = std::max(m, (q - 1) * d.s1 + (long long)(d.g - 1) * d.s0);
    return m;
}

bool nonneg(const Map &d) { return d.s0 >= 0 && d.s1 >= 0 && d.g >= 1; }

}  // namespace

cudaError_t gemm(const GemmArgs &a, cudaStream_t s) {
    if (a.M <= 0 || a.N <= 0 || a.K <= 0 || a.batch <= 0) return cudaSuccess;
    // every access in bounds: largest offset of each operand below its size
    const Map *maps[] = {&a.am, &a.ak, &a.abat, &a.bk, &a.bn, &a.bbat, &a.cm, &a.cn, &a.cbat};
    for (const Map *m : maps)
        if (!nonneg(*m)) return cudaErrorInvalidValue;
    if (max_at(a.abat, a.batch) + max_at(a.am, a.M) + max_at(a.ak, a.K) >= a.a_n ||
        max_at(a.bbat, a.batch) + max_at(a.bk, a.K) + max_at(a.bn, a.N) >= a.b_n ||
        max_at(a.cbat, a.batch) + max_at(a.cm, a.M) + max_at(a.cn, a.N) >= a.c_n)
        return cudaErrorInvalidValue;
    if (a.ksplit < 1 || (a.ksplit > 1 && (a.beta != 1.f || a.bias || a.C2)))
        return cudaErrorInvalidValue;
    const long long gy = (a.M + BM - 1) / BM, gz = (long long)a.batch * a.ksplit;
    if (gy > 65535 || gz > 65535) return cudaErrorInvalidValue;
    dim3 grid((a.N + BN - 1) / BN, (unsigned)gy, (unsigned)gz);
    gemm_kernel<<<grid, 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace fno
}  // namespace ehd
