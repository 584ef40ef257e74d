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
#include <utility>

#include "gemm_bf16.cuh"

namespace ehd {
namespace fno {

namespace {

constexpr int BM = 64, BN = 64, BK = 32, PK = BK + 8;

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

// Raw bits of one operand element: the FP32 value, or the BF16 value in the
// low half.
template <int BF>
__device__ __forceinline__ uint32_t ld_raw(const void *p, long long off) {
    return BF ? (uint32_t)__ldg(reinterpret_cast<const unsigned short *>(p) + off)
                   : __float_as_uint(__ldg(reinterpret_cast<const float *>(p) + off));
}
template <int BF>
__device__ __forceinline__ __nv_bfloat16 to_bf16(uint32_t raw) {
    return BF ? __ushort_as_bfloat16((unsigned short)raw)
                   : __float2bfloat16_rn(__uint_as_float(raw));
}

// One operand's share of a 64-row x 32-k tile.  Lanes run along whichever
// index has unit stride in memory, so a warp reads 32 consecutive elements:
//  - along k (rows_fast = 0): k = k0 + lane, rows warp + 4 r (r < 16); the
//    16 row offsets ro[r] are fixed for the block, one k offset per K step;
//  - along rows (rows_fast = 1): row tid % 64 (offset ro[0]), k = k0 + tid / 64
//    + 2 r; 16 k offsets per K step.
// Elements outside the product (row >= rows or k >= kend) read as zero.  BF:
// the operand is BF16 (else FP32); RF: rows_fast.
template <typename Off, int BF, int RF>
__device__ __forceinline__ void load_tile(uint32_t (&raw)[16], const void *P,
                                          const Off (&ro)[16], unsigned mask, const Map &km,
                                          int k0, int kend, int tid) {
    if (!RF) {
        const int k = k0 + (tid & 31);
        const bool kin = k < kend;
        const Off ko = kin ? at_off<Off>(km, k) : (Off)0;
        const unsigned m = kin ? mask : 0u;
#pragma unroll
        for (int r = 0; r < 16; ++r) raw[r] = (m >> r & 1u) ? ld_raw<BF>(P, ro[r] + ko) : 0u;
    } else {
        const int kb = k0 + (tid >> 6);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int k = kb + 2 * r;
            raw[r] = ((mask & 1u) && k < kend) ? ld_raw<BF>(P, ro[0] + at_off<Off>(km, k)) : 0u;
        }
    }
}

template <int BF, int RF>
__device__ __forceinline__ void store_tile(__nv_bfloat16 (*S)[PK], const uint32_t (&raw)[16],
                                           int tid) {
    if (!RF) {
#pragma unroll
        for (int r = 0; r < 16; ++r) S[(tid >> 5) + 4 * r][tid & 31] = to_bf16<BF>(raw[r]);
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) S[tid & 63][(tid >> 6) + 2 * r] = to_bf16<BF>(raw[r]);
    }
}

// row offsets of one operand's tile rows for this thread (see load_tile)
template <typename Off, int RF>
__device__ __forceinline__ void row_offsets(Off (&ro)[16], unsigned &mask, const Map &rm,
                                            Off base, int r0, int rows, int tid) {
    mask = 0;
    if (!RF) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int i = r0 + (tid >> 5) + 4 * r;
            ro[r] = base + (i < rows ? at_off<Off>(rm, i) : (Off)0);
            mask |= (i < rows ? 1u : 0u) << r;
        }
    } else {
        const int i = r0 + (tid & 63);
#pragma unroll
        for (int r = 0; r < 16; ++r) ro[r] = base;
        if (i < rows) {
            ro[0] = base + at_off<Off>(rm, i);
            mask = 1u;
        }
    }
}

// The next K step's operands are loaded into registers while the tensor
// cores work on the current one.  Off is int where every offset of the
// product fits in 31 bits, else long long.  The operand types (ABF, BBF) and
// staging directions (AR, BR) are compile-time, so each instance is
// straight-line code: with them as run-time switches the kernel stalled on
// instruction fetch.
template <typename Off, int ABF, int AR, int BBF, int BR>
__global__ void __launch_bounds__(128, 4) gemm_kernel(const GemmArgs a) {
    __shared__ __align__(16) __nv_bfloat16 As[BM][PK];
    __shared__ __align__(16) __nv_bfloat16 Bs[BN][PK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int gq = lane >> 2, tq = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int bidx = blockIdx.z / a.ksplit, split = blockIdx.z % a.ksplit;
    const int kper = ((a.K + a.ksplit - 1) / a.ksplit + BK - 1) / BK * BK;
    const int kbeg = split * kper;
    const int kend = min(a.K, kbeg + kper);

    Off aro[16], bro[16];
    unsigned amask, bmask;
    row_offsets<Off, AR>(aro, amask, a.am, at_off<Off>(a.abat, bidx), m0, a.M, tid);
    row_offsets<Off, BR>(bro, bmask, a.bn, at_off<Off>(a.bbat, bidx), n0, a.N, tid);

    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    uint32_t ra[16], rb[16];
    if (kbeg < kend) {
        load_tile<Off, ABF, AR>(ra, a.A, aro, amask, a.ak, kbeg, kend, tid);
        load_tile<Off, BBF, BR>(rb, a.B, bro, bmask, a.bk, kbeg, kend, tid);
    }
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        store_tile<ABF, AR>(As, ra, tid);
        store_tile<BBF, BR>(Bs, rb, tid);
        __syncthreads();
        if (k0 + BK < kend) {
            load_tile<Off, ABF, AR>(ra, a.A, aro, amask, a.ak, k0 + BK, kend, tid);
            load_tile<Off, BBF, BR>(rb, a.B, bro, bmask, a.bk, k0 + BK, kend, tid);
        }
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

    // epilogue: rows m0 + wm 32 + i 16 + gq + h 8, columns n0 + wn 32 + j 8 + 2 tq + c
    const Off coff = at_off<Off>(a.cbat, bidx);
    Off cmo[4], cno[8];
    unsigned cmask = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int m = m0 + wm * 32 + (t >> 1) * 16 + gq + (t & 1) * 8;
        cmo[t] = coff + (m < a.M ? at_off<Off>(a.cm, m) : (Off)0);
        cmask |= (m < a.M ? 1u : 0u) << t;
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int n = n0 + wn * 32 + (t >> 1) * 8 + tq * 2 + (t & 1);
        cno[t] = n < a.N ? at_off<Off>(a.cn, n) : (Off)0;
        cmask |= (n < a.N ? 1u : 0u) << (4 + t);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int tm = i * 2 + (e >> 1), tn = j * 2 + (e & 1);
                if (!((cmask >> tm) & (cmask >> (4 + tn)) & 1u)) continue;
                const Off off = cmo[tm] + cno[tn];
                float v = a.alpha * acc[i][j][e];
                if (a.ksplit > 1) {
                    atomicAdd(a.C + off, v);
                    continue;
                }
                if (a.beta != 0.f) v += a.beta * a.C[off];
                if (a.bias) v += a.bias[n0 + wn * 32 + j * 8 + tq * 2 + (e & 1)];
                a.C[off] = v;
                if (a.C2) a.C2[off] = gelu(v);
            }
}

}  // namespace

namespace {

// largest offset of the map over i = 0 .. n-1 (strides >= 0)
long long max_at(const Map &d, long long n) {
    if (n <= 0) return 0;
    if (d.g == (1 << 30)) return (n - 1) * d.s0;  // one level, as at()
    const long long q = (n - 1) / d.g, r = (n - 1) % d.g;
    long long m = q * d.s1 + r * d.s0;
    if (q >= 1) m = std::max(m, (q - 1) * d.s1 + (long long)(d.g - 1) * d.s0);
    return m;
}

bool nonneg(const Map &d) { return d.s0 >= 0 && d.s1 >= 0 && d.g >= 1; }

using Kern = void (*)(const GemmArgs);

template <typename Off, int C>
constexpr Kern kern() {
    return gemm_kernel<Off, (C >> 3) & 1, (C >> 2) & 1, (C >> 1) & 1, C & 1>;
}

// instance by code: bit 4 32-bit offsets, 3 A is BF16, 2 A staged along m,
// 1 B is BF16, 0 B staged along n
template <int... C>
const Kern *table(std::integer_sequence<int, C...>) {
    static const Kern t[] = {kern<long long, C>()..., kern<int, C>()...};
    return t;
}
const Kern *kernel_table() { return table(std::make_integer_sequence<int, 16>{}); }

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
    // lanes along the operand's unit-stride index: k where it has one, else
    // the row index (m of A, n of B)
    GemmArgs g = a;
    g.a_rows_fast = (a.ak.s0 != 1 && a.am.s0 == 1) ? 1 : 0;
    g.b_rows_fast = (a.bk.s0 != 1 && a.bn.s0 == 1) ? 1 : 0;
    // every offset below a_n, b_n or c_n: 32-bit offsets when all three fit
    const bool narrow = a.a_n < (1ll << 31) && a.b_n < (1ll << 31) && a.c_n < (1ll << 31);
    const int code = (narrow ? 16 : 0) | (a.a_bf16 ? 8 : 0) | (g.a_rows_fast ? 4 : 0) |
                     (a.b_bf16 ? 2 : 0) | (g.b_rows_fast ? 1 : 0);
    kernel_table()[code]<<<grid, 128, 0, s>>>(g);
    return cudaGetLastError();
}

}  // namespace fno
}  // namespace ehd
