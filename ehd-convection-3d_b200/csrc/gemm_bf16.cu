// gemm_bf16.cu -- the batched BF16 tensor-core product of gemm_bf16.cuh, and
// the weight and bias gradients of pointwise layers.
//
// gemm() sends a product to one of four kernels by its shape (the first three
// mma.sync.m16n8k16, BF16 operands, FP32 accumulation):
//  - rowwise_kernel: A FP32 with unit stride along k, 16 | K <= 128, N <= 128
//    (pointwise layers and their input gradients): B resident in shared
//    memory, A fragments straight from global memory, warps streaming 16-row
//    tiles;
//  - leftmul_kernel: one A for the whole batch, M, K <= 128, B FP32 with unit
//    stride along n (the truncated DFTs): A resident in shared memory, B
//    fragments straight from global memory in warp units of 8-32 columns;
//  - gemm_kernel, the general tiled product: 64 x 64 output tiles, K in steps
//    of 32, 128 threads, each warp a 32 x 32 quarter as 2 x 4 mma tiles;
//    operands staged in shared memory as BF16, A as [m][k] and B as [n][k],
//    so that every fragment register is one aligned 32-bit load of two
//    consecutive k;
//  - smallk_kernel, K <= 16 and N <= 128 with A and C row-major (the lift and
//    the projection's input gradient): BF16-rounded operands, FP32 FMAs,
//    bound by the bytes it writes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
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

// ---- row-streaming products ---------------------------------------------
//
// For products whose A is FP32 with unit stride along k (rows lda elements
// apart), K a multiple of 16 up to 128 and N up to 128 -- the pointwise layers
// and their input gradients.  B (K x N) is staged once per block in shared
// memory as BF16 [n][k]; each warp then streams 16-row tiles of A from global
// memory straight into its mma.sync A fragments (two FP32 per 64-bit load,
// converted to a BF16 pair), and writes its C fragments directly, two FP32
// per 64-bit store where C's rows allow.  Warps take tiles independently
// (no block barrier after the B stage); with KT <= 2 the next tile's loads
// are in flight during the current tile's products and epilogue.
constexpr int RW_WARPS = 8;

__device__ __forceinline__ float2 ldg2(const float *p) {
    return __ldg(reinterpret_cast<const float2 *>(p));
}

__device__ __forceinline__ uint32_t pack_bf16(float2 v) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
    return *reinterpret_cast<const uint32_t *>(&h);
}

template <int KT>
__device__ __forceinline__ void rw_load(float2 (&v)[KT][4], const float *A, int lda, int M,
                                        int tile, int gq, int tq) {
    const int r0 = tile * 16 + gq, r1 = r0 + 8;
    const bool ok0 = r0 < M, ok1 = r1 < M;
    const float *p0 = A + (size_t)(ok0 ? r0 : 0) * lda + 2 * tq;
    const float *p1 = A + (size_t)(ok1 ? r1 : 0) * lda + 2 * tq;
    const float2 z = make_float2(0.f, 0.f);
#pragma unroll
    for (int s = 0; s < KT; ++s) {
        v[s][0] = ok0 ? ldg2(p0 + 16 * s) : z;
        v[s][1] = ok1 ? ldg2(p1 + 16 * s) : z;
        v[s][2] = ok0 ? ldg2(p0 + 16 * s + 8) : z;
        v[s][3] = ok1 ? ldg2(p1 + 16 * s + 8) : z;
    }
}

template <int KT, int NT>
__global__ void __launch_bounds__(256) rowwise_kernel(const GemmArgs a, int lda, int ldc,
                                                      int pair_store) {
    constexpr int PKB = 16 * KT + 8;  // padded row of B (BF16 elements)
    constexpr bool PF = KT <= 2;      // prefetch the next tile
    extern __shared__ __align__(16) unsigned char rw_smem[];
    __nv_bfloat16 *Bs = reinterpret_cast<__nv_bfloat16 *>(rw_smem);  // [8 NT][PKB]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    const int bidx = blockIdx.y;
    {
        const long long boff = at(a.bbat, bidx);
        for (int i = tid; i < 8 * NT * 16 * KT; i += blockDim.x) {
            const int n = i / (16 * KT), k = i - n * (16 * KT);
            float v = 0.f;
            if (n < a.N && k < a.K) {
                const long long o = boff + at(a.bk, k) + at(a.bn, n);
                v = a.b_bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(a.B)[o])
                             : reinterpret_cast<const float *>(a.B)[o];
            }
            Bs[n * PKB + k] = __float2bfloat16_rn(v);
        }
    }
    __syncthreads();
    const float *A = reinterpret_cast<const float *>(a.A) + at(a.abat, bidx);
    float *C = a.C + at(a.cbat, bidx);
    float *C2 = a.C2 ? a.C2 + at(a.cbat, bidx) : nullptr;
    const int tiles = (a.M + 15) / 16;
    const int tstride = gridDim.x * RW_WARPS;
    int t = blockIdx.x * RW_WARPS + warp;
    float2 cur[KT][4];
    if (PF && t < tiles) rw_load<KT>(cur, A, lda, a.M, t, gq, tq);
    for (; t < tiles; t += tstride) {
        if (!PF) rw_load<KT>(cur, A, lda, a.M, t, gq, tq);
        uint32_t af[KT][4];
#pragma unroll
        for (int s = 0; s < KT; ++s)
#pragma unroll
            for (int e = 0; e < 4; ++e) af[s][e] = pack_bf16(cur[s][e]);
        if (PF && t + tstride < tiles) rw_load<KT>(cur, A, lda, a.M, t + tstride, gq, tq);
        float acc[NT][4];
#pragma unroll
        for (int j = 0; j < NT; ++j) {
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;
            const __nv_bfloat16 *bp = Bs + (8 * j + gq) * PKB + 2 * tq;
#pragma unroll
            for (int s = 0; s < KT; ++s) {
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(bp + 16 * s);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(bp + 16 * s + 8);
                mma16816(acc[j], af[s][0], af[s][1], af[s][2], af[s][3], b0, b1);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int m = t * 16 + gq + 8 * h;
            if (m >= a.M) continue;
            float *crow = C + (size_t)m * ldc;
            float *c2row = C2 ? C2 + (size_t)m * ldc : nullptr;
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const int n = 8 * j + 2 * tq;
                if (n >= a.N) continue;
                float v0 = a.alpha * acc[j][2 * h], v1 = a.alpha * acc[j][2 * h + 1];
                if (pair_store && n + 1 < a.N) {
                    if (a.beta != 0.f) {
                        const float2 o = *reinterpret_cast<const float2 *>(crow + n);
                        v0 += a.beta * o.x;
                        v1 += a.beta * o.y;
                    }
                    if (a.bias) {
                        v0 += __ldg(a.bias + n);
                        v1 += __ldg(a.bias + n + 1);
                    }
                    *reinterpret_cast<float2 *>(crow + n) = make_float2(v0, v1);
                    if (c2row) *reinterpret_cast<float2 *>(c2row + n) = make_float2(gelu(v0), gelu(v1));
                } else {
                    if (a.beta != 0.f) v0 += a.beta * crow[n];
                    if (a.bias) v0 += __ldg(a.bias + n);
                    crow[n] = v0;
                    if (c2row) c2row[n] = gelu(v0);
                    if (n + 1 < a.N) {
                        if (a.beta != 0.f) v1 += a.beta * crow[n + 1];
                        if (a.bias) v1 += __ldg(a.bias + n + 1);
                        crow[n + 1] = v1;
                        if (c2row) c2row[n + 1] = gelu(v1);
                    }
                }
            }
        }
    }
}

// ---- products by a small left matrix --------------------------------------
//
// For C[b][m][n] = alpha sum_k A[m][k] B[b][k][n] with one A for the whole
// batch, M, K <= 128, and B FP32 with unit stride along n -- the truncated
// DFTs of the FNO, whose B is the activation tensor and A the DFT matrix.  A
// is staged once per block in shared memory as BF16 [m][k]; each warp then
// takes units of 8 NT consecutive columns of one batch entry and loads its
// mma.sync B fragments straight from global memory (lanes along n: every
// load instruction reads four fully used 32-byte sectors), the next K step's
// fragments in flight during the current step's products, and writes its C
// fragments directly (64-bit stores where C's layout allows).
template <int NT>
__device__ __forceinline__ void lm_load(float (&rb)[NT][4], const float *B, const int (&bno)[NT],
                                        unsigned nmask, const Map &bk, int K, int s, int tq) {
    const int k0 = 16 * s + 2 * tq;
    int ko[4];
    bool kin[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int k = k0 + (e & 1) + (e >> 1) * 8;
        kin[e] = k < K;
        ko[e] = kin[e] ? at_off<int>(bk, k) : 0;
    }
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
            rb[j][e] = (kin[e] && (nmask >> j & 1u)) ? __ldg(B + bno[j] + ko[e]) : 0.f;
}

// C fragments of one warp unit (rows 16 i + gq + 8 h, columns n0 + 8 j + 2 tq
// and + 1) with alpha, beta, bias and the optional GELU output
template <int MT, int NT>
__device__ __forceinline__ void lm_epilogue(const GemmArgs &a, const float (&acc)[MT][NT][4],
                                            int bidx, int n0, int gq, int tq, int pair_store) {
    const int coff = at_off<int>(a.cbat, bidx);
    int cno[NT];
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        const int n = n0 + 8 * j + 2 * tq;
        cno[j] = n < a.N ? at_off<int>(a.cn, n) : 0;
    }
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int m = 16 * i + gq + 8 * h;
            if (m >= a.M) continue;
            const int mo = coff + at_off<int>(a.cm, m);
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const int n = n0 + 8 * j + 2 * tq;
                if (n >= a.N) continue;
                float v0 = a.alpha * acc[i][j][2 * h], v1 = a.alpha * acc[i][j][2 * h + 1];
                float *c = a.C + mo + cno[j];
                if (pair_store && n + 1 < a.N) {
                    if (a.beta != 0.f) {
                        const float2 o = *reinterpret_cast<const float2 *>(c);
                        v0 += a.beta * o.x;
                        v1 += a.beta * o.y;
                    }
                    if (a.bias) {
                        v0 += __ldg(a.bias + n);
                        v1 += __ldg(a.bias + n + 1);
                    }
                    *reinterpret_cast<float2 *>(c) = make_float2(v0, v1);
                    if (a.C2)
                        *reinterpret_cast<float2 *>(a.C2 + mo + cno[j]) =
                            make_float2(gelu(v0), gelu(v1));
                } else {
                    if (a.beta != 0.f) v0 += a.beta * *c;
                    if (a.bias) v0 += __ldg(a.bias + n);
                    *c = v0;
                    if (a.C2) a.C2[mo + cno[j]] = gelu(v0);
                    if (n + 1 < a.N) {
                        const int o1 = mo + at_off<int>(a.cn, n + 1);
                        if (a.beta != 0.f) v1 += a.beta * a.C[o1];
                        if (a.bias) v1 += __ldg(a.bias + n + 1);
                        a.C[o1] = v1;
                        if (a.C2) a.C2[o1] = gelu(v1);
                    }
                }
            }
        }
}

template <int MT, int NT>
__global__ void __launch_bounds__(256) leftmul_kernel(const GemmArgs a, int pair_store) {
    constexpr int NC = 8 * NT;
    extern __shared__ __align__(16) unsigned char lm_smem[];
    const int kt = (a.K + 15) / 16, KP = 16 * kt + 8;
    __nv_bfloat16 *As = reinterpret_cast<__nv_bfloat16 *>(lm_smem);  // [16 MT][KP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    for (int i = tid; i < 16 * MT * 16 * kt; i += blockDim.x) {
        const int m = i / (16 * kt), k = i - m * (16 * kt);
        float v = 0.f;
        if (m < a.M && k < a.K) {
            const long long o = at(a.am, m) + at(a.ak, k);
            v = a.a_bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(a.A)[o])
                         : reinterpret_cast<const float *>(a.A)[o];
        }
        As[m * KP + k] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    const float *B = reinterpret_cast<const float *>(a.B);
    const int chunks = (a.N + NC - 1) / NC;
    const long long units = (long long)a.batch * chunks;
    const long long ustep = (long long)gridDim.x * 8;
    // the B offsets of unit u's columns
    auto unit_cols = [&](long long u, int (&bno)[NT], unsigned &nmask) {
        const int bidx = (int)(u / chunks), n0 = (int)(u - (long long)bidx * chunks) * NC;
        const int boff = at_off<int>(a.bbat, bidx);
        nmask = 0;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int n = n0 + 8 * j + gq;
            bno[j] = boff + (n < a.N ? at_off<int>(a.bn, n) : 0);
            nmask |= (n < a.N ? 1u : 0u) << j;
        }
    };
    int bno[NT];
    unsigned nmask = 0;
    float rb[NT][4];
    long long u = (long long)blockIdx.x * 8 + warp;
    if (u < units) {
        unit_cols(u, bno, nmask);
        lm_load<NT>(rb, B, bno, nmask, a.bk, a.K, 0, tq);
    }
    for (; u < units; u += ustep) {
        const int bidx = (int)(u / chunks), n0 = (int)(u - (long long)bidx * chunks) * NC;
        float acc[MT][NT][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
        for (int s = 0; s < kt; ++s) {
            uint32_t bf[NT][2];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                bf[j][0] = pack_bf16(make_float2(rb[j][0], rb[j][1]));
                bf[j][1] = pack_bf16(make_float2(rb[j][2], rb[j][3]));
            }
            // the next K step's fragments in flight during this step's
            // products; after the last step, the next unit's first
            if (s + 1 < kt) {
                lm_load<NT>(rb, B, bno, nmask, a.bk, a.K, s + 1, tq);
            } else if (u + ustep < units) {
                unit_cols(u + ustep, bno, nmask);
                lm_load<NT>(rb, B, bno, nmask, a.bk, a.K, 0, tq);
            }
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const __nv_bfloat16 *ap = As + (16 * i + gq) * KP + 16 * s + 2 * tq;
                const uint32_t a0 = *reinterpret_cast<const uint32_t *>(ap);
                const uint32_t a1 = *reinterpret_cast<const uint32_t *>(ap + 8 * KP);
                const uint32_t a2 = *reinterpret_cast<const uint32_t *>(ap + 8);
                const uint32_t a3 = *reinterpret_cast<const uint32_t *>(ap + 8 * KP + 8);
#pragma unroll
                for (int j = 0; j < NT; ++j) mma16816(acc[i][j], a0, a1, a2, a3, bf[j][0], bf[j][1]);
            }
        }
        lm_epilogue<MT, NT>(a, acc, bidx, n0, gq, tq, pair_store);
    }
}


// ---- the same products with B staged by asynchronous copies ---------------
//
// Where every row of a warp unit's B block (NC = 8 NT consecutive columns at
// one k) starts on a 16-byte boundary, each warp streams its units' K steps
// into a ring of LM_STAGES shared-memory buffers of its own by cp.async (16
// bytes a lane per copy, no registers held while the copies fly), LM_STAGES - 1
// steps ahead of the products and across unit boundaries, and reads its
// fragments from shared memory (rows padded by 4 floats, so that the 32 lanes
// of a fragment load hit 32 distinct banks).  Columns past N and k past K are
// zero-filled by the copies.
constexpr int LM_STAGES = 3;

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int NT>
constexpr int lm_stage_floats() { return 16 * (8 * NT + 4); }

template <int MT, int NT>
__global__ void __launch_bounds__(256) leftmul_cp_kernel(const GemmArgs a, int pair_store) {
    constexpr int NC = 8 * NT, RS = NC + 4, STAGE = lm_stage_floats<NT>();
    constexpr int C4 = NC / 4, CH = 16 * C4, CPL = (CH + 31) / 32;
    extern __shared__ __align__(16) unsigned char lm_smem[];
    const int kt = (a.K + 15) / 16, KP = 16 * kt + 8;
    __nv_bfloat16 *As = reinterpret_cast<__nv_bfloat16 *>(lm_smem);  // [16 MT][KP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    float *ring = reinterpret_cast<float *>(lm_smem + ((size_t)16 * MT * KP * 2 + 15) / 16 * 16) +
                  (size_t)warp * LM_STAGES * STAGE;
    for (int i = tid; i < 16 * MT * 16 * kt; i += blockDim.x) {
        const int m = i / (16 * kt), k = i - m * (16 * kt);
        float v = 0.f;
        if (m < a.M && k < a.K) {
            const long long o = at(a.am, m) + at(a.ak, k);
            v = a.a_bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16 *>(a.A)[o])
                         : reinterpret_cast<const float *>(a.A)[o];
        }
        As[m * KP + k] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    const float *B = reinterpret_cast<const float *>(a.B);
    const int chunks = (a.N + NC - 1) / NC;
    const long long units = (long long)a.batch * chunks;
    const long long ustep = (long long)gridDim.x * 8;
    // copy cursor: unit lu, K step ls
    long long lu = (long long)blockIdx.x * 8 + warp;
    int ls = 0, lbase = 0, lcols = 0;
    auto set_unit = [&](long long u) {
        const int bidx = (int)(u / chunks), n0 = (int)(u - (long long)bidx * chunks) * NC;
        lbase = at_off<int>(a.bbat, bidx) + at_off<int>(a.bn, n0);
        lcols = a.N - n0 < NC ? a.N - n0 : NC;
    };
    if (lu < units) set_unit(lu);
    auto issue = [&](int slot) {
        if (lu < units) {
            float *dst = ring + slot * STAGE;
#pragma unroll
            for (int t = 0; t < CPL; ++t) {
                const int c = lane + 32 * t;
                if (CH % 32 == 0 || c < CH) {
                    const int r = c / C4, col = 4 * (c - r * C4), k = 16 * ls + r;
                    int nv = lcols - col;
                    nv = k < a.K ? (nv < 0 ? 0 : (nv > 4 ? 4 : nv)) : 0;
                    const float *src = nv > 0 ? B + lbase + at_off<int>(a.bk, k) + col : B;
                    cp_async16(dst + r * RS + col, src, 4 * nv);
                }
            }
            if (++ls == kt) {
                ls = 0;
                lu += ustep;
                if (lu < units) set_unit(lu);
            }
        }
        cp_commit();  // one group per call, empty or not: the waits count groups
    };
#pragma unroll
    for (int t = 0; t < LM_STAGES - 1; ++t) issue(t);
    int cslot = 0, islot = LM_STAGES - 1;
    for (long long u = (long long)blockIdx.x * 8 + warp; u < units; u += ustep) {
        const int bidx = (int)(u / chunks), n0 = (int)(u - (long long)bidx * chunks) * NC;
        float acc[MT][NT][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
        for (int s = 0; s < kt; ++s) {
            cp_wait<LM_STAGES - 2>();
            __syncwarp();  // every lane's copies of this step landed; the slot
                           // consumed last step is free for the next copies
            const float *st = ring + cslot * STAGE + gq;
            uint32_t bf[NT][2];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const float *c0 = st + 8 * j;
                bf[j][0] = pack_bf16(make_float2(c0[(2 * tq) * RS], c0[(2 * tq + 1) * RS]));
                bf[j][1] = pack_bf16(make_float2(c0[(2 * tq + 8) * RS], c0[(2 * tq + 9) * RS]));
            }
            issue(islot);
            cslot = cslot + 1 == LM_STAGES ? 0 : cslot + 1;
            islot = islot + 1 == LM_STAGES ? 0 : islot + 1;
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const __nv_bfloat16 *ap = As + (16 * i + gq) * KP + 16 * s + 2 * tq;
                const uint32_t a0 = *reinterpret_cast<const uint32_t *>(ap);
                const uint32_t a1 = *reinterpret_cast<const uint32_t *>(ap + 8 * KP);
                const uint32_t a2 = *reinterpret_cast<const uint32_t *>(ap + 8);
                const uint32_t a3 = *reinterpret_cast<const uint32_t *>(ap + 8 * KP + 8);
#pragma unroll
                for (int j = 0; j < NT; ++j) mma16816(acc[i][j], a0, a1, a2, a3, bf[j][0], bf[j][1]);
            }
        }
        lm_epilogue<MT, NT>(a, acc, bidx, n0, gq, tq, pair_store);
    }
    cp_wait<0>();
}


// ---- products with a small K -------------------------------------------------
//
// C[m][n] = alpha sum_k A[m][k] B[k][n] (+ beta C, + bias[n], GELU output) for
// K <= 16 and N <= 128 with A and C row-major: the FNO's lift (K = 9) and the
// projection's input gradient (K = 5).  They are bound by the output bytes, so
// they run on the FP32 pipes, K a template parameter: lane l holds B[k][n] of
// its columns n = l + 32 j in registers, each warp takes 32 rows at a time
// (their A values loaded one tile ahead into registers, staged in shared
// memory, read back as broadcasts).  Operands are rounded to BF16 as on the tensor-core paths, so
// every product is the same exact FP32 value; only the order of the K-term
// sum differs.
constexpr int SK_MAXK = 16, SK_MAXN = 128, SK_NJ = SK_MAXN / 32;

template <int BF, int KK>
__global__ void __launch_bounds__(256) smallk_kernel(const GemmArgs a) {
    __shared__ float As[8][32 * KK];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int N = a.N;
    float bv[KK][SK_NJ];
#pragma unroll
    for (int k = 0; k < KK; ++k)
#pragma unroll
        for (int j = 0; j < SK_NJ; ++j) {
            const int n = lane + 32 * j;
            float v = 0.f;
            if (n < N) {
                const long long o = at(a.bk, k) + at(a.bn, n);
                v = a.b_bf16 ? __bfloat162float(to_bf16<1>(ld_raw<1>(a.B, o)))
                             : __bfloat162float(to_bf16<0>(ld_raw<0>(a.B, o)));
            }
            bv[k][j] = v;
        }
    const long long lda = a.am.s0, ldc = a.cm.s0;
    float *as = As[warp];
    const long long tiles = ((long long)a.M + 31) / 32, tstep = (long long)gridDim.x * 8;
    // the next tile's A values in flight while this tile's rows are computed
    uint32_t araw[KK];
    auto load_tile = [&](long long t) {
        const long long m0 = t * 32;
        const int rows = a.M - m0 < 32 ? (int)(a.M - m0) : 32;
#pragma unroll
        for (int u = 0; u < KK; ++u) {
            const int i = lane + 32 * u, r = i / KK, k = i - r * KK;
            araw[u] = r < rows ? ld_raw<BF>(a.A, (m0 + r) * lda + k) : 0u;
        }
    };
    long long t = (long long)blockIdx.x * 8 + warp;
    if (t < tiles) load_tile(t);
    for (; t < tiles; t += tstep) {
        const long long m0 = t * 32;
        const int rows = a.M - m0 < 32 ? (int)(a.M - m0) : 32;
        __syncwarp();
#pragma unroll
        for (int u = 0; u < KK; ++u) as[lane + 32 * u] = __bfloat162float(to_bf16<BF>(araw[u]));
        __syncwarp();
        if (t + tstep < tiles) load_tile(t + tstep);
        for (int r = 0; r < rows; ++r) {
            float ar[KK];
#pragma unroll
            for (int k = 0; k < KK; ++k) ar[k] = as[r * KK + k];
            float *crow = a.C + (m0 + r) * ldc;
#pragma unroll
            for (int j = 0; j < SK_NJ; ++j) {
                const int n = lane + 32 * j;
                if (n < N) {
                    float acc = 0.f;
#pragma unroll
                    for (int k = 0; k < KK; ++k) acc = fmaf(ar[k], bv[k][j], acc);
                    float v = a.alpha * acc;
                    if (a.beta != 0.f) v += a.beta * crow[n];
                    if (a.bias) v += __ldg(a.bias + n);
                    crow[n] = v;
                    if (a.C2) a.C2[(m0 + r) * ldc + n] = gelu(v);
                }
            }
        }
    }
}

// ---- parameter gradients of pointwise layers ------------------------------
//
// G[m][n] += sum_r X[r][m] D[r][n] and gb[n] += sum_r D[r][n] over all rows r
// (X rows ldx apart, D rows ldd apart, M <= 16 MT, N <= 8 NT): the weight and
// bias gradients of a pointwise layer in one pass over X and D.  Each warp
// takes 16-row chunks; its mma.sync fragments come straight from global
// memory (lanes along the channel: every load reads four fully used 32-byte
// sectors), the bias sums are taken in FP32 from the same D values before
// they are rounded to BF16; the block reduces its warps' partial sums in
// shared memory and adds them to G and gb atomically.  Two blocks per SM: at
// 64 accumulators a thread (MT NT = 16) that spills a few registers and is
// faster than one block.
template <int MT, int NT>
__global__ void __launch_bounds__(256, 2) wgrad_kernel(const float *__restrict__ X, int ldx, int M,
                                                    const float *__restrict__ D, int ldd, int N,
                                                    long long rows, float *__restrict__ G,
                                                    int ldg, float *__restrict__ gb) {
    constexpr int NV = MT * NT * 128;         // partial sums of G per warp
    __shared__ float red[4][NV + NT * 8];     // warps w and w + 4 share a row
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    float acc[MT][NT][4], bs[NT];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
    for (int j = 0; j < NT; ++j) bs[j] = 0.f;
    const long long chunks = (rows + 15) / 16;
    for (long long c = (long long)blockIdx.x * 8 + warp; c < chunks; c += (long long)gridDim.x * 8) {
        const long long r0 = c * 16 + 2 * tq;
        // rows r0, r0 + 1, r0 + 8, r0 + 9 of this lane
        long long rr[4];
        bool rin[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            rr[e] = r0 + (e & 1) + (e >> 1) * 8;
            rin[e] = rr[e] < rows;
        }
        uint32_t bf[NT][2];
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int n = 8 * j + gq;
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e)
                v[e] = (rin[e] && n < N) ? __ldg(D + rr[e] * ldd + n) : 0.f;
            bs[j] += (v[0] + v[1]) + (v[2] + v[3]);
            bf[j][0] = pack_bf16(make_float2(v[0], v[1]));
            bf[j][1] = pack_bf16(make_float2(v[2], v[3]));
        }
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            const int m0 = 16 * i + gq, m1 = m0 + 8;
            float x[8];  // (m0, m1) x rows e
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                x[e] = (rin[e] && m0 < M) ? __ldg(X + rr[e] * ldx + m0) : 0.f;
                x[4 + e] = (rin[e] && m1 < M) ? __ldg(X + rr[e] * ldx + m1) : 0.f;
            }
            const uint32_t a0 = pack_bf16(make_float2(x[0], x[1]));
            const uint32_t a1 = pack_bf16(make_float2(x[4], x[5]));
            const uint32_t a2 = pack_bf16(make_float2(x[2], x[3]));
            const uint32_t a3 = pack_bf16(make_float2(x[6], x[7]));
#pragma unroll
            for (int j = 0; j < NT; ++j) mma16816(acc[i][j], a0, a1, a2, a3, bf[j][0], bf[j][1]);
        }
    }
    // bias sums of column 8 j + gq: the four lanes of a row group
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        bs[j] += __shfl_xor_sync(0xffffffffu, bs[j], 1);
        bs[j] += __shfl_xor_sync(0xffffffffu, bs[j], 2);
    }
    // warps 4..7 store their partial sums, warps 0..3 add theirs to them
    float *my = red[warp & 3];
    for (int half = 1; half >= 0; --half) {
        if ((warp >> 2) == half) {
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        float &r = my[((i * NT + j) * 4 + e) * 32 + lane];
                        r = half ? acc[i][j][e] : r + acc[i][j][e];
                    }
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                float &r = my[NV + 8 * j + gq];
                if (tq == 0) r = half ? bs[j] : r + bs[j];
            }
        }
        __syncthreads();
    }
    for (int t = tid; t < NV + NT * 8; t += blockDim.x) {
        float sum = 0.f;
#pragma unroll
        for (int w = 0; w < 4; ++w) sum += red[w][t];
        if (t < NV) {
            const int ln = t & 31, f = t >> 5;
            const int e = f & 3, j = (f >> 2) % NT, i = (f >> 2) / NT;
            const int m = 16 * i + (ln >> 2) + (e >> 1) * 8, n = 8 * j + (ln & 3) * 2 + (e & 1);
            if (m < M && n < N) atomicAdd(G + (size_t)m * ldg + n, sum);
        } else if (gb) {
            const int n = t - NV;
            if (n < N) atomicAdd(gb + n, sum);
        }
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

namespace {

using RowKern = void (*)(const GemmArgs, int, int, int);

template <int KT>
RowKern row_kernel(int nt) {
    switch (nt) {
        case 1: return rowwise_kernel<KT, 1>;
        case 2: return rowwise_kernel<KT, 2>;
        case 4: return rowwise_kernel<KT, 4>;
        case 8: return rowwise_kernel<KT, 8>;
        default: return rowwise_kernel<KT, 16>;
    }
}

bool aligned8(const void *p) { return ((uintptr_t)p & 7u) == 0; }
bool one_level(const Map &m) { return m.g == (1 << 30); }

// The row-streaming kernel when the product has its shape: A FP32 with unit
// stride along k, lda and the batch offsets even, 16 | K <= 128, N <= 128,
// unit stride along n in C, no split K.  Returns false to leave the product
// to the tiled kernel.
bool try_rowwise(const GemmArgs &a, cudaStream_t s, cudaError_t *err) {
    if (a.a_bf16 || a.ksplit != 1 || a.K % 16 != 0 || a.K > 128 || a.N > 128) return false;
    if (!one_level(a.am) || !one_level(a.ak) || !one_level(a.abat) || !one_level(a.cm) ||
        !one_level(a.cn) || !one_level(a.cbat))
        return false;
    // (the batch maps matter only with more than one product)
    const bool odd_abat = a.batch > 1 && (a.abat.s0 & 1);
    if (a.ak.s0 != 1 || a.cn.s0 != 1 || a.am.s0 < a.K || (a.am.s0 & 1) || odd_abat ||
        !aligned8(a.A) || a.am.s0 > (1ll << 30) || a.cm.s0 > (1ll << 30))
        return false;
    const int kt = a.K / 16;
    const int nt = a.N <= 8 ? 1 : a.N <= 16 ? 2 : a.N <= 32 ? 4 : a.N <= 64 ? 8 : 16;
    RowKern k = nullptr;
    switch (kt) {
        case 1: k = row_kernel<1>(nt); break;
        case 2: k = row_kernel<2>(nt); break;
        case 4: k = row_kernel<4>(nt); break;
        case 8: k = row_kernel<8>(nt); break;
        default: return false;  // K = 48, 80, 96, 112: the tiled kernel
    }
    const int pair = (a.cm.s0 % 2 == 0 && (a.batch == 1 || a.cbat.s0 % 2 == 0) && aligned8(a.C) &&
                      (!a.C2 || aligned8(a.C2)))
                         ? 1
                         : 0;
    const size_t smem = (size_t)8 * nt * (16 * kt + 8) * sizeof(__nv_bfloat16);
    int dev = 0, nsm = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem)) != cudaSuccess) {
        *err = e;
        return true;
    }
    const long long tiles = (a.M + 15) / 16;
    const long long want = (tiles + RW_WARPS - 1) / RW_WARPS;
    const long long per_batch = std::max(1ll, (long long)nsm * std::max(occ, 1) / a.batch);
    dim3 grid((unsigned)std::min(want, per_batch), (unsigned)a.batch, 1);
    k<<<grid, 256, smem, s>>>(a, (int)a.am.s0, (int)a.cm.s0, pair);
    *err = cudaGetLastError();
    return true;
}

using LeftKern = void (*)(const GemmArgs, int);

template <int NT>
LeftKern left_kernel_nt(int mt) {
    switch (mt) {
        case 1: return leftmul_kernel<1, NT>;
        case 2: return leftmul_kernel<2, NT>;
        case 3: return leftmul_kernel<3, NT>;
        case 4: return leftmul_kernel<4, NT>;
        case 5: return leftmul_kernel<5, NT < 4 ? NT : 2>;
        case 6: return leftmul_kernel<6, NT < 4 ? NT : 2>;
        case 7: return leftmul_kernel<7, NT < 4 ? NT : 2>;
        default: return leftmul_kernel<8, NT < 4 ? NT : 2>;
    }
}

// 8 NT columns per warp unit: the widest unit (at most 32 accumulators a
// thread, MT NT <= 8: more blocks per SM measured faster than wider units)
// that still gives 4096 units, so that every warp of a full GPU has several
// to interleave
int left_nt(int mt, long long batch, int N) {
    for (int nt = 4; nt > 1; nt /= 2)
        if (mt * nt <= 8 && batch * ((N + 8 * nt - 1) / (8 * nt)) >= 4096) return nt;
    return 1;
}

LeftKern left_kernel(int mt, int nt) {
    return nt == 4 ? left_kernel_nt<4>(mt) : nt == 2 ? left_kernel_nt<2>(mt) : left_kernel_nt<1>(mt);
}

template <int NT>
LeftKern left_cp_kernel_nt(int mt) {
    switch (mt) {
        case 1: return leftmul_cp_kernel<1, NT>;
        case 2: return leftmul_cp_kernel<2, NT>;
        case 3: return leftmul_cp_kernel<3, NT>;
        case 4: return leftmul_cp_kernel<4, NT>;
        case 5: return leftmul_cp_kernel<5, NT < 4 ? NT : 2>;
        case 6: return leftmul_cp_kernel<6, NT < 4 ? NT : 2>;
        case 7: return leftmul_cp_kernel<7, NT < 4 ? NT : 2>;
        default: return leftmul_cp_kernel<8, NT < 4 ? NT : 2>;
    }
}
LeftKern left_cp_kernel(int mt, int nt) {
    return nt == 4 ? left_cp_kernel_nt<4>(mt)
                   : nt == 2 ? left_cp_kernel_nt<2>(mt) : left_cp_kernel_nt<1>(mt);
}
// every row of every unit's B block on a 16-byte boundary (cp.async)
bool left_cp_aligned(const GemmArgs &a) {
    auto m4 = [](const Map &m) { return m.s0 % 4 == 0 && (one_level(m) || m.s1 % 4 == 0); };
    return ((uintptr_t)a.B & 15u) == 0 && m4(a.bk) && (a.batch == 1 || m4(a.bbat)) &&
           (one_level(a.bn) || a.bn.s1 % 4 == 0);
}

bool even_map(const Map &m) { return (m.s0 % 2 == 0) && (one_level(m) || m.s1 % 2 == 0); }

// The small-left-matrix kernel when the product has its shape: one A for the
// whole batch, M, K <= 128, B FP32 with unit stride along n (in runs of at
// least a warp unit's columns), no split K, every offset below 2^31.
bool try_leftmul(const GemmArgs &a, cudaStream_t s, cudaError_t *err) {
    if (a.b_bf16 || a.ksplit != 1 || a.M > 128 || a.K > 128) return false;
    if (a.batch > 1 && !(one_level(a.abat) && a.abat.s0 == 0)) return false;
    if (a.a_n >= (1ll << 31) || a.b_n >= (1ll << 31) || a.c_n >= (1ll << 31)) return false;
    const int mt = (a.M + 15) / 16, kt = (a.K + 15) / 16;
    const int nt = left_nt(mt, a.batch, a.N);
    if (a.bn.s0 != 1 || (!one_level(a.bn) && a.bn.g % (8 * nt) != 0)) return false;
    // 64-bit stores of column pairs: unit stride along n in runs of even
    // length, even strides elsewhere, 8-byte aligned outputs
    const bool pair = a.cn.s0 == 1 && (one_level(a.cn) || (a.cn.g % 2 == 0 && a.cn.s1 % 2 == 0)) &&
                      even_map(a.cm) && (a.batch == 1 || even_map(a.cbat)) && aligned8(a.C) &&
                      (!a.C2 || aligned8(a.C2));
    // B staged by asynchronous copies where its rows are 16-byte aligned
    const bool staged = left_cp_aligned(a);
    LeftKern k = staged ? left_cp_kernel(mt, nt) : left_kernel(mt, nt);
    size_t smem = (size_t)16 * mt * (16 * kt + 8) * sizeof(__nv_bfloat16);
    if (staged) {
        const int stage = nt == 4 ? lm_stage_floats<4>() : nt == 2 ? lm_stage_floats<2>()
                                                                   : lm_stage_floats<1>();
        smem = (smem + 15) / 16 * 16 + (size_t)8 * LM_STAGES * stage * sizeof(float);
    }
    int dev = 0, nsm = 0, occ = 0;
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024)
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess || (e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem)) != cudaSuccess) {
        *err = e;
        return true;
    }
    const long long units = (long long)a.batch * ((a.N + 8 * nt - 1) / (8 * nt));
    const long long blocks = std::min((units + 7) / 8, (long long)nsm * std::max(occ, 1));
    k<<<(unsigned)blocks, 256, smem, s>>>(a, pair ? 1 : 0);
    *err = cudaGetLastError();
    return true;
}

using SmallKern = void (*)(const GemmArgs);
template <int BF, int... KS>
std::array<SmallKern, sizeof...(KS)> smallk_row(std::integer_sequence<int, KS...>) {
    return {smallk_kernel<BF, KS + 1>...};
}
const std::array<std::array<SmallKern, SK_MAXK>, 2> &smallk_table() {
    static const std::array<std::array<SmallKern, SK_MAXK>, 2> t = {
        smallk_row<0>(std::make_integer_sequence<int, SK_MAXK>{}),
        smallk_row<1>(std::make_integer_sequence<int, SK_MAXK>{})};
    return t;
}

// The small-K kernel when the product has its shape: K <= 16, N <= 128, one
// product (no batch, no split K), A with unit stride along k and C along n.
bool try_smallk(const GemmArgs &a, cudaStream_t s, cudaError_t *err) {
    if (a.K > SK_MAXK || a.N > SK_MAXN || a.batch != 1 || a.ksplit != 1) return false;
    if (!one_level(a.ak) || a.ak.s0 != 1 || !one_level(a.am) || !one_level(a.cn) ||
        a.cn.s0 != 1 || !one_level(a.cm))
        return false;
    SmallKern k = smallk_table()[a.a_bf16 ? 1 : 0][a.K - 1];
    int dev = 0, nsm = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, 0)) != cudaSuccess) {
        *err = e;
        return true;
    }
    // one wave of resident blocks, each warp walking its tiles
    const long long tiles = ((long long)a.M + 31) / 32;
    const long long blocks = std::min((tiles + 7) / 8, (long long)nsm * std::max(occ, 1));
    k<<<(unsigned)blocks, 256, 0, s>>>(a);
    *err = cudaGetLastError();
    return true;
}

using WgradKern = void (*)(const float *, int, int, const float *, int, int, long long, float *,
                           int, float *);

template <int MT>
WgradKern wgrad_kernel_nt(int nt) {
    switch (nt) {
        case 1: return wgrad_kernel<MT, 1>;
        case 2: return wgrad_kernel<MT, (16 / MT >= 2 ? 2 : 1)>;
        case 4: return wgrad_kernel<MT, (16 / MT >= 4 ? 4 : 1)>;
        case 8: return wgrad_kernel<MT, (16 / MT >= 8 ? 8 : 1)>;
        default: return wgrad_kernel<MT, (16 / MT >= 8 ? 8 : 1)>;
    }
}

}  // namespace

cudaError_t weight_bias_grad(long long rows, int M, int N, const float *X, int ldx, const float *D,
                             int ldd, float *G, int ldg, float *gb, cudaStream_t s) {
    if (rows <= 0 || M <= 0 || N <= 0) return cudaSuccess;
    if (M > 128 || ldx < M || ldd < N || ldg < N) return cudaErrorInvalidValue;
    const int mt = M <= 16 ? 1 : M <= 32 ? 2 : M <= 64 ? 4 : 8;
    const int ntmax = std::min(8, 16 / mt);  // at most 64 accumulators a thread
    int dev = 0, nsm = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    // columns in passes of at most 8 ntmax
    for (int n0 = 0; n0 < N; n0 += 8 * ntmax) {
        const int nn = std::min(N - n0, 8 * ntmax);
        int nt = 1;
        while (8 * nt < nn) nt *= 2;
        WgradKern k = mt == 1 ? wgrad_kernel_nt<1>(nt) : mt == 2 ? wgrad_kernel_nt<2>(nt)
                    : mt == 4 ? wgrad_kernel_nt<4>(nt) : wgrad_kernel_nt<8>(nt);
        int occ = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, 0)) != cudaSuccess)
            return e;
        const long long chunks = (rows + 15) / 16;
        const long long blocks = std::min((chunks + 7) / 8, (long long)nsm * std::max(occ, 1));
        k<<<(unsigned)blocks, 256, 0, s>>>(X, ldx, M, D + n0, ldd, nn, rows, G + n0, ldg,
                                          gb ? gb + n0 : nullptr);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

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
    cudaError_t rerr = cudaSuccess;
    if (try_rowwise(a, s, &rerr) || try_leftmul(a, s, &rerr) || try_smallk(a, s, &rerr))
        return rerr;
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
