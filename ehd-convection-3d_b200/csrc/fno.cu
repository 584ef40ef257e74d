// fno.cu -- the Fourier neural operator of include/ehd_fno.h: parameters,
// forward pass, backward pass and Adam.  The pointwise layers, the truncated
// DFTs and their adjoints run on the BF16 tensor cores through the products
// of gemm_bf16.cu; the per-mode mixing (a batch of matrix-vector products,
// one per kept mode) runs in FP32 on the complex weights.
//
// Layouts.  Activations are channels-last, v[b][z][y][x][c] (W channels).
// The spectral convolution of a layer runs as three truncated DFTs, each a
// batched matrix product with a small DFT matrix, whose outputs are laid out
// so that the next product reads a plain matrix:
//   Xh[b][z][ri][y][kx][c]     after the real transform along x (kx < mx)
//   Yh[b][ri][z][ky][kx][c]    after the transform along y (2 my modes)
//   Zh[b][ri][kz][ky][kx][c]   after the transform along z (2 mz modes)
// ri is 0 for the real, 1 for the imaginary part.  The mode mixing multiplies,
// per mode, the complex W x W matrix R with every sample's complex channel
// vector (conj(R)^T in the adjoint).  The inverse transforms mirror the forward
// ones, ending with the real inverse along x (factor 2 on kx > 0) and the
// 1 / (NX NY NZ) normalisation.  The backward pass applies the transposed
// matrices in the reverse order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "ehd.h"
#include "ehd_fno.h"
#include "gemm_bf16.cuh"
#include "kernels.h"

using namespace ehd;
using namespace ehd::fno;

namespace {

struct Off {  // offsets of one layer's parameters in the FP32 vector
    size_t W, b, Rre, Rim;
};

__global__ void cast_bf16_kernel(const float *__restrict__ src, __nv_bfloat16 *__restrict__ dst,
                                 size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

// Mode mixing.  Per kept mode md, the complex W x W weight R[md] (FP32 Re and
// Im, [out][in]) acts on every sample's complex channel vector, with the
// real and imaginary parts at Zh[b][ri][md][c]:
//   out[b][md][o] = sum_i R[md][o][i] in[b][md][i]            (adj = 0)
//   out[b][md][i] = sum_o conj(R[md][o][i]) in[b][md][o]      (adj = 1)
// A mode is W^2 weights against a batch of samples: a weight-streaming
// batch of matrix-vector products, so it runs on the FP32 pipes, not the
// tensor cores.  One warp per mode: R staged in shared memory with rows
// padded to W + 1 (transposed for adj, so that lane = output channel reads
// a row without bank conflicts), inputs of up to 4 samples staged beside it.
__host__ __device__ inline size_t mix_warp_floats(int W) {
    return (size_t)2 * W * (W + 1) + (size_t)8 * W;
}

__global__ void mix_kernel(const float *__restrict__ re, const float *__restrict__ im,
                           const float *__restrict__ in, float *__restrict__ out, int modes, int W,
                           int B, int adj) {
    extern __shared__ float mix_smem[];
    const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int WP = W + 1;
    float *Rr = mix_smem + (size_t)warp * mix_warp_floats(W);
    float *Ri = Rr + (size_t)W * WP;
    float *X = Ri + (size_t)W * WP;  // [4 samples][re, im][W]
    const size_t plane = (size_t)modes * W, WW = (size_t)W * W;
    for (int md = blockIdx.x * nw + warp; md < modes; md += gridDim.x * nw) {
        const float *pr = re + (size_t)md * WW, *pi = im + (size_t)md * WW;
        __syncwarp();
        // eight rows of 32 weights of each part in flight per lane at a time
        for (int t0 = 0; t0 < W * W; t0 += 256) {
            float vr[8], vi[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int t = t0 + 32 * u + lane;
                vr[u] = t < W * W ? __ldg(pr + t) : 0.f;
                vi[u] = t < W * W ? __ldg(pi + t) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int t = t0 + 32 * u + lane;
                if (t >= W * W) break;
                const int o = t / W, i = t - o * W;
                const int r = adj ? i : o, c = adj ? o : i;
                Rr[r * WP + c] = vr[u];
                Ri[r * WP + c] = adj ? -vi[u] : vi[u];
            }
        }
        for (int b0 = 0; b0 < B; b0 += 4) {
            const int nb = min(4, B - b0);
            __syncwarp();
            for (int t = lane; t < nb * 2 * W; t += 32) {
                const int bb = t / (2 * W), rem = t - bb * 2 * W, ri = rem / W, c = rem - ri * W;
                X[t] = __ldg(in + (size_t)(b0 + bb) * 2 * plane + ri * plane + (size_t)md * W + c);
            }
            __syncwarp();
            for (int o = lane; o < W; o += 32) {
                float ar[4] = {0.f, 0.f, 0.f, 0.f}, ai[4] = {0.f, 0.f, 0.f, 0.f};
                const float *rr = Rr + o * WP, *rm = Ri + o * WP;
                for (int i = 0; i < W; ++i) {
                    const float r = rr[i], m = rm[i];
#pragma unroll
                    for (int bb = 0; bb < 4; ++bb) {
                        const float xr = X[bb * 2 * W + i], xi = X[bb * 2 * W + W + i];
                        ar[bb] = fmaf(r, xr, fmaf(-m, xi, ar[bb]));
                        ai[bb] = fmaf(r, xi, fmaf(m, xr, ai[bb]));
                    }
                }
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    if (bb >= nb) break;
                    float *po = out + (size_t)(b0 + bb) * 2 * plane + (size_t)md * W + o;
                    po[0] = ar[bb];
                    po[plane] = ai[bb];
                }
            }
        }
    }
}

// The same for W a template parameter (W = 8, 16, 32) and at most 4 samples:
// a lane holds its W^2/32 weights of each part and its share of the inputs in
// registers, and loads the next mode's while the products of this one run,
// so that one mode's loads are in flight at any time instead of one row
// batch of them.
template <int WT>
__global__ void mix_kernel_w(const float *__restrict__ re, const float *__restrict__ im,
                             const float *__restrict__ in, float *__restrict__ out, int modes,
                             int B, int adj) {
    constexpr int W = WT, WP = W + 1, V = (W * W + 31) / 32, XV = (8 * W + 31) / 32;
    extern __shared__ float mix_smem[];
    const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *Rr = mix_smem + (size_t)warp * mix_warp_floats(W);
    float *Ri = Rr + W * WP;
    float *X = Ri + W * WP;  // [4 samples][re, im][W]
    const size_t plane = (size_t)modes * W;
    float vr[V], vi[V], xv[XV];
    auto load = [&](int md) {
        const float *pr = re + (size_t)md * W * W, *pi = im + (size_t)md * W * W;
#pragma unroll
        for (int u = 0; u < V; ++u) {
            const int t = lane + 32 * u;
            vr[u] = t < W * W ? __ldg(pr + t) : 0.f;
            vi[u] = t < W * W ? __ldg(pi + t) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < XV; ++u) {
            const int t = lane + 32 * u;
            const int bb = t / (2 * W), rem = t - bb * 2 * W, ri = rem / W, c = rem - ri * W;
            xv[u] = bb < B ? __ldg(in + (size_t)bb * 2 * plane + ri * plane + (size_t)md * W + c)
                           : 0.f;
        }
    };
    int md = blockIdx.x * nw + warp;
    if (md < modes) load(md);
    for (; md < modes; md += gridDim.x * nw) {
        __syncwarp();
#pragma unroll
        for (int u = 0; u < V; ++u) {
            const int t = lane + 32 * u;
            if (t < W * W) {
                const int o = t / W, i = t - o * W;
                const int r = adj ? i : o, c = adj ? o : i;
                Rr[r * WP + c] = vr[u];
                Ri[r * WP + c] = adj ? -vi[u] : vi[u];
            }
        }
#pragma unroll
        for (int u = 0; u < XV; ++u)
            if (lane + 32 * u < 8 * W) X[lane + 32 * u] = xv[u];
        __syncwarp();
        const int next = md + gridDim.x * nw;
        if (next < modes) load(next);
        for (int o = lane; o < W; o += 32) {
            float ar[4] = {0.f, 0.f, 0.f, 0.f}, ai[4] = {0.f, 0.f, 0.f, 0.f};
            const float *rr = Rr + o * WP, *rm = Ri + o * WP;
#pragma unroll 8
            for (int i = 0; i < W; ++i) {
                const float r = rr[i], m = rm[i];
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    const float xr = X[bb * 2 * W + i], xi = X[bb * 2 * W + W + i];
                    ar[bb] = fmaf(r, xr, fmaf(-m, xi, ar[bb]));
                    ai[bb] = fmaf(r, xi, fmaf(m, xr, ai[bb]));
                }
            }
#pragma unroll
            for (int bb = 0; bb < 4; ++bb) {
                if (bb >= B) break;
                float *po = out + (size_t)bb * 2 * plane + (size_t)md * W + o;
                po[0] = ar[bb];
                po[plane] = ai[bb];
            }
        }
    }
}

// Gradient of R from the mixing's output gradient dout and its input x
// (both Zh layout), added to gRe, gIm ([mode][out][in]):
//   gRe[o][i] += sum_b dout_re[o] x_re[i] + dout_im[o] x_im[i]
//   gIm[o][i] += sum_b dout_im[o] x_re[i] - dout_re[o] x_im[i]
// One warp per mode, both vectors of up to 4 samples staged in shared
// memory, lanes along i (coalesced read-modify-write of the gradient rows).
__global__ void mix_wgrad_kernel(const float *__restrict__ dout, const float *__restrict__ x,
                                 float *__restrict__ gre, float *__restrict__ gim, int modes,
                                 int W, int B) {
    extern __shared__ float mix_smem[];
    const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *D = mix_smem + (size_t)warp * 16 * W;  // [4][re, im][W]
    float *X = D + 8 * W;
    const size_t plane = (size_t)modes * W, WW = (size_t)W * W;
    for (int md = blockIdx.x * nw + warp; md < modes; md += gridDim.x * nw) {
        float *gr = gre + (size_t)md * WW, *gm = gim + (size_t)md * WW;
        for (int b0 = 0; b0 < B; b0 += 4) {
            const int nb = min(4, B - b0);
            __syncwarp();
            for (int t = lane; t < 8 * W; t += 32) {
                const int bb = t / (2 * W), rem = t - bb * 2 * W, ri = rem / W, c = rem - ri * W;
                const size_t o = (size_t)(b0 + bb) * 2 * plane + ri * plane + (size_t)md * W + c;
                D[t] = bb < nb ? __ldg(dout + o) : 0.f;
                X[t] = bb < nb ? __ldg(x + o) : 0.f;
            }
            __syncwarp();
            // the gradient rows read eight at a time per lane, then updated
            for (int t0 = 0; t0 < W * W; t0 += 256) {
                float og[8], om[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int t = t0 + 32 * u + lane;
                    og[u] = t < W * W ? gr[t] : 0.f;
                    om[u] = t < W * W ? gm[t] : 0.f;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int t = t0 + 32 * u + lane;
                    if (t >= W * W) break;
                    const int o = t / W, i = t - o * W;
                    float sr = 0.f, sm = 0.f;
#pragma unroll
                    for (int bb = 0; bb < 4; ++bb) {
                        const float dr = D[bb * 2 * W + o], di = D[bb * 2 * W + W + o];
                        const float xr = X[bb * 2 * W + i], xi = X[bb * 2 * W + W + i];
                        sr = fmaf(dr, xr, fmaf(di, xi, sr));
                        sm = fmaf(di, xr, fmaf(-dr, xi, sm));
                    }
                    gr[t] = og[u] + sr;
                    gm[t] = om[u] + sm;
                }
            }
        }
    }
}

// d *= gelu'(z)
__global__ void gelu_back_kernel(float *__restrict__ d, const float *__restrict__ z, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        d[i] *= gelu_grad(z[i]);
}
__device__ __forceinline__ float4 gelu_back4(float4 a, float4 b) {
    return make_float4(a.x * gelu_grad(b.x), a.y * gelu_grad(b.y), a.z * gelu_grad(b.z),
                       a.w * gelu_grad(b.w));
}
// the same on 16-byte vectors (both arrays 16-byte aligned, n4 = n / 4), two
// vectors a thread in flight per iteration; elementwise the same arithmetic
__global__ void gelu_back4_kernel(float4 *__restrict__ d, const float4 *__restrict__ z, size_t n4) {
    const size_t st = (size_t)gridDim.x * blockDim.x;
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    for (; i + st < n4; i += 2 * st) {
        const float4 a = d[i], b = d[i + st], za = z[i], zb = z[i + st];
        d[i] = gelu_back4(a, za);
        d[i + st] = gelu_back4(b, zb);
    }
    if (i < n4) d[i] = gelu_back4(d[i], z[i]);
}

// du = 2 (u - t) / n and the sum of squares (FP64), reduced over the block
// before one atomic addition per block (256 threads)
__global__ void mse_kernel(const float *__restrict__ u, const float *__restrict__ t,
                           float *__restrict__ du, size_t n, double *sum) {
    __shared__ double ws[8];
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float e = u[i] - t[i];
        du[i] = 2.f * e / (float)n;
        s += (double)e * (double)e;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < 8; ++w) b += ws[w];
        atomicAdd(sum, b);
    }
}

__device__ __forceinline__ void adam_one(float &p, float g, float &m, float &v, float lr, float b1,
                                         float b2, float eps, float c1, float c2) {
    m = b1 * m + (1.f - b1) * g;
    v = b2 * v + (1.f - b2) * g * g;
    p -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        float pi = p[i], mi = m[i], vi = v[i];
        adam_one(pi, g[i], mi, vi, lr, b1, b2, eps, c1, c2);
        m[i] = mi;
        v[i] = vi;
        p[i] = pi;
    }
}
// the same on 16-byte vectors (all four arrays 16-byte aligned): the first
// 4 (n / 4) parameters as vectors, the last n % 4 by the first thread
__global__ void adam4_kernel(float *__restrict__ p, const float *__restrict__ g,
                             float *__restrict__ m, float *__restrict__ v, size_t n, float lr,
                             float b1, float b2, float eps, float c1, float c2) {
    const size_t n4 = n / 4;
    float4 *p4 = reinterpret_cast<float4 *>(p), *m4 = reinterpret_cast<float4 *>(m),
           *v4 = reinterpret_cast<float4 *>(v);
    const float4 *g4 = reinterpret_cast<const float4 *>(g);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4;
         i += (size_t)gridDim.x * blockDim.x) {
        float4 pi = p4[i], mi = m4[i], vi = v4[i];
        const float4 gi = g4[i];
        adam_one(pi.x, gi.x, mi.x, vi.x, lr, b1, b2, eps, c1, c2);
        adam_one(pi.y, gi.y, mi.y, vi.y, lr, b1, b2, eps, c1, c2);
        adam_one(pi.z, gi.z, mi.z, vi.z, lr, b1, b2, eps, c1, c2);
        adam_one(pi.w, gi.w, mi.w, vi.w, lr, b1, b2, eps, c1, c2);
        m4[i] = mi;
        v4[i] = vi;
        p4[i] = pi;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (size_t i = 4 * n4; i < n; ++i) {
            float pi = p[i], mi = m[i], vi = v[i];
            adam_one(pi, g[i], mi, vi, lr, b1, b2, eps, c1, c2);
            m[i] = mi;
            v[i] = vi;
            p[i] = pi;
        }
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

bool aligned16(const void *a) { return ((uintptr_t)a & 15) == 0; }

// d *= gelu'(z) over n elements, on vectors where the layout allows
void gelu_back(float *d, const float *z, size_t n, cudaStream_t s) {
    if (n % 4 == 0 && aligned16(d) && aligned16(z))
        gelu_back4_kernel<<<grid_for(n / 8), 256, 0, s>>>(reinterpret_cast<float4 *>(d),
                                                         reinterpret_cast<const float4 *>(z), n / 4);
    else
        gelu_back_kernel<<<grid_for(n), 256, 0, s>>>(d, z, n);
}

}  // namespace

struct ehd_fno {
    ehd_fno_config c{};
    cudaStream_t stream = nullptr;
    int X = 0, Y = 0, Z = 0, W = 0, L = 0, mx = 0, my2 = 0, mz2 = 0, H = 0, cin = 0, cout = 0;
    int modes = 0;  // mz2 * my2 * mx
    size_t P = 0;   // voxels per sample
    size_t nparam = 0;
    size_t oP = 0, op = 0, oQ1 = 0, oq1 = 0, oQ2 = 0, oq2 = 0;
    std::vector<Off> lo;
    std::vector<void *> allocs;
    float *param = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16 *pbf = nullptr;                 // BF16 copy of every parameter
    __nv_bfloat16 *Fx = nullptr, *Fy = nullptr, *Fz = nullptr, *Gx = nullptr, *Gy = nullptr,
                  *Gz = nullptr;
    double *lsum = nullptr;
    // activations for max_batch samples
    std::vector<float *> v, z, zh;                // v[0..L], z[0..L-1], zh[0..L-1]
    float *xh = nullptr, *yh = nullptr, *mh = nullptr, *hpre = nullptr, *h = nullptr,
          *u = nullptr, *du = nullptr, *dh = nullptr, *dv = nullptr, *dv2 = nullptr;
    int adam_t = 0;
};

namespace {

int fail(const std::string &m) { return set_error(EHD_ERR_INVALID, m.c_str()); }
int cuda_fail(const char *what, cudaError_t e) {
    return set_error(EHD_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

template <typename T>
cudaError_t alloc(ehd_fno *f, T **p, size_t n) {
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) {
        f->allocs.push_back(*p);
        e = cudaMemsetAsync(*p, 0, std::max<size_t>(n, 1) * sizeof(T), f->stream);
    }
    return e;
}

struct Dev {
    int prev = -1;
    explicit Dev(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~Dev() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
double uniform(uint64_t seed, uint64_t i) {
    return (double)(mix64(seed * 0x100000001B3ull + i) >> 11) * (1.0 / 9007199254740992.0);
}

// wave number of kept mode j along an axis of n points with m modes per sign
int wave(int j, int m, int n) { return j < m ? j : n - 2 * m + j; }

// the DFT matrices (see the file comment), rounded to BF16
cudaError_t make_dft(ehd_fno *f) {
    const int X = f->X, Y = f->Y, Z = f->Z, mx = f->mx, my2 = f->my2, mz2 = f->mz2;
    const double tp = 2.0 * M_PI;
    auto up = [&](__nv_bfloat16 **dst, const std::vector<double> &h) -> cudaError_t {
        std::vector<__nv_bfloat16> b(h.size());
        for (size_t i = 0; i < h.size(); ++i) b[i] = __float2bfloat16_rn((float)h[i]);
        cudaError_t e = alloc(f, dst, h.size());
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*dst, b.data(), b.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
    };
    // Fx [2mx][X]
    std::vector<double> fx(2 * (size_t)mx * X), gx((size_t)X * 2 * mx);
    const double norm = 1.0 / ((double)X * Y * Z);
    for (int k = 0; k < mx; ++k)
        for (int x = 0; x < X; ++x) {
            const double th = tp * (double)k * x / X;
            fx[(size_t)k * X + x] = std::cos(th);
            fx[(size_t)(mx + k) * X + x] = -std::sin(th);
            const double w = (k == 0 ? 1.0 : 2.0) * norm;
            gx[(size_t)x * 2 * mx + k] = w * std::cos(th);
            gx[(size_t)x * 2 * mx + mx + k] = -w * std::sin(th);
        }
    // complex forward [2 M][2 N] and inverse [2 N][2 M] for an axis of n points
    auto cplx = [&](int n, int m2, std::vector<double> &fw, std::vector<double> &iv) {
        fw.assign(4 * (size_t)m2 * n, 0.0);
        iv.assign(4 * (size_t)m2 * n, 0.0);
        for (int j = 0; j < m2; ++j)
            for (int i = 0; i < n; ++i) {
                const double th = tp * (double)wave(j, m2 / 2, n) * i / n;
                const double cs = std::cos(th), sn = std::sin(th);
                // forward, rows (ro, j), cols (ri, i): e^{-i th}
                fw[(size_t)j * 2 * n + i] = cs;
                fw[(size_t)j * 2 * n + n + i] = sn;
                fw[(size_t)(m2 + j) * 2 * n + i] = -sn;
                fw[(size_t)(m2 + j) * 2 * n + n + i] = cs;
                // inverse, rows (ro, i), cols (ri, j): e^{+i th}
                iv[(size_t)i * 2 * m2 + j] = cs;
                iv[(size_t)i * 2 * m2 + m2 + j] = -sn;
                iv[(size_t)(n + i) * 2 * m2 + j] = sn;
                iv[(size_t)(n + i) * 2 * m2 + m2 + j] = cs;
            }
    };
    std::vector<double> fy, gy, fz, gz;
    cplx(Y, my2, fy, gy);
    cplx(Z, mz2, fz, gz);
    cudaError_t e;
    if ((e = up(&f->Fx, fx)) != cudaSuccess || (e = up(&f->Gx, gx)) != cudaSuccess ||
        (e = up(&f->Fy, fy)) != cudaSuccess || (e = up(&f->Gy, gy)) != cudaSuccess ||
        (e = up(&f->Fz, fz)) != cudaSuccess || (e = up(&f->Gz, gz)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

// BF16 copies of the parameters the products read: every parameter but the
// spectral weights, which the mode mixing reads in FP32.
cudaError_t refresh(ehd_fno *f) {
    const size_t spec = (size_t)f->modes * f->W * f->W;
    size_t from = 0;
    for (int l = 0; l <= f->L; ++l) {
        const size_t to = l < f->L ? f->lo[l].Rre : f->nparam;
        if (to > from)
            cast_bf16_kernel<<<grid_for(to - from), 256, 0, f->stream>>>(f->param + from,
                                                                         f->pbf + from, to - from);
        if (l < f->L) from = f->lo[l].Rim + spec;
    }
    return cudaGetLastError();
}

// ---- products -----------------------------------------------------------------

// C[rows][n] (+)= A[rows][k] Bw[k][n] (+ bias), channels-last pointwise layer
GemmArgs pointwise(size_t rows, int K, int N, const float *A, const __nv_bfloat16 *Bw,
                   float *C, const float *bias, float *C2) {
    GemmArgs g;
    g.M = (int)rows;
    g.N = N;
    g.K = K;
    g.A = A;
    g.am = lin(K);
    g.ak = lin(1);
    g.B = Bw;
    g.b_bf16 = 1;
    g.bk = lin(N);
    g.bn = lin(1);
    g.C = C;
    g.cm = lin(N);
    g.cn = lin(1);
    g.bias = bias;
    g.C2 = C2;
    g.a_n = (long long)rows * K;
    g.b_n = (long long)K * N;
    g.c_n = (long long)rows * N;
    return g;
}

// D_in[rows][K] = D[rows][N] Bw^T (Bw stored [K][N])
GemmArgs input_grad(size_t rows, int K, int N, const float *D, const __nv_bfloat16 *Bw,
                    float *Din, float beta) {
    GemmArgs g;
    g.M = (int)rows;
    g.N = K;
    g.K = N;
    g.A = D;
    g.am = lin(N);
    g.ak = lin(1);
    g.B = Bw;
    g.b_bf16 = 1;
    g.bk = lin(1);
    g.bn = lin(N);
    g.C = Din;
    g.cm = lin(K);
    g.cn = lin(1);
    g.beta = beta;
    g.a_n = (long long)rows * N;
    g.b_n = (long long)K * N;
    g.c_n = (long long)rows * K;
    return g;
}

struct Dims {
    long long X, Y, Z, W, mx, my2, mz2, Mo, B;
    long long nv() const { return B * Z * Y * X * W; }           // v[b][z][y][x][c]
    long long nxh() const { return B * Z * 2 * Y * mx * W; }     // Xh
    long long nyh() const { return B * 2 * Z * my2 * mx * W; }   // Yh
    long long nzh() const { return B * 2 * Mo * W; }             // Zh
};

// the eight products of one spectral convolution (forward), and their
// adjoints; `tr` selects the transposed DFT matrix
GemmArgs x_fwd(const Dims &d, const __nv_bfloat16 *Fx, const float *v, float *xh, bool adj_of_inv) {
    // xh[q][(ri,kx)][(y,c)] = Fx[(ri,kx)][x] v[q][(y,x,c)] over q = (b, z), the
    // columns n = (y, c); adj_of_inv: Gx^T instead of Fx
    GemmArgs g;
    g.M = (int)(2 * d.mx);
    g.K = (int)d.X;
    g.N = (int)(d.Y * d.W);
    g.batch = (int)(d.B * d.Z);
    g.A = Fx;
    g.a_bf16 = 1;
    if (adj_of_inv) {  // Gx is [X][2mx]
        g.am = lin(1);
        g.ak = lin(2 * d.mx);
    } else {
        g.am = lin(d.X);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = v;
    g.bk = lin(d.W);
    g.bn = two(1, (int)d.W, d.X * d.W);
    g.bbat = lin(d.Y * d.X * d.W);
    g.C = xh;
    g.cm = two(d.W, (int)d.mx, d.Y * d.mx * d.W);
    g.cn = two(1, (int)d.W, d.mx * d.W);
    g.cbat = lin(2 * d.Y * d.mx * d.W);
    g.a_n = 2 * d.mx * d.X;
    g.b_n = d.nv();
    g.c_n = d.nxh();
    return g;
}

GemmArgs x_inv(const Dims &d, const __nv_bfloat16 *Gx, const float *xh, float *v, float beta,
               bool adj_of_fwd) {
    // v[q][(y,x,c)] (+)= Gx[x][(ri,kx)] xh[q][(ri,kx)][(y,c)] over q = (b, z), the
    // columns n = (y, c); adj_of_fwd: Fx^T
    GemmArgs g;
    g.M = (int)d.X;
    g.K = (int)(2 * d.mx);
    g.N = (int)(d.Y * d.W);
    g.batch = (int)(d.B * d.Z);
    g.A = Gx;
    g.a_bf16 = 1;
    if (adj_of_fwd) {  // Fx is [2mx][X]
        g.am = lin(1);
        g.ak = lin(d.X);
    } else {
        g.am = lin(2 * d.mx);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = xh;
    g.bk = two(d.W, (int)d.mx, d.Y * d.mx * d.W);
    g.bn = two(1, (int)d.W, d.mx * d.W);
    g.bbat = lin(2 * d.Y * d.mx * d.W);
    g.C = v;
    g.cm = lin(d.W);
    g.cn = two(1, (int)d.W, d.X * d.W);
    g.cbat = lin(d.Y * d.X * d.W);
    g.beta = beta;
    g.a_n = 2 * d.mx * d.X;
    g.b_n = d.nxh();
    g.c_n = d.nv();
    return g;
}

GemmArgs y_fwd(const Dims &d, const __nv_bfloat16 *F, const float *xh, float *yh, bool adj) {
    // yh[b][(ri,j)][z][kx,c] = Fy[(ri,j)][(ri',y)] xh[b][z][(ri',y)][kx,c]; adj: Gy^T
    GemmArgs g;
    g.M = (int)(2 * d.my2);
    g.K = (int)(2 * d.Y);
    g.N = (int)(d.mx * d.W);
    g.batch = (int)(d.B * d.Z);
    g.A = F;
    g.a_bf16 = 1;
    if (adj) {  // Gy is [2Y][2my2]
        g.am = lin(1);
        g.ak = lin(2 * d.my2);
    } else {
        g.am = lin(2 * d.Y);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = xh;
    g.bk = lin(d.mx * d.W);
    g.bn = lin(1);
    g.bbat = lin(2 * d.Y * d.mx * d.W);
    g.C = yh;
    g.cm = two(d.mx * d.W, (int)d.my2, d.Z * d.my2 * d.mx * d.W);
    g.cn = lin(1);
    g.cbat = two(d.my2 * d.mx * d.W, (int)d.Z, 2 * d.Z * d.my2 * d.mx * d.W);
    g.a_n = 4 * d.my2 * d.Y;
    g.b_n = d.nxh();
    g.c_n = d.nyh();
    return g;
}

GemmArgs y_inv(const Dims &d, const __nv_bfloat16 *G, const float *yh, float *xh, bool adj) {
    // xh[b][z][(ri,y)][kx,c] = Gy[(ri,y)][(ri',j)] yh[b][(ri',j)][z][kx,c]; adj: Fy^T
    GemmArgs g;
    g.M = (int)(2 * d.Y);
    g.K = (int)(2 * d.my2);
    g.N = (int)(d.mx * d.W);
    g.batch = (int)(d.B * d.Z);
    g.A = G;
    g.a_bf16 = 1;
    if (adj) {  // Fy is [2my2][2Y]
        g.am = lin(1);
        g.ak = lin(2 * d.Y);
    } else {
        g.am = lin(2 * d.my2);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = yh;
    g.bk = two(d.mx * d.W, (int)d.my2, d.Z * d.my2 * d.mx * d.W);
    g.bn = lin(1);
    g.bbat = two(d.my2 * d.mx * d.W, (int)d.Z, 2 * d.Z * d.my2 * d.mx * d.W);
    g.C = xh;
    g.cm = lin(d.mx * d.W);
    g.cn = lin(1);
    g.cbat = lin(2 * d.Y * d.mx * d.W);
    g.a_n = 4 * d.my2 * d.Y;
    g.b_n = d.nyh();
    g.c_n = d.nxh();
    return g;
}

GemmArgs z_fwd(const Dims &d, const __nv_bfloat16 *F, const float *yh, float *zh, bool adj) {
    // zh[b][(ri,kz)][ky,kx,c] = Fz[(ri,kz)][(ri',z)] yh[b][(ri',z)][ky,kx,c]; adj: Gz^T
    GemmArgs g;
    g.M = (int)(2 * d.mz2);
    g.K = (int)(2 * d.Z);
    g.N = (int)(d.my2 * d.mx * d.W);
    g.batch = (int)d.B;
    g.A = F;
    g.a_bf16 = 1;
    if (adj) {  // Gz is [2Z][2mz2]
        g.am = lin(1);
        g.ak = lin(2 * d.mz2);
    } else {
        g.am = lin(2 * d.Z);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = yh;
    g.bk = lin(d.my2 * d.mx * d.W);
    g.bn = lin(1);
    g.bbat = lin(2 * d.Z * d.my2 * d.mx * d.W);
    g.C = zh;
    g.cm = lin(d.my2 * d.mx * d.W);
    g.cn = lin(1);
    g.cbat = lin(2 * d.Mo * d.W);
    g.a_n = 4 * d.mz2 * d.Z;
    g.b_n = d.nyh();
    g.c_n = d.nzh();
    return g;
}

GemmArgs z_inv(const Dims &d, const __nv_bfloat16 *G, const float *zh, float *yh, bool adj) {
    // yh[b][(ri,z)][ky,kx,c] = Gz[(ri,z)][(ri',kz)] zh[b][(ri',kz)][ky,kx,c]; adj: Fz^T
    GemmArgs g;
    g.M = (int)(2 * d.Z);
    g.K = (int)(2 * d.mz2);
    g.N = (int)(d.my2 * d.mx * d.W);
    g.batch = (int)d.B;
    g.A = G;
    g.a_bf16 = 1;
    if (adj) {  // Fz is [2mz2][2Z]
        g.am = lin(1);
        g.ak = lin(2 * d.Z);
    } else {
        g.am = lin(2 * d.mz2);
        g.ak = lin(1);
    }
    g.abat = lin(0);
    g.B = zh;
    g.bk = lin(d.my2 * d.mx * d.W);
    g.bn = lin(1);
    g.bbat = lin(2 * d.Mo * d.W);
    g.C = yh;
    g.cm = lin(d.my2 * d.mx * d.W);
    g.cn = lin(1);
    g.cbat = lin(2 * d.Z * d.my2 * d.mx * d.W);
    g.a_n = 4 * d.mz2 * d.Z;
    g.b_n = d.nzh();
    g.c_n = d.nyh();
    return g;
}

// launches of the mixing kernels: warps per block by the shared memory a
// warp needs (at most 48 KB a block)
int mix_warps(int W, size_t per_warp_floats) {
    const size_t per = per_warp_floats * sizeof(float);
    return (int)std::max<size_t>(1, std::min<size_t>(8, (48u << 10) / per));
}

cudaError_t mix(const ehd_fno *f, int l, const float *in, float *out, int B, bool adj) {
    const int nw = mix_warps(f->W, mix_warp_floats(f->W));
    const unsigned blocks = (unsigned)std::min<size_t>((f->modes + nw - 1) / nw, 148 * 16);
    const size_t sm = nw * mix_warp_floats(f->W) * sizeof(float);
    const float *re = f->param + f->lo[l].Rre, *im = f->param + f->lo[l].Rim;
    const int a = adj ? 1 : 0;
    if (B <= 4 && (f->W == 8 || f->W == 16 || f->W == 32)) {
        if (f->W == 8) mix_kernel_w<8><<<blocks, 32 * nw, sm, f->stream>>>(re, im, in, out, f->modes, B, a);
        else if (f->W == 16) mix_kernel_w<16><<<blocks, 32 * nw, sm, f->stream>>>(re, im, in, out, f->modes, B, a);
        else mix_kernel_w<32><<<blocks, 32 * nw, sm, f->stream>>>(re, im, in, out, f->modes, B, a);
    } else {
        mix_kernel<<<blocks, 32 * nw, sm, f->stream>>>(re, im, in, out, f->modes, f->W, B, a);
    }
    return cudaGetLastError();
}

cudaError_t mix_wgrad(const ehd_fno *f, int l, const float *dout, const float *x, float *g, int B) {
    const int nw = mix_warps(f->W, (size_t)16 * f->W);
    const unsigned blocks = (unsigned)std::min<size_t>((f->modes + nw - 1) / nw, 148 * 16);
    mix_wgrad_kernel<<<blocks, 32 * nw, (size_t)nw * 16 * f->W * sizeof(float), f->stream>>>(
        dout, x, g + f->lo[l].Rre, g + f->lo[l].Rim, f->modes, f->W, B);
    return cudaGetLastError();
}

Dims dims(const ehd_fno *f, int B) {
    return Dims{f->X, f->Y, f->Z, f->W, f->mx, f->my2, f->mz2, f->modes, B};
}

#define FNO_CK(call)                                      \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(#call, e_); \
    } while (0)

int forward(ehd_fno *f, int B, const float *a) {
    const Dims d = dims(f, B);
    const size_t rows = (size_t)B * f->P;
    const __nv_bfloat16 *pb = f->pbf;
    cudaStream_t s = f->stream;
    FNO_CK(gemm(pointwise(rows, f->cin, f->W, a, pb + f->oP, f->v[0], f->param + f->op, nullptr), s));
    for (int l = 0; l < f->L; ++l) {
        const bool last = l == f->L - 1;
        float *zl = f->z[l];
        FNO_CK(gemm(pointwise(rows, f->W, f->W, f->v[l], pb + f->lo[l].W, zl, f->param + f->lo[l].b,
                              nullptr), s));
        FNO_CK(gemm(x_fwd(d, f->Fx, f->v[l], f->xh, false), s));
        FNO_CK(gemm(y_fwd(d, f->Fy, f->xh, f->yh, false), s));
        FNO_CK(gemm(z_fwd(d, f->Fz, f->yh, f->zh[l], false), s));
        FNO_CK(mix(f, l, f->zh[l], f->mh, B, false));
        FNO_CK(gemm(z_inv(d, f->Gz, f->mh, f->yh, false), s));
        FNO_CK(gemm(y_inv(d, f->Gy, f->yh, f->xh, false), s));
        GemmArgs g = x_inv(d, f->Gx, f->xh, zl, 1.f, false);
        g.C2 = last ? nullptr : f->v[l + 1];
        FNO_CK(gemm(g, s));
    }
    const float *vL = f->z[f->L - 1];
    FNO_CK(gemm(pointwise(rows, f->W, f->H, vL, pb + f->oQ1, f->hpre, f->param + f->oq1, f->h), s));
    FNO_CK(gemm(pointwise(rows, f->H, f->cout, f->h, pb + f->oQ2, f->u, f->param + f->oq2, nullptr),
                s));
    return EHD_OK;
}

int check_batch(const ehd_fno *f, int B) {
    if (B < 1 || B > f->c.max_batch) return fail("ehd_fno: batch outside 1..max_batch");
    return EHD_OK;
}

}  // namespace

extern "C" {

int ehd_fno_create(const ehd_fno_config *cfg, ehd_fno **out) {
    if (!cfg || !out) return fail("ehd_fno_create: NULL argument");
    *out = nullptr;
    const ehd_fno_config &c = *cfg;
    for (int r : c.reserved)
        if (r != 0) return fail("ehd_fno_create: reserved fields must be 0");
    if (c.nx < 2 || c.ny < 2 || c.nz < 2 || c.in_channels < 1 || c.out_channels < 1 ||
        c.width < 1 || c.layers < 1 || c.hidden < 1 || c.max_batch < 1)
        return fail("ehd_fno_create: sizes must be positive");
    if (c.modes_x < 1 || c.modes_x > c.nx / 2 - (c.nx % 2 == 0 ? 1 : 0) || c.modes_y < 1 ||
        2 * c.modes_y > c.ny || c.modes_z < 1 || 2 * c.modes_z > c.nz)
        return fail("ehd_fno_create: modes exceed the grid (modes_x < nx/2, 2 modes_y <= ny, "
                    "2 modes_z <= nz)");
    Dev dg(c.device);
    ehd_fno *f = new ehd_fno();
    f->c = c;
    f->X = c.nx;
    f->Y = c.ny;
    f->Z = c.nz;
    f->W = c.width;
    f->L = c.layers;
    f->mx = c.modes_x;
    f->my2 = 2 * c.modes_y;
    f->mz2 = 2 * c.modes_z;
    f->H = c.hidden;
    f->cin = c.in_channels;
    f->cout = c.out_channels;
    f->modes = f->mz2 * f->my2 * f->mx;
    f->P = (size_t)f->X * f->Y * f->Z;
    auto bail = [&](int code) {
        ehd_fno_destroy(f);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail("ehd_fno_create stream", e));
    // parameter layout
    size_t n = 0;
    const size_t W = f->W, H = f->H, WW = W * W, RM = (size_t)f->modes * WW;
    f->oP = n;
    n += (size_t)f->cin * W;
    f->op = n;
    n += W;
    for (int l = 0; l < f->L; ++l) {
        Off o{};
        o.W = n;
        n += WW;
        o.b = n;
        n += W;
        o.Rre = n;
        n += RM;
        o.Rim = n;
        n += RM;
        f->lo.push_back(o);
    }
    f->oQ1 = n;
    n += W * H;
    f->oq1 = n;
    n += H;
    f->oQ2 = n;
    n += H * f->cout;
    f->oq2 = n;
    n += f->cout;
    f->nparam = n;
    // initial values: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for the pointwise
    // layers and their biases, U(0, 1) / (W W) for both parts of R
    std::vector<float> h(n, 0.f);
    uint64_t ctr = 0;
    auto fill = [&](size_t off, size_t cnt, double lo, double hi) {
        for (size_t i = 0; i < cnt; ++i) h[off + i] = (float)(lo + (hi - lo) * uniform(c.seed, ctr++));
    };
    auto dense = [&](size_t off, size_t fan_in, size_t cnt) {
        const double b = 1.0 / std::sqrt((double)fan_in);
        fill(off, cnt, -b, b);
    };
    dense(f->oP, f->cin, (size_t)f->cin * W);
    dense(f->op, f->cin, W);
    for (int l = 0; l < f->L; ++l) {
        dense(f->lo[l].W, W, WW);
        dense(f->lo[l].b, W, W);
        fill(f->lo[l].Rre, RM, 0.0, 1.0 / (double)WW);
        fill(f->lo[l].Rim, RM, 0.0, 1.0 / (double)WW);
    }
    dense(f->oQ1, W, W * H);
    dense(f->oq1, W, H);
    dense(f->oQ2, H, H * f->cout);
    dense(f->oq2, H, f->cout);
    // buffers
    const size_t B = c.max_batch, rows = B * f->P;
    const size_t nxh = B * f->Z * 2 * f->Y * f->mx * W;
    const size_t nyh = B * 2 * f->Z * f->my2 * f->mx * W;
    const size_t nzh = B * 2 * (size_t)f->modes * W;
    if ((e = alloc(f, &f->param, n)) != cudaSuccess || (e = alloc(f, &f->grad, n)) != cudaSuccess ||
        (e = alloc(f, &f->adam_m, n)) != cudaSuccess || (e = alloc(f, &f->adam_v, n)) != cudaSuccess ||
        (e = alloc(f, &f->pbf, n)) != cudaSuccess ||
        (e = alloc(f, &f->lsum, 1)) != cudaSuccess ||
        (e = alloc(f, &f->xh, nxh)) != cudaSuccess || (e = alloc(f, &f->yh, nyh)) != cudaSuccess ||
        (e = alloc(f, &f->mh, nzh)) != cudaSuccess || (e = alloc(f, &f->hpre, rows * H)) != cudaSuccess ||
        (e = alloc(f, &f->h, rows * H)) != cudaSuccess ||
        (e = alloc(f, &f->u, rows * f->cout)) != cudaSuccess ||
        (e = alloc(f, &f->du, rows * f->cout)) != cudaSuccess ||
        (e = alloc(f, &f->dh, rows * H)) != cudaSuccess || (e = alloc(f, &f->dv, rows * W)) != cudaSuccess ||
        (e = alloc(f, &f->dv2, rows * W)) != cudaSuccess)
        return bail(cuda_fail("ehd_fno_create allocation", e));
    f->v.assign(f->L + 1, nullptr);
    f->z.assign(f->L, nullptr);
    f->zh.assign(f->L, nullptr);
    for (int l = 0; l < f->L; ++l) {
        if ((e = alloc(f, &f->z[l], rows * W)) != cudaSuccess ||
            (e = alloc(f, &f->zh[l], nzh)) != cudaSuccess)
            return bail(cuda_fail("ehd_fno_create allocation", e));
    }
    for (int l = 0; l < f->L; ++l)  // v[L] is z[L-1] (no activation after the last layer)
        if ((e = alloc(f, &f->v[l], rows * W)) != cudaSuccess)
            return bail(cuda_fail("ehd_fno_create allocation", e));
    f->v[f->L] = f->z[f->L - 1];
    if ((e = cudaMemcpy(f->param, h.data(), n * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = make_dft(f)) != cudaSuccess || (e = refresh(f)) != cudaSuccess ||
        (e = cudaStreamSynchronize(f->stream)) != cudaSuccess)
        return bail(cuda_fail("ehd_fno_create set-up", e));
    *out = f;
    return EHD_OK;
}

int ehd_fno_destroy(ehd_fno *f) {
    if (!f) return EHD_OK;
    Dev dg(f->c.device);
    if (f->stream) cudaStreamSynchronize(f->stream);
    for (void *p : f->allocs) cudaFree(p);
    if (f->stream) cudaStreamDestroy(f->stream);
    delete f;
    return EHD_OK;
}

int ehd_fno_param_count(const ehd_fno *f, int64_t *count) {
    if (!f || !count) return fail("ehd_fno_param_count: NULL argument");
    *count = (int64_t)f->nparam;
    return EHD_OK;
}

int ehd_fno_get_params(ehd_fno *f, float *host) {
    if (!f || !host) return fail("ehd_fno_get_params: NULL argument");
    Dev dg(f->c.device);
    FNO_CK(cudaMemcpyAsync(host, f->param, f->nparam * sizeof(float), cudaMemcpyDeviceToHost,
                           f->stream));
    FNO_CK(cudaStreamSynchronize(f->stream));
    return EHD_OK;
}

int ehd_fno_set_params(ehd_fno *f, const float *host) {
    if (!f || !host) return fail("ehd_fno_set_params: NULL argument");
    Dev dg(f->c.device);
    FNO_CK(cudaMemcpyAsync(f->param, host, f->nparam * sizeof(float), cudaMemcpyHostToDevice,
                           f->stream));
    FNO_CK(refresh(f));
    FNO_CK(cudaStreamSynchronize(f->stream));
    return EHD_OK;
}

int ehd_fno_get_grads(ehd_fno *f, float *host) {
    if (!f || !host) return fail("ehd_fno_get_grads: NULL argument");
    Dev dg(f->c.device);
    FNO_CK(cudaMemcpyAsync(host, f->grad, f->nparam * sizeof(float), cudaMemcpyDeviceToHost,
                           f->stream));
    FNO_CK(cudaStreamSynchronize(f->stream));
    return EHD_OK;
}

int ehd_fno_forward(ehd_fno *f, int B, const float *a, float *u) {
    if (!f || !a || !u) return fail("ehd_fno_forward: NULL argument");
    if (int r = check_batch(f, B)) return r;
    Dev dg(f->c.device);
    if (int r = forward(f, B, a)) return r;
    FNO_CK(cudaMemcpyAsync(u, f->u, (size_t)B * f->P * f->cout * sizeof(float),
                           cudaMemcpyDeviceToDevice, f->stream));
    return EHD_OK;
}

int ehd_fno_backward(ehd_fno *f, int B, const float *a, const float *target, double *loss) {
    if (!f || !a || !target) return fail("ehd_fno_backward: NULL argument");
    if (int r = check_batch(f, B)) return r;
    Dev dg(f->c.device);
    cudaStream_t s = f->stream;
    if (int r = forward(f, B, a)) return r;
    const Dims d = dims(f, B);
    const size_t rows = (size_t)B * f->P;
    const size_t nout = rows * f->cout;
    float *g = f->grad;
    const __nv_bfloat16 *pb = f->pbf;
    FNO_CK(cudaMemsetAsync(g, 0, f->nparam * sizeof(float), s));
    FNO_CK(cudaMemsetAsync(f->lsum, 0, sizeof(double), s));
    mse_kernel<<<grid_for(nout), 256, 0, s>>>(f->u, target, f->du, nout, f->lsum);
    FNO_CK(cudaGetLastError());
    // projection
    FNO_CK(weight_bias_grad((long long)rows, f->H, f->cout, f->h, f->H, f->du, f->cout,
                            g + f->oQ2, f->cout, g + f->oq2, s));
    FNO_CK(gemm(input_grad(rows, f->H, f->cout, f->du, pb + f->oQ2, f->dh, 0.f), s));
    gelu_back(f->dh, f->hpre, rows * f->H, s);
    FNO_CK(cudaGetLastError());
    const float *vL = f->z[f->L - 1];
    FNO_CK(weight_bias_grad((long long)rows, f->W, f->H, vL, f->W, f->dh, f->H, g + f->oQ1, f->H,
                            g + f->oq1, s));
    FNO_CK(gemm(input_grad(rows, f->W, f->H, f->dh, pb + f->oQ1, f->dv, 0.f), s));
    // Fourier layers: f->dv holds the gradient of v[l+1]
    for (int l = f->L - 1; l >= 0; --l) {
        float *dz = f->dv;  // gradient of the pre-activation, in place
        if (l != f->L - 1) {
            gelu_back(dz, f->z[l], rows * f->W, s);
            FNO_CK(cudaGetLastError());
        }
        const Off &o = f->lo[l];
        FNO_CK(weight_bias_grad((long long)rows, f->W, f->W, f->v[l], f->W, dz, f->W, g + o.W,
                                f->W, g + o.b, s));
        FNO_CK(gemm(input_grad(rows, f->W, f->W, dz, pb + o.W, f->dv2, 0.f), s));
        // adjoint of the spectral convolution
        FNO_CK(gemm(x_fwd(d, f->Gx, dz, f->xh, true), s));
        FNO_CK(gemm(y_fwd(d, f->Gy, f->xh, f->yh, true), s));
        FNO_CK(gemm(z_fwd(d, f->Gz, f->yh, f->mh, true), s));
        FNO_CK(mix_wgrad(f, l, f->mh, f->zh[l], g, B));
        FNO_CK(mix(f, l, f->mh, f->zh[l], B, true));  // zh[l] is free now
        FNO_CK(gemm(z_inv(d, f->Fz, f->zh[l], f->yh, true), s));
        FNO_CK(gemm(y_inv(d, f->Fy, f->yh, f->xh, true), s));
        FNO_CK(gemm(x_inv(d, f->Fx, f->xh, f->dv2, 1.f, true), s));
        std::swap(f->dv, f->dv2);
    }
    // lift
    FNO_CK(weight_bias_grad((long long)rows, f->cin, f->W, a, f->cin, f->dv, f->W, g + f->oP, f->W,
                            g + f->op, s));
    if (loss) {
        double sum = 0.0;
        FNO_CK(cudaMemcpyAsync(&sum, f->lsum, sizeof(double), cudaMemcpyDeviceToHost, s));
        FNO_CK(cudaStreamSynchronize(s));
        *loss = sum / (double)nout;
    }
    return EHD_OK;
}

int ehd_fno_adam_step(ehd_fno *f, float lr, float b1, float b2, float eps) {
    if (!f || !(lr > 0) || !(b1 >= 0 && b1 < 1) || !(b2 >= 0 && b2 < 1) || !(eps > 0))
        return fail("ehd_fno_adam_step: bad arguments");
    Dev dg(f->c.device);
    f->adam_t += 1;
    const float c1 = 1.f - std::pow(b1, (float)f->adam_t), c2 = 1.f - std::pow(b2, (float)f->adam_t);
    if (aligned16(f->param) && aligned16(f->grad) && aligned16(f->adam_m) && aligned16(f->adam_v))
        adam4_kernel<<<grid_for(f->nparam / 4 + 1), 256, 0, f->stream>>>(
            f->param, f->grad, f->adam_m, f->adam_v, f->nparam, lr, b1, b2, eps, c1, c2);
    else
        adam_kernel<<<grid_for(f->nparam), 256, 0, f->stream>>>(
            f->param, f->grad, f->adam_m, f->adam_v, f->nparam, lr, b1, b2, eps, c1, c2);
    FNO_CK(cudaGetLastError());
    FNO_CK(refresh(f));
    return EHD_OK;
}

int ehd_fno_synchronize(ehd_fno *f) {
    if (!f) return fail("ehd_fno_synchronize: NULL argument");
    Dev dg(f->c.device);
    FNO_CK(cudaStreamSynchronize(f->stream));
    return EHD_OK;
}

int ehd_bf16_gemm(int M, int N, int K, int batch, const float *A, int64_t a_row, int64_t a_col,
                  int64_t ab, const float *B, int64_t b_row, int64_t b_col, int64_t bb, float *C,
                  int64_t c_row, int64_t c_col, int64_t cb, float alpha, float beta,
                  void *stream) {
    if (!A || !B || !C || M < 1 || N < 1 || K < 1 || batch < 1)
        return fail("ehd_bf16_gemm: bad arguments");
    GemmArgs g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.batch = batch;
    g.A = A;
    g.am = lin(a_row);
    g.ak = lin(a_col);
    g.abat = lin(ab);
    g.B = B;
    g.bk = lin(b_row);
    g.bn = lin(b_col);
    g.bbat = lin(bb);
    g.C = C;
    g.cm = lin(c_row);
    g.cn = lin(c_col);
    g.cbat = lin(cb);
    g.alpha = alpha;
    g.beta = beta;
    // the caller's arrays are taken to span exactly the largest offsets
    // (negative strides are rejected by gemm())
    auto span = [](long long n0, long long s0, long long n1, long long s1, long long n2,
                   long long s2) {
        return (n0 - 1) * std::max<long long>(s0, 0) + (n1 - 1) * std::max<long long>(s1, 0) +
               (n2 - 1) * std::max<long long>(s2, 0) + 1;
    };
    g.a_n = span(M, a_row, K, a_col, batch, ab);
    g.b_n = span(K, b_row, N, b_col, batch, bb);
    g.c_n = span(M, c_row, N, c_col, batch, cb);
    cudaError_t e = gemm(g, (cudaStream_t)stream);
    return e == cudaSuccess ? EHD_OK : cuda_fail("ehd_bf16_gemm", e);
}

}  // extern "C"
