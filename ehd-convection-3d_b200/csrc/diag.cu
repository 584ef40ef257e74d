// diag.cu -- scalar diagnostics reduced on the device in FP64.
//
// The reference copies q and Ez to the host every 1000 steps and loops there
// (current, LBM.cu:1647-1671; record_umax, LBM.cu:1673-1713).  Here one
// deterministic two-stage reduction (fixed block partition, fixed tree order)
// produces, in FP64:
//   [0] sum_xy q(NZ-1) Ez(NZ-1) with q(NZ-1) = 2 q(NZ-2) - q(NZ-3) and
//       Ez(NZ-1) = Ez(NZ-2) (the current before the factor K dy^2)
//   [1] sum rho |u|^2      [2] sum q
//   [3] max uz with uz(NZ-1) extrapolated like record_umax, floor 0
//   [4] count of non-finite rho, u, v, w, q
#include <math.h>

#include "common.cuh"
#include "kernels.h"

namespace ehd {

namespace {
constexpr int kDiagThreads = 256;
constexpr int kNQ = 5;

__device__ __forceinline__ void block_reduce(double (&v)[kNQ], double *sm) {
    // sm: kNQ * (kDiagThreads / 32)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < kNQ; ++k) {
            const double t = __shfl_xor_sync(0xffffffffu, v[k], o);
            v[k] = (k == 3) ? fmax(v[k], t) : v[k] + t;
        }
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < kNQ; ++k) sm[k * (kDiagThreads / 32) + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < kNQ; ++k)
            v[k] = lane < kDiagThreads / 32 ? sm[k * (kDiagThreads / 32) + lane]
                                            : (k == 3 ? 0.0 : 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int k = 0; k < kNQ; ++k) {
                const double t = __shfl_xor_sync(0xffffffffu, v[k], o);
                v[k] = (k == 3) ? fmax(v[k], t) : v[k] + t;
            }
        }
    }
}
}  // namespace

template <typename R>
__global__ void __launch_bounds__(kDiagThreads)
diag_stage1(const R *__restrict__ rho, const R *__restrict__ u, const R *__restrict__ v,
            const R *__restrict__ w, const R *__restrict__ q, const R *__restrict__ phip,
            const double *__restrict__ ez00, const double *__restrict__ ez, double inv2dz,
            int nx, int ny, int nz, double *__restrict__ partial) {
    __shared__ double sm[kNQ * (kDiagThreads / 32)];
    const long long nxy = (long long)nx * ny;
    const long long n = nxy * nz;
    const long long chunk = (n + gridDim.x - 1) / gridDim.x;
    const long long beg = chunk * blockIdx.x;
    const long long end = beg + chunk < n ? beg + chunk : n;
    double acc[kNQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (long long i = beg + threadIdx.x; i < end; i += kDiagThreads) {
        const double r = rho[i], uu = u[i], vv = v[i], ww = w[i], qq = q[i];
        acc[1] += r * (uu * uu + vv * vv + ww * ww);
        acc[2] += qq;
        if (!isfinite(r) || !isfinite(uu) || !isfinite(vv) || !isfinite(ww) || !isfinite(qq))
            acc[4] += 1.0;
        const long long z = i / nxy;
        double uz = ww;
        if (z == nz - 1) {
            const long long p = i - (z * nxy);
            uz = 2.0 * (double)w[(nz - 2) * nxy + p] - (double)w[(nz - 3) * nxy + p];
            const double qt = 2.0 * (double)q[(nz - 2) * nxy + p] - (double)q[(nz - 3) * nxy + p];
            double e;
            if (ez != nullptr) {
                e = ez[i];
            } else {
                // Ez(NZ-1) = Ez(NZ-2) = (phi(NZ-3) - phi(NZ-1)) / (2 dz), phi'(NZ-1) = 0
                e = ez00[nz - 2] + (double)phip[(nz - 3) * nxy + p] * inv2dz;
            }
            acc[0] += qt * e;
        }
        acc[3] = fmax(acc[3], uz);
    }
    block_reduce(acc, sm);
    if (threadIdx.x == 0)
        for (int k = 0; k < kNQ; ++k) partial[(size_t)blockIdx.x * kNQ + k] = acc[k];
}

__global__ void __launch_bounds__(kDiagThreads)
diag_stage2(const double *__restrict__ partial, int nblocks, double *__restrict__ result) {
    __shared__ double sm[kNQ * (kDiagThreads / 32)];
    double acc[kNQ] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += kDiagThreads)
        for (int k = 0; k < kNQ; ++k)
            acc[k] = (k == 3) ? fmax(acc[k], partial[(size_t)b * kNQ + k])
                              : acc[k] + partial[(size_t)b * kNQ + k];
    block_reduce(acc, sm);
    if (threadIdx.x == 0)
        for (int k = 0; k < kNQ; ++k) result[k] = acc[k];
}

template <typename R>
cudaError_t launch_diag(const DiagArgs &a, cudaStream_t s) {
    diag_stage1<R><<<a.nblocks, kDiagThreads, 0, s>>>(
        (const R *)a.rho, (const R *)a.u, (const R *)a.v, (const R *)a.w, (const R *)a.q,
        (const R *)a.phip, a.ez00, a.ez, a.inv2dz, a.nx, a.ny, a.nz, a.partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    diag_stage2<<<1, kDiagThreads, 0, s>>>(a.partial, a.nblocks, a.result);
    return cudaGetLastError();
}

template cudaError_t launch_diag<float>(const DiagArgs &, cudaStream_t);
template cudaError_t launch_diag<double>(const DiagArgs &, cudaStream_t);

// The current alone ([0] above) from the collector plane: q(NZ-2), q(NZ-3)
// and phi'(NZ-3) of one plane instead of the whole field, the same per-node
// term, a fixed partition of the plane into blocks and a fixed tree order.
namespace {
__device__ __forceinline__ double block_sum(double v, double *sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < kDiagThreads / 32 ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}
}  // namespace

template <typename R>
__global__ void __launch_bounds__(kDiagThreads)
current_stage1(const R *__restrict__ q, const R *__restrict__ phip,
               const double *__restrict__ ez00, const double *__restrict__ ez, double inv2dz,
               int nxy, int nz, double *__restrict__ partial) {
    __shared__ double sm[kDiagThreads / 32];
    const int chunk = (nxy + gridDim.x - 1) / gridDim.x;
    const int beg = chunk * blockIdx.x;
    const int end = beg + chunk < nxy ? beg + chunk : nxy;
    const size_t top = (size_t)(nz - 1) * nxy;
    double acc = 0.0;
    for (int p = beg + threadIdx.x; p < end; p += kDiagThreads) {
        const double qt = 2.0 * (double)q[(size_t)(nz - 2) * nxy + p] - (double)q[(size_t)(nz - 3) * nxy + p];
        const double e = ez != nullptr ? ez[top + p]
                                       : ez00[nz - 2] + (double)phip[(size_t)(nz - 3) * nxy + p] * inv2dz;
        acc += qt * e;
    }
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kDiagThreads)
current_stage2(const double *__restrict__ partial, int nblocks, double *__restrict__ result) {
    __shared__ double sm[kDiagThreads / 32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kDiagThreads) acc += partial[b];
    acc = block_sum(acc, sm);
    if (threadIdx.x == 0) result[0] = acc;
}

template <typename R>
cudaError_t launch_current(const DiagArgs &a, cudaStream_t s) {
    const int nxy = a.nx * a.ny;
    int nb = (nxy + 4 * kDiagThreads - 1) / (4 * kDiagThreads);
    nb = nb < 1 ? 1 : (nb > a.nblocks ? a.nblocks : nb);
    current_stage1<R><<<nb, kDiagThreads, 0, s>>>((const R *)a.q, (const R *)a.phip, a.ez00, a.ez,
                                                  a.inv2dz, nxy, a.nz, a.partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    current_stage2<<<1, kDiagThreads, 0, s>>>(a.partial, nb, a.result);
    return cudaGetLastError();
}
template cudaError_t launch_current<float>(const DiagArgs &, cudaStream_t);
template cudaError_t launch_current<double>(const DiagArgs &, cudaStream_t);

}  // namespace ehd
