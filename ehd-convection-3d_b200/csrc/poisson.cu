// poisson.cu -- Poisson solve for the potential and its mean-field E.
//
// The reference (main.cu:190-206, poisson.cu:78-167) odd-extends the source
// s = -q/eps in z to NE = 2(NZ-1) planes (odd_extension), runs a complex 3D
// FFT of NX x NY x NE points in FP64 (cuFFT Z2Z), divides each mode by
// mu = kx^2 + ky^2 + (4/dz^2) sin^2(kz dz/2) (gpu_derivative), transforms back
// and keeps the real part (odd_extract).  The odd extension makes the z part a
// DST-I, which diagonalises exactly the 3-point Dirichlet Laplacian with
// eigenvalues (4/dz^2) sin^2(kz dz/2).  This file solves the same discrete
// problem without the doubled, complex z transform:
//
//   K1 rows_fwd : per x-row, s = -q/eps, complex FFT along x in shared memory,
//                 keep kx = 0..NX/2 (real input); FP64 row sums of s.
//   K2 cols     : per plane, FFT along y of tiles of kx columns; the block of
//                 the first tile also reduces the FP64 row sums to the plane
//                 sum.  Output in FP64.
//   K3 zsolve   : per (kx, ky), the tridiagonal system
//                 phi(z-1) - (2 + k^2 dz^2) phi(z) + phi(z+1) = dz^2 s(z),
//                 phi(0) = phi(NZ-1) = 0, by the Thomas algorithm in FP64.
//                 The electrode voltage enters as -V/dz^2 on the plane z = 1
//                 (poisson.cu:97), i.e. only in the (0,0) mode, whose FP64
//                 solution is the mean potential phi00(z) (plus V at z = 0);
//                 the (0,0) mode of the fluctuation is zeroed.
//   K2 cols     : inverse FFT along y, output in the compute type.
//   K4 rows_inv : per x-row, Hermitian completion, inverse FFT along x,
//                 phi' = Re / (NX NY).
//
// phi = phi00(z) + phi'(x,y,z).  E = -grad(phi) is not stored: the step kernel
// takes central differences of phi' and adds ez00(z), the mean-field Ez.
//
// FFTs are radix-2/3/4/5 Stockham autosort passes in shared memory (any
// NX, NY of the form 2^a 3^b 5^c), twiddles from an FP64-accurate table.
#include "common.cuh"
#include "kernels.h"

namespace ehd {

namespace {

template <typename R2> __device__ __forceinline__ R2 cadd(R2 a, R2 b) { return {a.x + b.x, a.y + b.y}; }
template <typename R2> __device__ __forceinline__ R2 csub(R2 a, R2 b) { return {a.x - b.x, a.y - b.y}; }
template <typename R2> __device__ __forceinline__ R2 cmul(R2 a, R2 b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// i * s * a for s = +-1
template <typename R2, typename R> __device__ __forceinline__ R2 cis(R2 a, R s) {
    return {-s * a.y, s * a.x};
}
template <typename R2, typename R> __device__ __forceinline__ R2 cscale(R2 a, R s) {
    return {a.x * s, a.y * s};
}

// One batch of `batch` length-N transforms held contiguously in `a`; `b` is
// scratch of the same size.  Returns the buffer holding the result.  sign -1
// forward (exp(-2 pi i jk/N)), +1 inverse, unnormalised.
template <typename R>
__device__ typename Cplx<R>::T *fft_smem(typename Cplx<R>::T *a, typename Cplx<R>::T *b,
                                         const FftPlan &pl,
                                         const typename Cplx<R>::T *__restrict__ tw, R sign,
                                         int batch) {
    using R2 = typename Cplx<R>::T;
    const int N = pl.n;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nthr = blockDim.x * blockDim.y;
    int Ns = 1;
    for (int s = 0; s < pl.nrad; ++s) {
        const int Rr = pl.rad[s];
        const int nb = N / Rr;
        const int tstep = N / (Ns * Rr);
        const int total = batch * nb;
        for (int t = tid; t < total; t += nthr) {
            const int line = t / nb;
            const int j = t - line * nb;
            const int k = j % Ns;
            const R2 *in = a + (size_t)line * N;
            R2 *out = b + (size_t)line * N;
            const int base = (j / Ns) * Ns * Rr + k;
            R2 v[5];
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                if (r < Rr) {
                    R2 x = in[j + r * nb];
                    if (r > 0 && k > 0) {
                        R2 w = __ldg(tw + r * k * tstep);
                        w.y *= -sign;  // table holds exp(-2 pi i m/N): conjugate for inverse
                        x = cmul(x, w);
                    }
                    v[r] = x;
                }
            }
            if (Rr == 2) {
                out[base] = cadd(v[0], v[1]);
                out[base + Ns] = csub(v[0], v[1]);
            } else if (Rr == 4) {
                const R2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
                const R2 s13 = cadd(v[1], v[3]), d13 = cis(csub(v[1], v[3]), sign);
                out[base] = cadd(s02, s13);
                out[base + Ns] = cadd(d02, d13);
                out[base + 2 * Ns] = csub(s02, s13);
                out[base + 3 * Ns] = csub(d02, d13);
            } else if (Rr == 3) {
                const R h3 = (R)0.86602540378443864676;  // sqrt(3)/2
                const R2 t1 = cadd(v[1], v[2]);
                const R2 t2 = csub(v[0], cscale(t1, (R)0.5));
                const R2 t3 = cis(cscale(csub(v[1], v[2]), h3), sign);
                out[base] = cadd(v[0], t1);
                out[base + Ns] = cadd(t2, t3);
                out[base + 2 * Ns] = csub(t2, t3);
            } else {  // 5
                const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
                const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
                const R2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
                const R2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
                const R2 a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
                const R2 a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
                const R2 b1 = cis(cadd(cscale(t3, s1), cscale(t4, s2)), sign);
                const R2 b2 = cis(csub(cscale(t3, s2), cscale(t4, s1)), sign);
                out[base] = cadd(v[0], cadd(t1, t2));
                out[base + Ns] = cadd(a1, b1);
                out[base + 4 * Ns] = csub(a1, b1);
                out[base + 2 * Ns] = cadd(a2, b2);
                out[base + 3 * Ns] = csub(a2, b2);
            }
        }
        __syncthreads();
        R2 *t = a;
        a = b;
        b = t;
        Ns *= Rr;
    }
    return a;
}

template <typename R2> __device__ __forceinline__ R2 to_c(double2 v);
template <> __device__ __forceinline__ float2 to_c<float2>(double2 v) {
    return make_float2((float)v.x, (float)v.y);
}
template <> __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d(double2 v) { return v; }

}  // namespace

// K1: s = -q/eps on the planes z = 1..NZ-2 (odd_extension's interior rows,
// poisson.cu:96-106), FFT along x, half spectrum out; FP64 row sums.
template <typename R>
__global__ void __launch_bounds__(256)
poisson_rows_fwd(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spec,
                 double *__restrict__ rowsum, const typename Cplx<R>::T *__restrict__ tw,
                 FftPlan pl, int nx, int ny, int nxh, int pitch, int rows, double eps) {
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)rows * nx;
    const int zi = blockIdx.y;  // plane z = zi + 1
    const int y0 = blockIdx.x * rows;
    const int tid = threadIdx.x;
    const R *qp = q + (size_t)nx * ny * (zi + 1);
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, x = t - r * nx;
        const int y = y0 + r;
        R val = 0;
        if (y < ny) val = -qp[(size_t)nx * y + x] / (R)eps;
        a[t] = R2{val, (R)0};
    }
    // FP64 row sums: one warp per row, fixed order
    const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < rows; r += nwarps) {
        const int y = y0 + r;
        if (y >= ny) continue;
        double s = 0.0;
        for (int x = lane; x < nx; x += 32) s += -(double)qp[(size_t)nx * y + x] / eps;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) rowsum[(size_t)zi * ny + y] = s;
    }
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tw, (R)-1, rows);
    R2 *sp = spec + (size_t)zi * ny * pitch;
    for (int t = tid; t < rows * nxh; t += blockDim.x) {
        const int r = t / nxh, k = t - r * nxh;
        const int y = y0 + r;
        if (y < ny) sp[(size_t)pitch * y + k] = res[(size_t)r * nx + k];
    }
}

// K2: FFT along y of `cols` kx columns of one plane.  Forward: compute-type
// spectrum in, FP64 out, plus the FP64 plane sum.  Inverse: FP64 in,
// compute type out.
template <typename R, typename SrcT, typename DstT>
__global__ void __launch_bounds__(256)
poisson_cols(const SrcT *__restrict__ src, DstT *__restrict__ dst,
             const typename Cplx<R>::T *__restrict__ tw, FftPlan pl, int ny, int nxh,
             int pitch, int cols, R sign, const double *__restrict__ rowsum,
             double *__restrict__ planesum) {
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)cols * ny;
    const int zi = blockIdx.y;
    const int k0 = blockIdx.x * cols;
    const int tid = threadIdx.x;
    const size_t off = (size_t)zi * ny * pitch;
    for (int t = tid; t < ny * cols; t += blockDim.x) {
        const int y = t / cols, cidx = t - y * cols;
        const int k = k0 + cidx;
        R2 v = R2{(R)0, (R)0};
        if (k < nxh) v = to_c<R2>(to_d(src[off + (size_t)pitch * y + k]));
        a[(size_t)cidx * ny + y] = v;
    }
    if (planesum != nullptr && blockIdx.x == 0 && tid < 32) {
        double s = 0.0;
        for (int y = tid; y < ny; y += 32) s += rowsum[(size_t)zi * ny + y];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (tid == 0) planesum[zi + 1] = s;
    }
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tw, sign, cols);
    for (int t = tid; t < ny * cols; t += blockDim.x) {
        const int y = t / cols, cidx = t - y * cols;
        const int k = k0 + cidx;
        if (k < nxh) {
            const R2 v = res[(size_t)cidx * ny + y];
            DstT o;
            o.x = v.x;
            o.y = v.y;
            dst[off + (size_t)pitch * y + k] = o;
        }
    }
}

// K3: Thomas algorithm per (kx, ky) mode in FP64, in place on specd.
__global__ void poisson_zsolve(double2 *__restrict__ specd, const double *__restrict__ kx2,
                               const double *__restrict__ ky2,
                               const double *__restrict__ planesum,
                               double *__restrict__ phi00, double *__restrict__ ez00, int nx,
                               int ny, int nz, int nxh, int pitch, double dz, double voltage) {
    extern __shared__ double cps[];  // [z][thread]
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const long long m = (long long)blockIdx.x * nthr + tid;
    const int n = nz - 2;  // unknowns z = 1..nz-2
    if (m >= (long long)nxh * ny) return;
    const int ky = (int)(m / nxh), kx = (int)(m - (long long)ky * nxh);
    const size_t plane = (size_t)ny * pitch;
    const size_t off = (size_t)pitch * ky + kx;
    const double dz2 = dz * dz;
    if (kx == 0 && ky == 0) {
        // mean mode: planesum (FP64) plus the Dirichlet lift -V/dz^2 on z = 1,
        // unnormalised like the forward DFT (times NX*NY).
        const double nxy = (double)nx * (double)ny;
        double cp_prev = 0.0, dp_prev = 0.0;
        for (int i = 0; i < n; ++i) {
            double d = planesum[i + 1];
            if (i == 0) d += -voltage / dz2 * nxy;
            d *= dz2;
            const double cp = 1.0 / (-2.0 - cp_prev);
            const double dp = (d - dp_prev) * cp;
            cps[(size_t)i * nthr + tid] = cp;
            specd[(size_t)i * plane + off] = make_double2(dp, 0.0);
            cp_prev = cp;
            dp_prev = dp;
        }
        double xn = 0.0;
        const double norm = 1.0 / nxy;
        phi00[nz - 1] = 0.0;
        phi00[0] = voltage;
        for (int i = n - 1; i >= 0; --i) {
            const double dp = specd[(size_t)i * plane + off].x;
            const double xi = dp - cps[(size_t)i * nthr + tid] * xn;
            phi00[i + 1] = xi * norm;
            specd[(size_t)i * plane + off] = make_double2(0.0, 0.0);
            xn = xi;
        }
        for (int z = 1; z <= nz - 2; ++z) ez00[z] = 0.5 * (phi00[z - 1] - phi00[z + 1]) / dz;
        ez00[0] = ez00[1];
        ez00[nz - 1] = ez00[nz - 2];
        return;
    }
    const double beta = 2.0 + (kx2[kx] + ky2[ky]) * dz2;
    double cp_prev = 0.0, dpr = 0.0, dpi = 0.0;
    for (int i = 0; i < n; ++i) {
        const double2 s = specd[(size_t)i * plane + off];
        const double cp = 1.0 / (-beta - cp_prev);
        dpr = (s.x * dz2 - dpr) * cp;
        dpi = (s.y * dz2 - dpi) * cp;
        cps[(size_t)i * nthr + tid] = cp;
        specd[(size_t)i * plane + off] = make_double2(dpr, dpi);
        cp_prev = cp;
    }
    double xr = 0.0, xi = 0.0;
    for (int i = n - 1; i >= 0; --i) {
        const double2 dp = specd[(size_t)i * plane + off];
        const double cp = cps[(size_t)i * nthr + tid];
        xr = dp.x - cp * xr;
        xi = dp.y - cp * xi;
        specd[(size_t)i * plane + off] = make_double2(xr, xi);
    }
}

// K4: Hermitian completion, inverse FFT along x, phi' = Re/(NX NY)
// (odd_extract, poisson.cu:154-167, for the interior planes).
template <typename R>
__global__ void __launch_bounds__(256)
poisson_rows_inv(const typename Cplx<R>::T *__restrict__ spec, R *__restrict__ phip,
                 const typename Cplx<R>::T *__restrict__ tw, FftPlan pl, int nx, int ny,
                 int nxh, int pitch, int rows) {
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)rows * nx;
    const int zi = blockIdx.y;
    const int y0 = blockIdx.x * rows;
    const int tid = threadIdx.x;
    const R2 *sp = spec + (size_t)zi * ny * pitch;
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, k = t - r * nx;
        const int y = y0 + r;
        R2 v = R2{(R)0, (R)0};
        if (y < ny) {
            if (k < nxh) {
                v = sp[(size_t)pitch * y + k];
            } else {
                v = sp[(size_t)pitch * y + (nx - k)];
                v.y = -v.y;
            }
        }
        a[t] = v;
    }
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tw, (R)1, rows);
    const R norm = (R)(1.0 / ((double)nx * (double)ny));
    R *pp = phip + (size_t)nx * ny * (zi + 1);
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, x = t - r * nx;
        const int y = y0 + r;
        if (y < ny) pp[(size_t)nx * y + x] = res[t].x * norm;
    }
}

size_t poisson_zsolve_smem(int nz, int threads) {
    return (size_t)(nz > 2 ? nz - 2 : 1) * threads * sizeof(double);
}

// Opt in to more than 48 KB of dynamic shared memory.  Skipped while the
// stream is being captured into a graph: the attribute is set by the first,
// uncaptured launch on the device.
template <typename K>
static cudaError_t set_smem(K kern, size_t bytes, cudaStream_t s) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &st);
    if (e != cudaSuccess) return e;
    if (st != cudaStreamCaptureStatusNone) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename R>
cudaError_t launch_poisson(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    cudaError_t e;
    const int nzi = a.nz - 2;
    const int rows = a.rows_per_block, cols = a.cols_per_block;
    // K1
    {
        const size_t sm = (size_t)2 * rows * a.nx * sizeof(R2);
        if ((e = set_smem(poisson_rows_fwd<R>, sm, s)) != cudaSuccess) return e;
        dim3 grid((a.ny + rows - 1) / rows, nzi);
        poisson_rows_fwd<R><<<grid, 256, sm, s>>>((const R *)a.q, (R2 *)a.spec, a.rowsum,
                                                   (const R2 *)a.twx, a.px, a.nx, a.ny, a.nxh,
                                                   a.pitch, rows, a.eps);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // K2 forward
    {
        const size_t sm = (size_t)2 * cols * a.ny * sizeof(R2);
        auto kf = poisson_cols<R, R2, double2>;
        if ((e = set_smem(kf, sm, s)) != cudaSuccess) return e;
        dim3 grid((a.nxh + cols - 1) / cols, nzi);
        kf<<<grid, 256, sm, s>>>((const R2 *)a.spec, a.specd, (const R2 *)a.twy, a.py, a.ny,
                                 a.nxh, a.pitch, cols, (R)-1, a.rowsum, a.planesum);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // K3
    {
        const int thr = 64;
        const size_t sm = poisson_zsolve_smem(a.nz, thr);
        if ((e = set_smem(poisson_zsolve, sm, s)) != cudaSuccess) return e;
        const long long modes = (long long)a.nxh * a.ny;
        poisson_zsolve<<<(unsigned)((modes + thr - 1) / thr), thr, sm, s>>>(
            a.specd, a.kx2, a.ky2, a.planesum, a.phi00, a.ez00, a.nx, a.ny, a.nz, a.nxh,
            a.pitch, a.dz, a.voltage);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // K2 inverse
    {
        const size_t sm = (size_t)2 * cols * a.ny * sizeof(R2);
        auto ki = poisson_cols<R, double2, R2>;
        if ((e = set_smem(ki, sm, s)) != cudaSuccess) return e;
        dim3 grid((a.nxh + cols - 1) / cols, nzi);
        ki<<<grid, 256, sm, s>>>(a.specd, (R2 *)a.spec, (const R2 *)a.twy, a.py, a.ny, a.nxh,
                                 a.pitch, cols, (R)1, nullptr, nullptr);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // K4
    {
        const size_t sm = (size_t)2 * rows * a.nx * sizeof(R2);
        if ((e = set_smem(poisson_rows_inv<R>, sm, s)) != cudaSuccess) return e;
        dim3 grid((a.ny + rows - 1) / rows, nzi);
        poisson_rows_inv<R><<<grid, 256, sm, s>>>((const R2 *)a.spec, (R *)a.phip,
                                                   (const R2 *)a.twx, a.px, a.nx, a.ny, a.nxh,
                                                   a.pitch, rows);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template cudaError_t launch_poisson<float>(const PoissonArgs &, cudaStream_t);
template cudaError_t launch_poisson<double>(const PoissonArgs &, cudaStream_t);

}  // namespace ehd
