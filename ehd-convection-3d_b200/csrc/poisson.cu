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
//   K1 rows_fwd : per x-row, s' = -(q - q_m(z))/eps (q_m: the plane's reference
//                 charge, taken out so the FP32 transform carries only the
//                 fluctuation), FFT along x, keep kx = 0..NX/2 (real input);
//                 FP64 row sums of s'.
//   K2 cols     : per plane, FFT along y of tiles of kx columns, in place; the
//                 block of the first tile reduces the FP64 row sums to the
//                 plane sum.
//   K3 zsolve   : per (kx, ky) != (0,0), the tridiagonal system
//                 phi(z-1) - (2 + k^2 dz^2) phi(z) + phi(z+1) = dz^2 s(z),
//                 phi(0) = phi(NZ-1) = 0, by the Thomas algorithm in FP64
//                 (pivots from a table built once per context, the forward
//                 sweep in an FP64 scratch), in place.  The (0,0) mode in
//                 FP64 from the plane sums plus NX NY q_m, with the electrode
//                 voltage entering as -V/dz^2 on the plane z = 1
//                 (poisson.cu:97): the mean potential phi00(z) (V at z = 0)
//                 and its Ez; the (0,0) mode of the fluctuation is 0.
//   K2 cols     : inverse FFT along y.
//   K4 rows_inv : per x-row, Hermitian completion, inverse FFT along x,
//                 phi' = Re / (NX NY).
//
// phi = phi00(z) + phi'(x,y,z).  E = -grad(phi) is not stored: the step kernel
// takes central differences of phi' and adds ez00(z), the mean-field Ez.
//
// FFTs: for N = 64, 128, 256, 512 the x and y transforms use compile-time
// Stockham passes of radix 8/16 (fft.cuh), two real x-rows packed into one
// complex transform; other sizes use run-time passes of radix 2/3/4/5 and,
// for any other prime factor p, a direct radix-p pass over symmetric pairs
// of outputs.  Twiddles come from an FP64-accurate table.
#include <cmath>

#include "common.cuh"
#include "fft.cuh"
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
// scratch of the same size; `tw` the table exp(-2 pi i m/N), m < N (in shared
// memory).  Returns the buffer holding the result.  sign -1 forward
// (exp(-2 pi i jk/N)), +1 inverse, unnormalised.
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
        if (Rr > 5) {
            // Odd prime radix p: the inputs are twiddled in place first, then
            // each work item forms one pair of outputs (q, p - q) from the
            // symmetric sums s_r = x_r + x_{p-r} and differences
            // d_r = x_r - x_{p-r}:  out_q = A + i sign B, out_{p-q} = A - i sign B,
            // A = x_0 + sum_r s_r cos(2 pi r q / p), B = sum_r d_r sin(2 pi r q / p),
            // r = 1..(p-1)/2; item q = 0 forms the plain sum.
            for (int t = tid; t < batch * N; t += nthr) {
                const int line = t / N, e = t - line * N;
                const int r = e / nb, j = e - r * nb;
                const int k = j % Ns;
                if (r > 0 && k > 0) {
                    R2 w = tw[r * k * tstep];
                    w.y *= -sign;
                    a[t] = cmul(a[t], w);
                }
            }
            __syncthreads();
            const int h = Rr / 2;
            const int per = nb * (h + 1);
            const int pstep = N / Rr;  // table index of exp(-2 pi i / p)
            for (int t = tid; t < batch * per; t += nthr) {
                const int line = t / per, rem = t - line * per;
                const int j = rem / (h + 1), qq = rem - j * (h + 1);
                const int k = j % Ns;
                const R2 *in = a + (size_t)line * N;
                R2 *out = b + (size_t)line * N;
                const int base = (j / Ns) * Ns * Rr + k;
                const R2 x0 = in[j];
                if (qq == 0) {
                    R2 sum = x0;
                    for (int r = 1; r < Rr; ++r) sum = cadd(sum, in[j + r * nb]);
                    out[base] = sum;
                } else {
                    R2 A = x0, B = R2{(R)0, (R)0};
                    int m = qq;  // r qq mod p
                    for (int r = 1; r <= h; ++r) {
                        const R2 xr = in[j + r * nb], xm = in[j + (Rr - r) * nb];
                        const R2 w = tw[m * pstep];  // (cos, -sin) of 2 pi m / p
                        A.x += (xr.x + xm.x) * w.x;
                        A.y += (xr.y + xm.y) * w.x;
                        B.x -= (xr.x - xm.x) * w.y;
                        B.y -= (xr.y - xm.y) * w.y;
                        m += qq;
                        if (m >= Rr) m -= Rr;
                    }
                    const R2 iB = cis(B, sign);
                    out[base + qq * Ns] = cadd(A, iB);
                    out[base + (Rr - qq) * Ns] = csub(A, iB);
                }
            }
            __syncthreads();
            R2 *tsw = a;
            a = b;
            b = tsw;
            Ns *= Rr;
            continue;
        }
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
                        R2 w = tw[r * k * tstep];
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

}  // namespace

// ---------------------------------------------------------------------------
// run-time radix kernels (any size)
// ---------------------------------------------------------------------------

// K1: s' = -(q - q_m)/eps on the planes z = 1..NZ-2 (odd_extension's interior
// rows, poisson.cu:96-106), FFT along x of two real rows per complex
// transform, half spectrum out; FP64 row sums.
template <typename R>
__global__ void __launch_bounds__(256)
poisson_rows_fwd(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spec,
                 double *__restrict__ rowsum, const typename Cplx<R>::T *__restrict__ tw,
                 const double *__restrict__ qmean, FftPlan pl, int nx, int ny, int nxh, int pitch,
                 int rows, double eps,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        q = (const R *)gp.q;
        spec = (typename Cplx<R>::T *)gp.spec;
        rowsum = (double *)gp.rowsum;
        qmean = (const double *)gp.qmean;
    }
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)rows * nx;
    R2 *tws = b + (size_t)rows * nx;
    const int zi = blockIdx.y;  // plane z = zi + 1
    const int y0 = blockIdx.x * 2 * rows;  // transform r holds rows y0 + 2r, + 1
    const int tid = threadIdx.x;
    for (int i = tid; i < nx; i += blockDim.x) tws[i] = tw[i];
    const R *qp = q + (size_t)nx * ny * (zi + 1);
    const R qm = (R)qmean[2 * (zi + 1) + 1];
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, x = t - r * nx;
        const int ya = y0 + 2 * r, yb = ya + 1;
        R va = 0, vb = 0;
        if (ya < ny) va = -(qp[(size_t)nx * ya + x] - qm) / (R)eps;
        if (yb < ny) vb = -(qp[(size_t)nx * yb + x] - qm) / (R)eps;
        a[t] = R2{va, vb};
    }
    const int warp = tid >> 5, lane = tid & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < 2 * rows; r += nwarps) {
        const int y = y0 + r;
        if (y >= ny) continue;
        double sum = 0.0;
        for (int x = lane; x < nx; x += 32) sum += (double)qp[(size_t)nx * y + x] - (double)qm;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) rowsum[(size_t)zi * ny + y] = -sum / eps;
    }
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tws, (R)-1, rows);
    // two real rows per transform: A[k] = (Z[k] + conj Z[N-k]) / 2,
    // B[k] = (Z[k] - conj Z[N-k]) / (2i)
    R2 *sp = spec + (size_t)zi * ny * pitch;
    for (int t = tid; t < rows * nxh; t += blockDim.x) {
        const int r = t / nxh, k = t - r * nxh;
        const int ya = y0 + 2 * r, yb = ya + 1;
        const R2 zk = res[(size_t)r * nx + k];
        const R2 zn = res[(size_t)r * nx + (k == 0 ? 0 : nx - k)];
        if (ya < ny) sp[(size_t)pitch * ya + k] = R2{(R)0.5 * (zk.x + zn.x), (R)0.5 * (zk.y - zn.y)};
        if (yb < ny) sp[(size_t)pitch * yb + k] = R2{(R)0.5 * (zk.y + zn.y), (R)0.5 * (zn.x - zk.x)};
    }
}

// FP64 plane sum of the row sums, fixed order (one warp).
__device__ __forceinline__ void plane_sum_warp(const double *__restrict__ rowsum,
                                               double *__restrict__ planesum, int zi, int ny) {
    const int lane = threadIdx.x & 31;
    double sum = 0.0;
    for (int y = lane; y < ny; y += 32) sum += rowsum[(size_t)zi * ny + y];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) planesum[zi + 1] = sum;
}

// K2: FFT along y of `cols` kx columns of one plane, in place; the forward
// pass also reduces the FP64 plane sum.
template <typename R>
__global__ void __launch_bounds__(256)
poisson_cols(typename Cplx<R>::T *__restrict__ spec, const typename Cplx<R>::T *__restrict__ tw,
             FftPlan pl, int ny, int nxh, int pitch, int cols, R sign,
             const double *__restrict__ rowsum, double *__restrict__ planesum,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        if (rowsum) rowsum = (const double *)gp.rowsum;
        if (planesum) planesum = (double *)gp.planesum;
    }
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)cols * ny;
    R2 *tws = b + (size_t)cols * ny;
    const int zi = blockIdx.y;
    const int k0 = blockIdx.x * cols;
    const int tid = threadIdx.x;
    for (int i = tid; i < ny; i += blockDim.x) tws[i] = tw[i];
    const size_t off = (size_t)zi * ny * pitch;
    for (int t = tid; t < ny * cols; t += blockDim.x) {
        const int y = t / cols, cidx = t - y * cols;
        const int k = k0 + cidx;
        R2 v = R2{(R)0, (R)0};
        if (k < nxh) v = spec[off + (size_t)pitch * y + k];
        a[(size_t)cidx * ny + y] = v;
    }
    if (planesum != nullptr && blockIdx.x == 0 && tid < 32) plane_sum_warp(rowsum, planesum, zi, ny);
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tws, sign, cols);
    for (int t = tid; t < ny * cols; t += blockDim.x) {
        const int y = t / cols, cidx = t - y * cols;
        const int k = k0 + cidx;
        if (k < nxh) spec[off + (size_t)pitch * y + k] = res[(size_t)cidx * ny + y];
    }
}

// K4: Hermitian completion, inverse FFT along x, phi' = Re/(NX NY)
// (odd_extract, poisson.cu:154-167, for the interior planes).
template <typename R>
__global__ void __launch_bounds__(256)
poisson_rows_inv(const typename Cplx<R>::T *__restrict__ spec, R *__restrict__ phip,
                 const typename Cplx<R>::T *__restrict__ tw, FftPlan pl, int nx, int ny,
                 int nxh, int pitch, int rows,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (const typename Cplx<R>::T *)gp.spec;
        phip = (R *)gp.phip;
    }
    using R2 = typename Cplx<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)rows * nx;
    R2 *tws = b + (size_t)rows * nx;
    const int zi = blockIdx.y;
    const int y0 = blockIdx.x * 2 * rows;  // transform r holds rows y0 + 2r, + 1
    const int tid = threadIdx.x;
    for (int i = tid; i < nx; i += blockDim.x) tws[i] = tw[i];
    const R2 *sp = spec + (size_t)zi * ny * pitch;
    // Z = A + i B over the full length, A and B the Hermitian-completed rows;
    // the imaginary parts of the bins 0 and N/2, which a real row ignores,
    // are dropped so that they do not leak into the other row
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, k = t - r * nx;
        const int ya = y0 + 2 * r, yb = ya + 1;
        const int kk = k < nxh ? k : nx - k;
        R2 A = ya < ny ? sp[(size_t)pitch * ya + kk] : R2{(R)0, (R)0};
        R2 B = yb < ny ? sp[(size_t)pitch * yb + kk] : R2{(R)0, (R)0};
        if (kk == 0 || 2 * kk == nx) {
            A.y = 0;
            B.y = 0;
        }
        if (k >= nxh) {
            A.y = -A.y;
            B.y = -B.y;
        }
        a[t] = R2{A.x - B.y, A.y + B.x};
    }
    __syncthreads();
    R2 *res = fft_smem<R>(a, b, pl, tws, (R)1, rows);
    const R norm = (R)(1.0 / ((double)nx * (double)ny));
    R *pp = phip + (size_t)nx * ny * (zi + 1);
    for (int t = tid; t < rows * nx; t += blockDim.x) {
        const int r = t / nx, x = t - r * nx;
        const int ya = y0 + 2 * r, yb = ya + 1;
        if (ya < ny) pp[(size_t)nx * ya + x] = res[t].x * norm;
        if (yb < ny) pp[(size_t)nx * yb + x] = res[t].y * norm;
    }
}

// ---------------------------------------------------------------------------
// compile-time radix kernels (N = 64, 128, 256, 512)
// ---------------------------------------------------------------------------

// per-transform stride in shared memory: padded, and odd in 8-byte units so
// the transposed (column-major) accesses do not collide on one bank
template <int N> __host__ __device__ constexpr int tstride() { return fft::padded(N) + 1; }
template <int N> constexpr int per_block() { return 256 / fft::Plan<N>::G; }
// rows of a split-path slab: the n = L/2 - 1 interior planes rounded up to
// whole rounds of 32 rows (8 warps of 4 FFT64s)
template <int L> constexpr int slab_rows() { return (L / 2 - 1 + 31) / 32 * 32; }

template <typename R, int N>
__device__ __forceinline__ void load_twiddles(typename Cplx<R>::T *tws,
                                              const typename Cplx<R>::T *__restrict__ tw) {
    for (int i = threadIdx.x; i < N; i += blockDim.x) tws[i] = tw[i];
}

// K1, two real rows (y, y+1) per complex transform: z = a + i b, then
// A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / (2i).
template <typename R, int N>
__global__ void __launch_bounds__(256)
poisson_rows_fwd_fast(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spec,
                      double *__restrict__ rowsum, const typename Cplx<R>::T *__restrict__ tw,
                      const double *__restrict__ qmean, int ny, int nxh, int pitch, double eps,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        q = (const R *)gp.q;
        spec = (typename Cplx<R>::T *)gp.spec;
        rowsum = (double *)gp.rowsum;
        qmean = (const double *)gp.qmean;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::Plan<N>::G, TB = per_block<N>(), P = tstride<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + N;
    const int zi = blockIdx.y;
    const int y0 = blockIdx.x * 2 * TB;
    const int tid = threadIdx.x;
    const R *qp = q + (size_t)N * ny * (zi + 1);
    const R qm = (R)qmean[2 * (zi + 1) + 1];
    const R ieps = (R)(1.0 / eps);
    load_twiddles<R, N>(tws, tw);
    {
        // every load of the tile in flight before the first shared store
        constexpr int IT = TB * N / 256;
        R va[IT], vb[IT];
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = tid + 256 * r;
            const int tr = i / N, x = i - tr * N;
            const int ya = y0 + 2 * tr, yb = ya + 1;
            va[r] = ya < ny ? qp[(size_t)N * ya + x] : qm;
            vb[r] = yb < ny ? qp[(size_t)N * yb + x] : qm;
        }
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = tid + 256 * r;
            const int tr = i / N, x = i - tr * N;
            buf[tr * P + fft::pad(x)] = R2{-(va[r] - qm) * ieps, -(vb[r] - qm) * ieps};
        }
    }
    {  // FP64 row sums, one warp per row, fixed order
        const int warp = tid >> 5, lane = tid & 31;
        for (int r = warp; r < 2 * TB; r += 8) {
            const int y = y0 + r;
            if (y >= ny) continue;
            double sum = 0.0;
            for (int x = lane; x < N; x += 32) sum += (double)qp[(size_t)N * y + x] - (double)qm;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) rowsum[(size_t)zi * ny + y] = -sum / eps;
        }
    }
    __syncthreads();
    const int tr = tid / G, j = tid - tr * G;
    fft::run_tile<N, -1>(buf + tr * P, tws, j);
    R2 *sp = spec + (size_t)zi * ny * pitch;
    for (int i = tid; i < TB * nxh; i += 256) {
        const int t2 = i / nxh, k = i - t2 * nxh;
        const int ya = y0 + 2 * t2, yb = ya + 1;
        const R2 zk = buf[t2 * P + fft::pad(k)];
        const R2 zn = buf[t2 * P + fft::pad(k == 0 ? 0 : N - k)];
        const R2 A = R2{(R)0.5 * (zk.x + zn.x), (R)0.5 * (zk.y - zn.y)};
        const R2 B = R2{(R)0.5 * (zk.y + zn.y), (R)0.5 * (zn.x - zk.x)};
        if (ya < ny) sp[(size_t)pitch * ya + k] = A;
        if (yb < ny) sp[(size_t)pitch * yb + k] = B;
    }
}

// K2 for NY = N: tiles of TB kx columns, loaded transposed (coalesced along kx).
template <typename R, int N, int S>
__global__ void __launch_bounds__(256)
poisson_cols_fast(typename Cplx<R>::T *__restrict__ spec,
                  const typename Cplx<R>::T *__restrict__ tw, int nxh, int pitch,
                  const double *__restrict__ rowsum, double *__restrict__ planesum,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        if (rowsum) rowsum = (const double *)gp.rowsum;
        if (planesum) planesum = (double *)gp.planesum;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::Plan<N>::G, TB = per_block<N>(), P = tstride<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + N;
    const int zi = blockIdx.y;
    const int k0 = blockIdx.x * TB;
    const int tid = threadIdx.x;
    const size_t off = (size_t)zi * N * pitch;
    load_twiddles<R, N>(tws, tw);
    // thread tid serves column c = tid % TB and rows y = tid / TB + (256 / TB) r
    constexpr int IT = TB * N / 256, YS = 256 / TB;
    const int c = tid % TB, yt = tid / TB;
    const bool valid = k0 + c < nxh;
    R2 *col = spec + off + k0 + c;
    {
        R2 v[IT];
#pragma unroll
        for (int r = 0; r < IT; ++r)
            v[r] = valid ? col[(size_t)pitch * (yt + YS * r)] : R2{(R)0, (R)0};
#pragma unroll
        for (int r = 0; r < IT; ++r) buf[c * P + fft::pad(yt + YS * r)] = v[r];
    }
    if (S < 0 && blockIdx.x == 0 && tid < 32) plane_sum_warp(rowsum, planesum, zi, N);
    __syncthreads();
    const int tr = tid / G, j = tid - tr * G;
    fft::run_tile<N, S>(buf + tr * P, tws, j);
    if (valid) {
#pragma unroll
        for (int r = 0; r < IT; ++r)
            col[(size_t)pitch * (yt + YS * r)] = buf[c * P + fft::pad(yt + YS * r)];
    }
}

// K4 for NX = N, two rows per transform: Z = A + i B over the full length
// (A, B Hermitian-completed; the imaginary parts of the k = 0 and k = N/2
// bins, which a real transform ignores, are dropped), inverse FFT,
// phi'(y) = Re Z / (NX NY), phi'(y+1) = Im Z / (NX NY).
template <typename R, int N>
__global__ void __launch_bounds__(256)
poisson_rows_inv_fast(const typename Cplx<R>::T *__restrict__ spec, R *__restrict__ phip,
                      const typename Cplx<R>::T *__restrict__ tw, int ny, int nxh, int pitch,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (const typename Cplx<R>::T *)gp.spec;
        phip = (R *)gp.phip;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::Plan<N>::G, TB = per_block<N>(), P = tstride<N>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + N;
    const int zi = blockIdx.y;
    const int y0 = blockIdx.x * 2 * TB;
    const int tid = threadIdx.x;
    const R2 *sp = spec + (size_t)zi * ny * pitch;
    load_twiddles<R, N>(tws, tw);
    {
        constexpr int IT = TB * N / 256;
        R2 va[IT], vb[IT];
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = tid + 256 * r;
            const int tr = i / N, k = i - tr * N;
            const int ya = y0 + 2 * tr, yb = ya + 1;
            const int kk = k < nxh ? k : N - k;
            va[r] = ya < ny ? sp[(size_t)pitch * ya + kk] : R2{(R)0, (R)0};
            vb[r] = yb < ny ? sp[(size_t)pitch * yb + kk] : R2{(R)0, (R)0};
        }
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = tid + 256 * r;
            const int tr = i / N, k = i - tr * N;
            const int kk = k < nxh ? k : N - k;
            R2 A = va[r], B = vb[r];
            if (kk == 0 || kk == N / 2) {
                A.y = 0;
                B.y = 0;
            }
            if (k >= nxh) {
                A.y = -A.y;
                B.y = -B.y;
            }
            buf[tr * P + fft::pad(k)] = R2{A.x - B.y, A.y + B.x};
        }
    }
    __syncthreads();
    const int tr = tid / G, j = tid - tr * G;
    fft::run_tile<N, 1>(buf + tr * P, tws, j);
    const R norm = (R)(1.0 / ((double)N * (double)ny));
    R *pp = phip + (size_t)N * ny * (zi + 1);
    for (int i = tid; i < TB * N; i += 256) {
        const int t2 = i / N, x = i - t2 * N;
        const int ya = y0 + 2 * t2, yb = ya + 1;
        const R2 zv = buf[t2 * P + fft::pad(x)];
        if (ya < ny) pp[(size_t)N * ya + x] = zv.x * norm;
        if (yb < ny) pp[(size_t)N * yb + x] = zv.y * norm;
    }
}

// ---------------------------------------------------------------------------
// z solve
// ---------------------------------------------------------------------------

// K3: per mode (kx, ky), the Thomas algorithm in FP64 with the pivots
// cp_i = 1/(-beta - cp_{i-1}) read from cpt[i][mode] and the forward sweep d'
// kept in the FP64 scratch dpw[i][mode]; loads are issued in register batches
// of kZB planes ahead of the dependent chain.  The result overwrites the
// spectrum.  The thread of the (0,0) mode solves the mean mode instead:
// right-hand side per plane the FP64 plane sum of s' plus NX NY (-q_m/eps),
// with the electrode voltage entering as -V/dz^2 (NX NY) on z = 1
// (poisson.cu:97); phi00(z) = x / (NX NY), phi00(0) = V, phi00(NZ-1) = 0,
// and its central-difference Ez with the electrode copy (poisson.cu:44-73).
// The (0,0) entries of the spectrum are set to 0.
constexpr int kZB = 8;

template <typename R>
__global__ void __launch_bounds__(128)
poisson_zsolve(typename Cplx<R>::T *__restrict__ spec, const double *__restrict__ cpt,
               double2 *__restrict__ dpw, const double *__restrict__ planesum,
               const double *__restrict__ qmean, double *__restrict__ phi00,
               double *__restrict__ ez00, int nx, int ny, int nz, int nxh, int pitch,
               double dz, double eps, double voltage,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        dpw = (double2 *)gp.dpw;
        planesum = (const double *)gp.planesum;
        qmean = (const double *)gp.qmean;
        phi00 = (double *)gp.phi00;
        ez00 = (double *)gp.ez00;
    }
    using R2 = typename Cplx<R>::T;
    const int modes = nxh * ny;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes) return;
    const int n = nz - 2;
    const int ky = m / nxh, kx = m - ky * nxh;
    const size_t plane = (size_t)ny * pitch;
    R2 *sp = spec + (size_t)pitch * ky + kx;
    const double dz2 = dz * dz;
    if (m == 0) {
        const double nxy = (double)nx * (double)ny;
        double dp = 0.0;
        for (int i = 0; i < n; ++i) {
            double d = planesum[i + 1] + nxy * (-(double)(R)qmean[2 * (i + 1) + 1] / eps);
            if (i == 0) d += -voltage / dz2 * nxy;
            dp = (d * dz2 - dp) * cpt[(size_t)i * modes];
            dpw[(size_t)i * modes] = make_double2(dp, 0.0);
            sp[(size_t)i * plane] = R2{(R)0, (R)0};
        }
        double x = dp;
        phi00[n] = x / nxy;
        for (int i = n - 2; i >= 0; --i) {
            x = dpw[(size_t)i * modes].x - cpt[(size_t)i * modes] * x;
            phi00[i + 1] = x / nxy;
        }
        phi00[0] = voltage;
        phi00[nz - 1] = 0.0;
        for (int z = 1; z <= nz - 2; ++z) ez00[z] = 0.5 * (phi00[z - 1] - phi00[z + 1]) / dz;
        ez00[0] = ez00[1];
        ez00[nz - 1] = ez00[nz - 2];
        return;
    }
    double dr = 0.0, di = 0.0;
    for (int i0 = 0; i0 < n; i0 += kZB) {
        R2 sv[kZB];
        double cv[kZB];
#pragma unroll
        for (int j = 0; j < kZB; ++j) {
            const int i = i0 + j < n ? i0 + j : n - 1;
            sv[j] = sp[(size_t)i * plane];
            cv[j] = __ldg(cpt + (size_t)i * modes + m);
        }
#pragma unroll
        for (int j = 0; j < kZB; ++j) {
            if (i0 + j < n) {
                dr = ((double)sv[j].x * dz2 - dr) * cv[j];
                di = ((double)sv[j].y * dz2 - di) * cv[j];
                dpw[(size_t)(i0 + j) * modes + m] = make_double2(dr, di);
            }
        }
    }
    double xr = dr, xi = di;
    sp[(size_t)(n - 1) * plane] = R2{(R)xr, (R)xi};
    for (int i1 = n - 2; i1 >= 0; i1 -= kZB) {
        double2 dv[kZB];
        double cv[kZB];
#pragma unroll
        for (int j = 0; j < kZB; ++j) {
            const int i = i1 - j >= 0 ? i1 - j : 0;
            dv[j] = dpw[(size_t)i * modes + m];
            cv[j] = __ldg(cpt + (size_t)i * modes + m);
        }
#pragma unroll
        for (int j = 0; j < kZB; ++j) {
            if (i1 - j >= 0) {
                xr = dv[j].x - cv[j] * xr;
                xi = dv[j].y - cv[j] * xi;
                sp[(size_t)(i1 - j) * plane] = R2{(R)xr, (R)xi};
            }
        }
    }
}

// x, hidden from the optimiser: the values derived from it inside a loop are
// recomputed in each iteration instead of being hoisted into registers that
// stay live over the whole loop
__device__ __forceinline__ int opaque(int x) {
    int y;
    asm volatile("mov.b32 %0, %1;" : "=r"(y) : "r"(x));
    return y;
}

// correctly rounded reciprocal
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }

// K3 (fast sizes): the same z solve by the sine transform the reference's
// odd extension amounts to, for L = 2 (NZ - 1) in the compile-time FFT sizes,
// in the compute type.  Per mode the interior column x_1..x_n (n = NZ - 2) is
// extended oddly to length L, y = [0, x_1..x_n, 0, -x_n..-x_1], so that its
// DFT is Y_k = -2i S_k with S_k = sum_j x_j sin(pi j k / (n + 1)) (DST-I).
// The 3-point operator x_{j-1} - beta x_j + x_{j+1} has the eigenvalues
// -(lambda_k + h dz^2), lambda_k = 4 sin^2(pi k / L), on sin(pi j k / (n+1)),
// and the same DFT applied to the scaled, still odd, spectrum gives
//   x_j = (dz^2 / L) DFT[ Y_k / (lambda_k + h dz^2) ]_j,
// with h = kx^2 + ky^2 (main.cu:110-129) and the terms k = 0, L/2 zero.
// lambda_k comes from an FP64 table: 2 - 2 cos(2 pi k / L) in the compute type
// would cancel for small k.  TB modes per block, consecutive in the flattened
// index m = ky nxh + kx.
//
// The (0,0) mode is solved by the block holding m = 0 in FP64 and apart from
// the transforms: right-hand side as in poisson_zsolve, and with beta = 2 the
// inverse of the Dirichlet operator is known in closed form,
//   x_i = -sum_j min(i, j) (n + 1 - max(i, j)) / (n + 1) d_j dz^2,
// one thread per plane.  That block writes phi00 and its Ez.
template <typename R, int L>
__global__ void __launch_bounds__(256)
poisson_zdst(typename Cplx<R>::T *__restrict__ spec, const typename Cplx<R>::T *__restrict__ twz,
             const R *__restrict__ lamz, const double *__restrict__ planesum,
             const double *__restrict__ qmean, double *__restrict__ phi00,
             double *__restrict__ ez00, int nx, int ny, int nxh, int pitch, double dz,
             double eps, double voltage, double kx0, double ky0,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        planesum = (const double *)gp.planesum;
        qmean = (const double *)gp.qmean;
        phi00 = (double *)gp.phi00;
        ez00 = (double *)gp.ez00;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::WPlan<L>::G, TB = 256 / G, P = tstride<L>();
    constexpr int n = L / 2 - 1, nz = n + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + L;
    __shared__ double mrhs[n > 0 ? n : 1], mphi[nz];
    __shared__ R hdz2[TB];  // (kx^2 + ky^2) dz^2 of transform t, < 0: no mode
    const int tid = threadIdx.x;
    const int modes = nxh * ny;
    const int m0 = blockIdx.x * TB;
    const size_t plane = (size_t)ny * pitch;
    const double dz2 = dz * dz;
    for (int i = tid; i < L; i += 256) tws[i] = twz[i];
    // thread tid serves transform t = tid % TB and planes zi = tid / TB + (256 / TB) r
    constexpr int YS = 256 / TB, IT = (n + YS - 1) / YS;
    const int t = tid % TB, zt = tid / TB;
    const int m = m0 + t;
    const bool valid = m < modes && m != 0;
    size_t goff = 0;
    if (m < modes) {
        const int ky = m / nxh, kx = m - ky * nxh;
        goff = (size_t)ky * pitch + kx;
        if (zt == 0) {
            const double wx = kx * kx0, wy = (ky <= ny / 2 ? ky : ky - ny) * ky0;
            hdz2[t] = m == 0 ? (R)-1 : (R)((wx * wx + wy * wy) * dz2);
        }
    } else if (zt == 0) {
        hdz2[t] = (R)-1;
    }
    {
        R2 v[IT];
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int zi = zt + YS * r;
            v[r] = valid && zi < n ? spec[(size_t)zi * plane + goff] : R2{(R)0, (R)0};
        }
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int zi = zt + YS * r;
            if (zi < n) {
                buf[t * P + fft::pad(zi + 1)] = v[r];
                buf[t * P + fft::pad(L - 1 - zi)] = R2{-v[r].x, -v[r].y};
            }
        }
    }
    if (tid < TB) {
        buf[tid * P + fft::pad(0)] = R2{(R)0, (R)0};
        buf[tid * P + fft::pad(L / 2)] = R2{(R)0, (R)0};
    }
    if (m0 == 0) {
        const double nxy = (double)nx * (double)ny;
        for (int i = tid; i < n; i += 256) {
            double d = planesum[i + 1] + nxy * (-(double)(R)qmean[2 * (i + 1) + 1] / eps);
            if (i == 0) d += -voltage / dz2 * nxy;
            mrhs[i] = d * dz2;
        }
    }
    __syncthreads();
    {
        // the two transforms of each mode warp-synchronous (G threads of one
        // warp), the division applied by the first one's last pass
        const int tr = tid / G, j = tid - tr * G;
        R2 *tb = buf + tr * P;
        const R h = hdz2[tr];
        auto ld = [&](int m) { return tb[fft::pad(m)]; };
        auto div = [&](int k, R2 v) {
            if (k == 0 || k == L / 2 || h < (R)0) return R2{(R)0, (R)0};
            const R f = rcp(lamz[k < L / 2 ? k : L - k] + h);
            return R2{v.x * f, v.y * f};
        };
        if constexpr (L == 64 || L == 256) {
            fft::wfilter_sq<L, G, -1, -1>(tb, tws, j, ld, div,
                                         [&](int m, R2 v) { tb[fft::pad(m)] = v; });
        } else {
            fft::WPlan<L>::template run<-1>(tb, tws, j, ld,
                                            [&](int k, R2 v) { tb[fft::pad(k)] = div(k, v); });
            __syncwarp();
            fft::WPlan<L>::template run<-1>(tb, tws, j, ld,
                                            [&](int m, R2 v) { tb[fft::pad(m)] = v; });
        }
    }
    __syncthreads();
    const R sc = (R)(dz2 / (double)L);
    if (m < modes) {
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int zi = zt + YS * r;
            if (zi < n) {
                const R2 w = buf[t * P + fft::pad(zi + 1)];
                spec[(size_t)zi * plane + goff] = R2{w.x * sc, w.y * sc};
            }
        }
    }
    if (m0 == 0) {
        const double nxy = (double)nx * (double)ny;
        for (int i = tid; i < nz; i += 256) {
            double x = 0.0;
            if (i == 0) {
                x = voltage;
            } else if (i < nz - 1) {
                for (int jj = 1; jj <= n; ++jj) {
                    const int lo = i < jj ? i : jj, hi = i < jj ? jj : i;
                    x -= (double)(lo * (n + 1 - hi)) * mrhs[jj - 1];
                }
                x = x / (double)(n + 1) / nxy;
            }
            mphi[i] = x;
            phi00[i] = x;
        }
        __syncthreads();
        for (int z = tid; z < nz; z += 256) {
            const int zc = z < 1 ? 1 : (z > nz - 2 ? nz - 2 : z);
            ez00[z] = 0.5 * (mphi[zc - 1] - mphi[zc + 1]) / dz;
        }
    }
}

// K3 for any L = 2 (NZ - 1) whose transforms fit in shared memory: the
// sine-transform z solve of poisson_zdst with run-time radix passes
// (fft_smem) instead of compile-time ones.  tb modes per block, consecutive
// in m = ky nxh + kx; the odd extensions of the block's modes are held as tb
// contiguous length-L transforms (two buffers for the Stockham passes).  The
// block holding m = 0 solves the (0,0) mode in FP64 in closed form.
template <typename R>
__global__ void __launch_bounds__(256)
poisson_zdst_rt(typename Cplx<R>::T *__restrict__ spec, const typename Cplx<R>::T *__restrict__ twz,
                const R *__restrict__ lamz, FftPlan pl, const double *__restrict__ planesum,
                const double *__restrict__ qmean, double *__restrict__ phi00,
                double *__restrict__ ez00, int nx, int ny, int nxh, int pitch, int tb, double dz,
                double eps, double voltage, double kx0, double ky0,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        planesum = (const double *)gp.planesum;
        qmean = (const double *)gp.qmean;
        phi00 = (double *)gp.phi00;
        ez00 = (double *)gp.ez00;
    }
    using R2 = typename Cplx<R>::T;
    const int L = pl.n, n = L / 2 - 1, nz = n + 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *a = reinterpret_cast<R2 *>(smem_raw);
    R2 *b = a + (size_t)tb * L;
    R2 *tws = b + (size_t)tb * L;                                   // L
    double *mrhs = reinterpret_cast<double *>(tws + L);             // n
    double *mphi = mrhs + n;                                          // nz
    R *hdz2 = reinterpret_cast<R *>(mphi + nz);                       // tb
    const int tid = threadIdx.x;
    const int modes = nxh * ny;
    const int m0 = blockIdx.x * tb;
    const size_t plane = (size_t)ny * pitch;
    const double dz2 = dz * dz;
    for (int i = tid; i < L; i += 256) tws[i] = twz[i];
    for (int t = tid; t < tb; t += 256) {
        const int m = m0 + t;
        R h = (R)-1;
        if (m < modes && m != 0) {
            const int ky = m / nxh, kx = m - ky * nxh;
            const double wx = kx * kx0, wy = (ky <= ny / 2 ? ky : ky - ny) * ky0;
            h = (R)((wx * wx + wy * wy) * dz2);
        }
        hdz2[t] = h;
        a[(size_t)t * L] = R2{(R)0, (R)0};
        a[(size_t)t * L + L / 2] = R2{(R)0, (R)0};
    }
    for (int i = tid; i < tb * n; i += 256) {
        const int zi = i / tb, t = i - zi * tb;
        const int m = m0 + t;
        R2 v = R2{(R)0, (R)0};
        if (m < modes && m != 0) {
            const int ky = m / nxh, kx = m - ky * nxh;
            v = spec[(size_t)zi * plane + (size_t)ky * pitch + kx];
        }
        a[(size_t)t * L + zi + 1] = v;
        a[(size_t)t * L + L - 1 - zi] = R2{-v.x, -v.y};
    }
    const bool mean_block = m0 == 0;
    if (mean_block) {
        const double nxy = (double)nx * (double)ny;
        for (int i = tid; i < n; i += 256) {
            double d = planesum[i + 1] + nxy * (-(double)(R)qmean[2 * (i + 1) + 1] / eps);
            if (i == 0) d += -voltage / dz2 * nxy;
            mrhs[i] = d * dz2;
        }
    }
    __syncthreads();
    R2 *r1 = fft_smem<R>(a, b, pl, tws, (R)-1, tb);
    for (int i = tid; i < tb * L; i += 256) {
        const int t = i / L, k = i - t * L;
        const R h = hdz2[t];
        R2 y = r1[i];
        if (k == 0 || k == L / 2 || h < (R)0) {
            y = R2{(R)0, (R)0};
        } else {
            const R f = rcp(lamz[k < L / 2 ? k : L - k] + h);
            y = R2{y.x * f, y.y * f};
        }
        r1[i] = y;
    }
    __syncthreads();
    R2 *r2 = fft_smem<R>(r1, r1 == a ? b : a, pl, tws, (R)-1, tb);
    const R sc = (R)(dz2 / (double)L);
    for (int i = tid; i < tb * n; i += 256) {
        const int zi = i / tb, t = i - zi * tb;
        const int m = m0 + t;
        if (m < modes) {
            const int ky = m / nxh, kx = m - ky * nxh;
            const R2 w = r2[(size_t)t * L + zi + 1];
            spec[(size_t)zi * plane + (size_t)ky * pitch + kx] = R2{w.x * sc, w.y * sc};
        }
    }
    if (mean_block) {
        const double nxy = (double)nx * (double)ny;
        for (int i = tid; i < nz; i += 256) {
            double x = 0.0;
            if (i == 0) {
                x = voltage;
            } else if (i < nz - 1) {
                for (int jz = 1; jz <= n; ++jz) {
                    const int lo = i < jz ? i : jz, hi = i < jz ? jz : i;
                    x -= (double)(lo * (n + 1 - hi)) * mrhs[jz - 1];
                }
                x = x / (double)(n + 1) / nxy;
            }
            mphi[i] = x;
            phi00[i] = x;
        }
        __syncthreads();
        for (int z = tid; z < nz; z += 256) {
            const int zc = z < 1 ? 1 : (z > nz - 2 ? nz - 2 : z);
            ez00[z] = 0.5 * (mphi[zc - 1] - mphi[zc + 1]) / dz;
        }
    }
}

// ---------------------------------------------------------------------------
// split-y path: three launches instead of five
// ---------------------------------------------------------------------------
//
// For NY = 64 S (S = 1, 2, 4, 8) the y transform of length NY is split as
// y = n + 64 m (n < 64, m < S), ky = S k' + j (k' < 64, j < S):
//   forward   Y[S k' + j] = FFT64_n( a_j[n] )[k'],
//             a_j[n] = W_NY^(j n) sum_m x[n + 64 m] W_S^(j m)
//   inverse   x[n + 64 m] = sum_j W_S^(-j m) b_j[n],
//             b_j[n] = W_NY^(-j n) IFFT64_k'( Y[S k' + j] )[n]
// (W_N = exp(-2 pi i / N)).  The x-row kernels form a_j (after the forward x
// transform) and consume b_j (before the inverse one); in between one slab
// kernel per (kx, j) holds a_j for every plane z on chip and runs the forward
// FFT64 along n, the tridiagonal (Thomas) z solve of each of its 64 modes, and
// the inverse FFT64, so the spectrum goes through L2 twice instead of four
// times.
// The split spectrum is laid out [j][kx][z - 1][n], so that a slab is one
// contiguous block.
namespace {

// rows (ya, yb) of transform tr of a split-row block (two real rows per
// complex transform): S = 1 pairs consecutive rows; S >= 2 pairs
// n + 64 a and n + 64 (a + S/2) of group n = block * GB + tr / (S/2)
template <int S, int TB>
__device__ __forceinline__ void split_rows(int tr, int &ya, int &yb, int &g, int &a) {
    if constexpr (S == 1) {
        g = 2 * tr;
        a = 0;
        ya = blockIdx.x * 2 * TB + 2 * tr;
        yb = ya + 1;
    } else {
        constexpr int GB = 2 * TB / S;
        g = tr / (S / 2);
        a = tr - g * (S / 2);
        ya = blockIdx.x * GB + g + 64 * a;
        yb = ya + 32 * S;
    }
}

// x * exp(-2 pi i e / 8) for e = 0..7, by swaps, negations and one scale by
// sqrt(1/2) (no multiplication by zero); in unrolled loops e is a constant
template <typename R2>
__device__ __forceinline__ R2 mul_w8(R2 x, int e) {
    using R = decltype(x.x);
    const R r = (R)0.70710678118654752440;
    switch (e & 7) {
        case 0: return x;
        case 1: return R2{r * (x.x + x.y), r * (x.y - x.x)};
        case 2: return R2{x.y, -x.x};
        case 3: return R2{r * (x.y - x.x), -r * (x.x + x.y)};
        case 4: return R2{-x.x, -x.y};
        case 5: return R2{-r * (x.x + x.y), r * (x.x - x.y)};
        case 6: return R2{-x.y, x.x};
        default: return R2{r * (x.x - x.y), r * (x.x + x.y)};
    }
}
// x * W_S^k = x * exp(-2 pi i k / S), S = 1, 2, 4, 8
template <int S, typename R2>
__device__ __forceinline__ R2 mul_ws(R2 x, int k) {
    return mul_w8(x, (k % S) * (8 / S));
}

// x-spectrum of row part (0: ya, 1: yb) of a packed transform at bin k < nxh
template <typename R2, typename R>
__device__ __forceinline__ R2 unpack_bin(const R2 *buf, int k, int part, int N) {
    const R2 zk = buf[fft::pad(k)];
    const R2 zn = buf[fft::pad((N - k) & (N - 1))];
    return part == 0 ? R2{(R)0.5 * (zk.x + zn.x), (R)0.5 * (zk.y - zn.y)}
                     : R2{(R)0.5 * (zk.y + zn.y), (R)0.5 * (zn.x - zk.x)};
}

}  // namespace

// K1 of the split path: s' = -(q - q_m)/eps, x-FFT of two real rows per
// transform, FP64 row sums, then the radix-S first stage of the y transform,
// written as a_j[n] into spl[j][kx][z - 1][n].
template <typename R, int N, int S>
__global__ void __launch_bounds__(256)
poisson_rows_fwd_split(const R *__restrict__ q, typename Cplx<R>::T *__restrict__ spl,
                       double *__restrict__ rowsum, const typename Cplx<R>::T *__restrict__ tw,
                       const typename Cplx<R>::T *__restrict__ twy,
                       const double *__restrict__ qmean, int nzi, int nxh, double eps,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        q = (const R *)gp.q;
        spl = (typename Cplx<R>::T *)gp.spec;
        rowsum = (double *)gp.rowsum;
        qmean = (const double *)gp.qmean;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::Plan<N>::G, TB = per_block<N>(), P = tstride<N>();
    constexpr int NY = 64 * S, GB = 2 * TB / S;
    static_assert(GB >= 1, "a block holds whole row groups");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + N;
    const int zi = blockIdx.y;
    const int tid = threadIdx.x;
    const R *qp = q + (size_t)N * NY * (zi + 1);
    const R qm = (R)qmean[2 * (zi + 1) + 1];
    const R ieps = (R)(1.0 / eps);
    load_twiddles<R, N>(tws, tw);
    // each warp loads a contiguous run of the block's (transform, x) items,
    // 32 consecutive x at a time, and sums its rows from the registers
    constexpr int IT = TB * N / 256;            // items per thread
    constexpr int WI = 32 * IT;                 // items per warp
    constexpr int SEG = WI >= N ? 1 : N / WI;   // warps per transform
    constexpr int TPW = WI >= N ? WI / N : 1;   // transforms per warp
    constexpr int RPT = IT / TPW;               // items per thread and transform
    __shared__ double part[2 * TB * SEG];
    {
        const int warp = tid >> 5, lane = tid & 31;
        R va[IT], vb[IT];
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = warp * WI + 32 * r + lane;
            const int tr = i / N, x = i - tr * N;
            int ya, yb, g, a;
            split_rows<S, TB>(tr, ya, yb, g, a);
            va[r] = qp[(size_t)N * ya + x];
            vb[r] = qp[(size_t)N * yb + x];
        }
#pragma unroll
        for (int r = 0; r < IT; ++r) {
            const int i = warp * WI + 32 * r + lane;
            const int tr = i / N, x = i - tr * N;
            buf[tr * P + fft::pad(x)] = R2{-(va[r] - qm) * ieps, -(vb[r] - qm) * ieps};
        }
        // FP64 sums of q - q_m of both rows of each transform, fixed order
#pragma unroll
        for (int c = 0; c < TPW; ++c) {
            double sa = 0.0, sb = 0.0;
#pragma unroll
            for (int u = 0; u < RPT; ++u) {
                sa += (double)va[c * RPT + u] - (double)qm;
                sb += (double)vb[c * RPT + u] - (double)qm;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sa += __shfl_xor_sync(0xffffffffu, sa, o);
                sb += __shfl_xor_sync(0xffffffffu, sb, o);
            }
            if (lane == 0) {
                const int i0 = warp * WI + 32 * RPT * c;
                const int tr = i0 / N, seg = SEG > 1 ? (i0 - tr * N) / WI : 0;
                part[(2 * tr) * SEG + seg] = sa;
                part[(2 * tr + 1) * SEG + seg] = sb;
            }
        }
    }
    __syncthreads();
    if (tid < 2 * TB) {
        double sum = 0.0;
#pragma unroll
        for (int k = 0; k < SEG; ++k) sum += part[tid * SEG + k];
        int ya, yb, g, a;
        split_rows<S, TB>(tid >> 1, ya, yb, g, a);
        rowsum[(size_t)zi * NY + ((tid & 1) ? yb : ya)] = -sum / eps;
    }
    {
        const int tr = tid / G, jj = tid - tr * G;
        fft::run_tile<N, -1>(buf + tr * P, tws, jj);
    }
    // items (g, kx), g fastest: the S rows n + 64 m of group g at bin kx, a
    // radix-S DFT over m, the twiddle W_NY^(j n), S outputs of GB consecutive
    // n per (j, kx)
    const int nblk = S == 1 ? 2 * TB : GB;
    const int n0 = blockIdx.x * nblk;
    // the twiddles W_NY^(j n) of the block's n, from shared memory
    __shared__ R2 twn[S == 1 ? 1 : S * GB];
    if constexpr (S > 1) {
        for (int i = tid; i < S * GB; i += 256) twn[i] = twy[(i / GB) * (n0 + i % GB)];
        __syncthreads();
    }
    for (int i = tid; i < nxh * nblk; i += 256) {
        const int g = i % nblk, kx = i / nblk;
        const int n = n0 + g;
        if constexpr (S == 1) {
            spl[((size_t)kx * nzi + zi) * 64 + n] = unpack_bin<R2, R>(buf + (g >> 1) * P, kx, g & 1, N);
        } else {
            R2 x[S];
#pragma unroll
            for (int m = 0; m < S; ++m)
                x[m] = unpack_bin<R2, R>(buf + (g * (S / 2) + (m % (S / 2))) * P, kx,
                                         m < S / 2 ? 0 : 1, N);
#pragma unroll
            for (int j = 0; j < S; ++j) {
                R2 acc = x[0];
#pragma unroll
                for (int m = 1; m < S; ++m) acc = cadd(acc, mul_ws<S>(x[m], j * m));
                if (j != 0 && n != 0) acc = cmul(acc, twn[j * GB + g]);
                spl[(((size_t)j * nxh + kx) * nzi + zi) * 64 + n] = acc;
            }
        }
    }
}

// pivot rows of a mode in the split path's table: the two-sided Thomas
// solve of n = L/2 - 1 (odd) planes eliminates (n - 1)/2 planes from each
// electrode with the same pivots c_0..c_{m-1}, then the middle plane with
// mu = 1/(-beta - 2 c_{m-1})
template <int L> constexpr int slab_piv_rows() { return (L / 2 - 1 + 1) / 2; }
// dynamic shared memory of the slab kernel: the FFT64 twiddles, the output
// twiddles, the block's pivot rows [r][k'] and the slab
template <typename R, int L>
constexpr size_t slab_smem() {
    return sizeof(typename Cplx<R>::T) * ((size_t)128 + (size_t)slab_rows<L>() * tstride<64>()) +
           sizeof(R) * (size_t)slab_piv_rows<L>() * 64;
}
// resident blocks per SM that their shared memory allows (two at most)
template <typename R, int L>
constexpr int slab_min_blocks() {
    return 2 * slab_smem<R, L>() + 4096 <= 227 * 1024 ? 2 : 1;
}

// 16-byte asynchronous copy global -> shared (cp.async), and the wait for all
// of a thread's copies
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// K2 of the split path, one block per (kx, j): the slab a_j[z - 1][n] of all
// interior planes in shared memory; FFT64 along n (ky = S k' + j), the
// tridiagonal z solve of each of the 64 modes, inverse FFT64, the twiddle
// W_NY^(-j n), written back in place as b_j.  The z solve is the system of
// poisson_zsolve, phi(z-1) - beta phi(z) + phi(z+1) = dz^2 s(z),
// beta = 2 + (kx^2 + ky^2) dz^2, phi = 0 on the electrodes, solved from both
// ends at once in FP64 arithmetic: one thread eliminates the upper half of the
// planes downwards and one the lower half upwards with the same pivots (the
// matrix is symmetric Toeplitz), they meet at the middle plane, and each
// substitutes back over its half.  The pivots come from the table built once
// per context, in the compute type.  The 64-point
// transforms are warp-synchronous (fft::WPlan): the rows n of a plane are
// transformed on their way in from global memory and on their way out, so the
// block synchronises only between the three phases; the block's pivots
// arrive by cp.async during the first.  Block x = 0 of y = 0 (one more block
// than kx columns) forms the FP64 plane sums of the source and solves the
// (0,0) mode in closed form (as poisson_zdst), writing phi00 and its Ez, on
// its own beside the slabs; the (0,0) mode of the fluctuation is 0.
template <typename R, int L, int S>
__global__ void __launch_bounds__(256, slab_min_blocks<R, L>())
poisson_slab(typename Cplx<R>::T *__restrict__ spl, const typename Cplx<R>::T *__restrict__ twy,
             const R *__restrict__ cps, const double *__restrict__ rowsum,
             double *__restrict__ planesum, const double *__restrict__ qmean,
             double *__restrict__ phi00, double *__restrict__ ez00, int nx, int nxh, double dz,
             double eps, double voltage, const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spl = (typename Cplx<R>::T *)gp.spec;
        rowsum = (const double *)gp.rowsum;
        planesum = (double *)gp.planesum;
        qmean = (const double *)gp.qmean;
        phi00 = (double *)gp.phi00;
        ez00 = (double *)gp.ez00;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int NY = 64 * S;
    constexpr int n = L / 2 - 1, nz = n + 2;
    constexpr int P64 = tstride<64>();
    constexpr int NR = slab_rows<L>();  // slab rows, whole rounds of 32
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const double dz2 = dz * dz;
    if (blockIdx.x == 0) {
        if (blockIdx.y != 0) return;
        __shared__ double mrhs[n], mphi[nz];
        // FP64 plane sums of the source (fixed order), then the right-hand
        // side of the mean mode (poisson.cu:97 for the voltage on z = 1); the
        // row sums of four planes in flight at a time, in chunks of up to
        // four rows a lane
        const double nxy = (double)nx * (double)NY;
        constexpr int PW = 4, YL = NY / 32, YC = YL < 4 ? YL : 4;
        for (int z0 = warp * PW; z0 < n; z0 += 8 * PW) {
            double acc[PW];
#pragma unroll
            for (int u = 0; u < PW; ++u) acc[u] = 0.0;
#pragma unroll 1
            for (int t0 = 0; t0 < YL; t0 += YC) {
                double v[PW][YC];
#pragma unroll
                for (int u = 0; u < PW; ++u)
#pragma unroll
                    for (int t = 0; t < YC; ++t)
                        v[u][t] = z0 + u < n ? rowsum[(size_t)(z0 + u) * NY + lane + 32 * (t0 + t)]
                                             : 0.0;
#pragma unroll
                for (int u = 0; u < PW; ++u)
#pragma unroll
                    for (int t = 0; t < YC; ++t) acc[u] += v[u][t];
            }
#pragma unroll
            for (int u = 0; u < PW; ++u) {
                const int zi = z0 + u;
                double sum = acc[u];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                if (lane == 0 && zi < n) {
                    planesum[zi + 1] = sum;
                    double d = sum + nxy * (-(double)(R)qmean[2 * (zi + 1) + 1] / eps);
                    if (zi == 0) d += -voltage / dz2 * nxy;
                    mrhs[zi] = d * dz2;
                }
            }
        }
        __syncthreads();
        for (int i = tid; i < nz; i += 256) {
            double x = 0.0;
            if (i == 0) {
                x = voltage;
            } else if (i < nz - 1) {
                for (int jz = 1; jz <= n; ++jz) {
                    const int lo = i < jz ? i : jz, hi = i < jz ? jz : i;
                    x -= (double)(lo * (n + 1 - hi)) * mrhs[jz - 1];
                }
                x = x / (double)(n + 1) / nxy;
            }
            mphi[i] = x;
            phi00[i] = x;
        }
        __syncthreads();
        for (int z = tid; z < nz; z += 256) {
            const int zc = z < 1 ? 1 : (z > nz - 2 ? nz - 2 : z);
            ez00[z] = 0.5 * (mphi[zc - 1] - mphi[zc + 1]) / dz;
        }
        return;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tw64 = reinterpret_cast<R2 *>(smem_raw);
    R2 *twj = tw64 + 64;  // conj W_NY^(j n), n < 64
    R *piv = reinterpret_cast<R *>(twj + 64);
    R2 *slab = reinterpret_cast<R2 *>(piv + slab_piv_rows<L>() * 64);
    const int kx = blockIdx.x - 1, j = blockIdx.y;
    R2 *base = spl + ((size_t)j * nxh + kx) * n * 64;
    {
        // the block's pivot rows [r][k'], contiguous in the table
        constexpr int PR = slab_piv_rows<L>(), V = 16 / sizeof(R), NV = PR * 64 / V;
        const R *src = cps + ((size_t)kx * S + j) * PR * 64;
        for (int i = tid; i < NV; i += 256) cp_async16(piv + V * i, src + V * i);
    }
    for (int i = tid; i < 64; i += 256) {
        tw64[i] = twy[S * i];
        R2 w = twy[(j * i) % NY];
        w.y = -w.y;
        twj[i] = w;
    }
    __syncthreads();
    // phase 1: forward FFT64 of each plane's row on its way in, 4 rows a
    // warp; each thread's inputs t8 + 8 r of the next round's row are loaded
    // while this round's row is transformed (the first pass takes its inputs
    // in that order)
    const int g8 = lane >> 3, t8 = lane & 7;
    R2 cur[8];
    {
        const int zi = warp * 4 + g8;
        const R2 *src = base + (size_t)zi * 64;
#pragma unroll
        for (int r = 0; r < 8; ++r) cur[r] = zi < n ? src[t8 + 8 * r] : R2{(R)0, (R)0};
    }
#pragma unroll 1
    for (int zi = warp * 4 + g8; zi < NR; zi += 32) {
        const int zn = zi + 32;
        const R2 *srcn = base + (size_t)zn * 64;
        R2 nxt[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) nxt[r] = zn < n ? srcn[t8 + 8 * r] : R2{(R)0, (R)0};
        R2 *row = slab + zi * P64;
        int c = 0;
        fft::WPlan<64>::template run<-1>(
            row, tw64, opaque(t8), [&](int) { return cur[c++]; },
            [&](int m, R2 v) { row[fft::pad(m)] = v; });
#pragma unroll
        for (int r = 0; r < 8; ++r) cur[r] = nxt[r];
    }
    cp_async_wait_all();
    __syncthreads();
    // phase 2: the two-sided Thomas solve of the 64 modes k', 16 modes a warp:
    // lanes 0-15 take the planes 0..m-1 from the top, lanes 16-31 the planes
    // n-1..n-m from the bottom; loads issued kB planes ahead of the chain
    static_assert(n % 2 == 1, "odd number of interior planes");
    if (tid < 128) {
        constexpr int m = (n - 1) / 2, kB = 8;
        const int kp = (warp << 4) | (lane & 15), side = lane >> 4;
        R2 *col = slab + fft::pad(kp);
        const R *pc = piv + kp;
        // plane of elimination step k on this side
        auto plane = [&](int k) { return side ? n - 1 - k : k; };
        // the (0,0) mode is solved like the others (every lane takes part in
        // the exchange) and stored as 0
        const R keep = (kx == 0 && S * kp + j == 0) ? (R)0 : (R)1;
        {
            double dr = 0.0, di = 0.0;
#pragma unroll 1
            for (int k0 = 0; k0 < m; k0 += kB) {
                R2 sv[kB];
                R cv[kB];
#pragma unroll
                for (int u = 0; u < kB; ++u) {
                    const int k = k0 + u < m ? k0 + u : m - 1;
                    sv[u] = col[plane(k) * P64];
                    cv[u] = pc[k * 64];
                }
#pragma unroll
                for (int u = 0; u < kB; ++u) {
                    if (k0 + u < m) {
                        dr = ((double)sv[u].x * dz2 - dr) * (double)cv[u];
                        di = ((double)sv[u].y * dz2 - di) * (double)cv[u];
                        col[plane(k0 + u) * P64] = R2{(R)dr, (R)di};
                    }
                }
            }
            // the middle plane from both sides' last eliminated rows
            const double or_ = __shfl_xor_sync(0xffffffffu, dr, 16);
            const double oi = __shfl_xor_sync(0xffffffffu, di, 16);
            const R2 sm = col[m * P64];
            const double mu = (double)pc[m * 64];
            double xr = ((double)sm.x * dz2 - dr - or_) * mu;
            double xi = ((double)sm.y * dz2 - di - oi) * mu;
            __syncwarp();
            if (side == 0) col[m * P64] = R2{(R)xr * keep, (R)xi * keep};
#pragma unroll 1
            for (int k1 = m - 1; k1 >= 0; k1 -= kB) {
                R2 dv[kB];
                R cv[kB];
#pragma unroll
                for (int u = 0; u < kB; ++u) {
                    const int k = k1 - u >= 0 ? k1 - u : 0;
                    dv[u] = col[plane(k) * P64];
                    cv[u] = pc[k * 64];
                }
#pragma unroll
                for (int u = 0; u < kB; ++u) {
                    if (k1 - u >= 0) {
                        xr = (double)dv[u].x - (double)cv[u] * xr;
                        xi = (double)dv[u].y - (double)cv[u] * xi;
                        col[plane(k1 - u) * P64] = R2{(R)xr * keep, (R)xi * keep};
                    }
                }
            }
        }
    }
    __syncthreads();
    // phase 3: inverse FFT64 of each row and the twiddle on the way out
#pragma unroll 1
    for (int zi = warp * 4 + g8; zi < NR; zi += 32) {
        const bool act = zi < n;
        R2 *dst = base + (size_t)zi * 64;
        R2 *row = slab + zi * P64;
        fft::WPlan<64>::template run<1>(
            row, tw64, opaque(t8), [&](int m) { return row[fft::pad(m)]; },
            [&](int m, R2 v) {
                if (act) dst[m] = j * m != 0 ? cmul(v, twj[m]) : v;
            });
    }
}

// ---- the y transform and z solve of NY x NZ columns in one kernel ----------
//
// The five-kernel path's middle three (forward y FFT of the columns, the
// sine-transform z solve, inverse y FFT) in one launch where NY and
// L = 2 (NZ - 1) are compile-time sizes and NY is not 64 S (the split-y path's
// grids): one block per TB consecutive kx columns holds them for every
// interior plane in shared memory ([c][z - 1][y], rows padded), loaded and
// stored with the TB columns running fastest (TB consecutive 8-byte values of
// the spectrum per (z, y)).  Every transform is warp-synchronous
// (fft::WPlan): the y rows in place, the z columns through the odd extension
// as poisson_slab.  The block of kx = 0 also forms the FP64 plane sums of the
// source and solves the (0,0) mode in closed form, as poisson_zdst.
template <typename R, int NY, int L>
constexpr int yz_cols() {
    constexpr size_t col = sizeof(typename Cplx<R>::T) * (size_t)(L / 2 - 1) * tstride<NY>();
    constexpr int tb = (int)((80 * 1024) / col);
    return tb < 1 ? 1 : (tb > 4 ? 4 : tb);
}
template <typename R, int NY, int L>
constexpr int yz_rows() {  // slab rows TB n, rounded up to whole rounds of the row warps
    constexpr int per = 8 * (32 / fft::WPlan<NY>::G);
    return (yz_cols<R, NY, L>() * (L / 2 - 1) + per - 1) / per * per;
}
template <typename R, int NY, int L>
constexpr size_t yz_smem() {
    return sizeof(typename Cplx<R>::T) *
           ((size_t)NY + L + (size_t)yz_rows<R, NY, L>() * tstride<NY>() +
            (size_t)8 * (32 / fft::WPlan<L>::G) * tstride<L>());
}

template <typename R, int NY, int L>
__global__ void __launch_bounds__(256)
poisson_yz(typename Cplx<R>::T *__restrict__ spec, const typename Cplx<R>::T *__restrict__ twy,
           const typename Cplx<R>::T *__restrict__ twz, const R *__restrict__ lamz,
           const double *__restrict__ rowsum, double *__restrict__ planesum,
           const double *__restrict__ qmean, double *__restrict__ phi00,
           double *__restrict__ ez00, int nx, int nxh, int pitch, double dz, double eps,
           double voltage, double kx0, double ky0, const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spec = (typename Cplx<R>::T *)gp.spec;
        rowsum = (const double *)gp.rowsum;
        planesum = (double *)gp.planesum;
        qmean = (const double *)gp.qmean;
        phi00 = (double *)gp.phi00;
        ez00 = (double *)gp.ez00;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int n = L / 2 - 1, nz = n + 2;
    constexpr int TB = yz_cols<R, NY, L>(), NRY = yz_rows<R, NY, L>();
    constexpr int PY = tstride<NY>(), PL = tstride<L>();
    constexpr int GY = fft::WPlan<NY>::G, TPWY = 32 / GY;
    constexpr int GZ = fft::WPlan<L>::G, TPWZ = 32 / GZ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tyy = reinterpret_cast<R2 *>(smem_raw);
    R2 *twl = tyy + NY;
    R2 *slab = twl + L;  // [c][zi][y]
    R2 *zb = slab + NRY * PY;
    __shared__ double mrhs[n], mphi[nz];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kxb = blockIdx.x * TB;
    const bool mean_block = blockIdx.x == 0;
    const double dz2 = dz * dz;
    const size_t plane = (size_t)NY * pitch;
    for (int i = tid; i < NY; i += 256) tyy[i] = twy[i];
    for (int i = tid; i < L; i += 256) twl[i] = twz[i];
    if (mean_block) {
        // FP64 plane sums of the source (fixed order, as plane_sum_warp), then
        // the right-hand side of the mean mode (poisson.cu:97)
        const double nxy = (double)nx * (double)NY;
        for (int zi = warp; zi < n; zi += 8) {
            double sum = 0.0;
            for (int y = lane; y < NY; y += 32) sum += rowsum[(size_t)zi * NY + y];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) {
                planesum[zi + 1] = sum;
                double d = sum + nxy * (-(double)(R)qmean[2 * (zi + 1) + 1] / eps);
                if (zi == 0) d += -voltage / dz2 * nxy;
                mrhs[zi] = d * dz2;
            }
        }
    }
    for (int i = tid; i < TB * n * NY; i += 256) {
        const int c = i % TB, rest = i / TB, y = rest % NY, zi = rest / NY;
        const int kx = kxb + c;
        slab[(c * n + zi) * PY + fft::pad(y)] =
            kx < nxh ? spec[(size_t)zi * plane + (size_t)y * pitch + kx] : R2{(R)0, (R)0};
    }
    __syncthreads();
    // forward y FFT of every (c, z) row, TPWY rows a warp
    {
        const int g = lane / GY, t0 = lane - g * GY;
#pragma unroll 1
        for (int r = warp * TPWY + g; r < NRY; r += 8 * TPWY) {
            R2 *row = slab + r * PY;
            const bool act = r < TB * n;
            fft::WPlan<NY>::template run<-1>(
                row, tyy, opaque(t0),
                [&](int m) { return act ? row[fft::pad(m)] : R2{(R)0, (R)0}; },
                [&](int m, R2 v) { row[fft::pad(m)] = v; });
        }
    }
    __syncthreads();
    // z solve of every (c, ky) column, TPWZ a warp
    {
        const R sc = (R)(dz2 / (double)L);
        const int g = lane / GZ, t0 = lane - g * GZ;
        R2 *zw = zb + (warp * TPWZ + g) * PL;
        constexpr int NCOL = TB * NY, NCR = (NCOL + 8 * TPWZ - 1) / (8 * TPWZ) * (8 * TPWZ);
#pragma unroll 1
        for (int cc = warp * TPWZ + g; cc < NCR; cc += 8 * TPWZ) {
            const int t = opaque(t0);
            const bool act = cc < NCOL;
            const int c = act ? cc / NY : 0, ky = act ? cc - (cc / NY) * NY : 0;
            const int kx = kxb + c;
            const double wx = kx * kx0, wy = (ky <= NY / 2 ? ky : ky - NY) * ky0;
            const R h = (!act || kx >= nxh || (kx == 0 && ky == 0)) ? (R)-1
                                                                      : (R)((wx * wx + wy * wy) * dz2);
            R2 *col = slab + c * n * PY + fft::pad(ky);
            auto ld = [&](int m) {
                const bool up = m < L / 2;
                // (rows 0..n-1 of the column; m = 0 and L/2 read row 0, unused)
                const R2 v = col[(up ? (m > 0 ? m - 1 : 0) : (m == L / 2 ? 0 : L - 1 - m)) * PY];
                return (!act || m == 0 || m == L / 2) ? R2{(R)0, (R)0}
                                                      : (up ? v : R2{-v.x, -v.y});
            };
            auto div = [&](int k, R2 v) {
                if (k == 0 || k == L / 2 || h < (R)0) return R2{(R)0, (R)0};
                const R f = rcp(lamz[k < L / 2 ? k : L - k] + h);
                return R2{v.x * f, v.y * f};
            };
            auto st = [&](int m, R2 v) {
                if (act && m >= 1 && m <= n) col[(m - 1) * PY] = R2{v.x * sc, v.y * sc};
            };
            if constexpr (L == 64 || L == 256) {
                fft::wfilter_sq<L, GZ, -1, -1>(zw, twl, t, ld, div, st);
            } else {
                fft::WPlan<L>::template run<-1>(zw, twl, t, ld,
                                                [&](int k, R2 v) { zw[fft::pad(k)] = div(k, v); });
                __syncwarp();
                fft::WPlan<L>::template run<-1>(zw, twl, opaque(t0),
                                                [&](int m) { return zw[fft::pad(m)]; }, st);
                __syncwarp();
            }
        }
    }
    __syncthreads();
    // inverse y FFT of every row
    {
        const int g = lane / GY, t0 = lane - g * GY;
#pragma unroll 1
        for (int r = warp * TPWY + g; r < NRY; r += 8 * TPWY) {
            R2 *row = slab + r * PY;
            fft::WPlan<NY>::template run<1>(
                row, tyy, opaque(t0), [&](int m) { return row[fft::pad(m)]; },
                [&](int m, R2 v) { row[fft::pad(m)] = v; });
        }
    }
    __syncthreads();
    for (int i = tid; i < TB * n * NY; i += 256) {
        const int c = i % TB, rest = i / TB, y = rest % NY, zi = rest / NY;
        const int kx = kxb + c;
        if (kx < nxh) spec[(size_t)zi * plane + (size_t)y * pitch + kx] = slab[(c * n + zi) * PY + fft::pad(y)];
    }
    if (mean_block) {
        const double nxy = (double)nx * (double)NY;
        for (int i = tid; i < nz; i += 256) {
            double x = 0.0;
            if (i == 0) {
                x = voltage;
            } else if (i < nz - 1) {
                for (int jz = 1; jz <= n; ++jz) {
                    const int lo = i < jz ? i : jz, hi = i < jz ? jz : i;
                    x -= (double)(lo * (n + 1 - hi)) * mrhs[jz - 1];
                }
                x = x / (double)(n + 1) / nxy;
            }
            mphi[i] = x;
            phi00[i] = x;
        }
        __syncthreads();
        for (int z = tid; z < nz; z += 256) {
            const int zc = z < 1 ? 1 : (z > nz - 2 ? nz - 2 : z);
            ez00[z] = 0.5 * (mphi[zc - 1] - mphi[zc + 1]) / dz;
        }
    }
}

// K3 of the split path: x[n + 64 m] = sum_j W_S^(-j m) b_j[n] from
// spl[j][kx][z - 1][n], Hermitian completion of two rows per transform,
// inverse x-FFT, phi' = Re / (NX NY) (odd_extract, poisson.cu:154-167).
template <typename R, int N, int S>
__global__ void __launch_bounds__(256)
poisson_rows_inv_split(const typename Cplx<R>::T *__restrict__ spl, R *__restrict__ phip,
                       const typename Cplx<R>::T *__restrict__ tw,
                       const typename Cplx<R>::T *__restrict__ twy, int nzi, int nxh,
    const PoissonPtrs *__restrict__ grp) {
    if (grp) {  // one instance of a group launch per blockIdx.z
        const PoissonPtrs &gp = grp[blockIdx.z];
        spl = (const typename Cplx<R>::T *)gp.spec;
        phip = (R *)gp.phip;
    }
    using R2 = typename Cplx<R>::T;
    constexpr int G = fft::Plan<N>::G, TB = per_block<N>(), P = tstride<N>();
    constexpr int NY = 64 * S, GB = 2 * TB / S;
    constexpr int NB = S == 1 ? 2 * TB : GB;  // consecutive n per block
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R2 *tws = reinterpret_cast<R2 *>(smem_raw);
    R2 *buf = tws + N;
    const int zi = blockIdx.y;
    const int tid = threadIdx.x;
    const int n0 = blockIdx.x * NB;
    load_twiddles<R, N>(tws, tw);
    // items (g, kx), g fastest (S = 1: g a transform, rows n0 + 2g, + 1):
    // b_j of the group's n at bin kx, the inverse radix-S DFT over j, and the
    // packed inputs Z = A + i B of its transforms at k = kx and k = N - kx
    // (Hermitian completion; the imaginary parts of the bins 0 and N/2 dropped)
    // every item's loads are issued before the first item is combined
    constexpr int NI = S == 1 ? TB : GB;
    constexpr int NIT = ((N / 2 + 1) * NI + 255) / 256;  // items per thread (nxh = N/2 + 1)
    constexpr int NL = S == 1 ? 2 : S;                   // loads per item
    R2 bv[NIT][NL];
#pragma unroll
    for (int t = 0; t < NIT; ++t) {
        const int i = tid + 256 * t;
        if (i < nxh * NI) {
            const int g = i % NI, kx = i / NI;
#pragma unroll
            for (int j = 0; j < NL; ++j)
                bv[t][j] = S == 1 ? spl[((size_t)kx * nzi + zi) * 64 + n0 + 2 * g + j]
                                  : spl[(((size_t)j * nxh + kx) * nzi + zi) * 64 + n0 + g];
        }
    }
#pragma unroll
    for (int t = 0; t < NIT; ++t) {
        const int i = tid + 256 * t;
        if (i >= nxh * NI) break;
        const int g = i % NI, kx = i / NI;
        R2 xm[NL];
        if constexpr (S == 1) {
            xm[0] = bv[t][0];
            xm[1] = bv[t][1];
        } else {
#pragma unroll
            for (int m = 0; m < S; ++m) {
                R2 acc = bv[t][0];
#pragma unroll
                for (int j = 1; j < S; ++j) acc = cadd(acc, mul_ws<S>(bv[t][j], S - (j * m) % S));
                xm[m] = acc;
            }
        }
        constexpr int NT = S == 1 ? 1 : S / 2;  // transforms per item
#pragma unroll
        for (int a2 = 0; a2 < NT; ++a2) {
            R2 A = S == 1 ? xm[0] : xm[a2], B = S == 1 ? xm[1] : xm[a2 + S / 2];
            const int tr = S == 1 ? g : g * (S / 2) + a2;
            if (kx == 0 || kx == N / 2) {
                A.y = 0;
                B.y = 0;
            }
            buf[tr * P + fft::pad(kx)] = R2{A.x - B.y, A.y + B.x};
            if (kx != 0 && kx != N / 2) buf[tr * P + fft::pad(N - kx)] = R2{A.x + B.y, B.x - A.y};
        }
    }
    __syncthreads();
    {
        const int tr = tid / G, jj = tid - tr * G;
        fft::run_tile<N, 1>(buf + tr * P, tws, jj);
    }
    const R norm = (R)(1.0 / ((double)N * (double)NY));
    R *pp = phip + (size_t)N * NY * (zi + 1);
    for (int i = tid; i < TB * N; i += 256) {
        const int t2 = i / N, x = i - t2 * N;
        int ya, yb, g, a;
        split_rows<S, TB>(t2, ya, yb, g, a);
        const R2 zv = buf[t2 * P + fft::pad(x)];
        pp[(size_t)N * ya + x] = zv.x * norm;
        pp[(size_t)N * yb + x] = zv.y * norm;
    }
}

// ---------------------------------------------------------------------------
// launcher
// ---------------------------------------------------------------------------

// Opt in to more than 48 KB of dynamic shared memory (to the device's
// maximum, see allow_max_dynamic_smem).  Skipped while the stream is being
// captured into a graph: the attribute is set by the first, uncaptured launch
// on the device.
template <typename K>
static cudaError_t set_smem(K kern, size_t bytes, cudaStream_t s) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &st);
    if (e != cudaSuccess) return e;
    if (st != cudaStreamCaptureStatusNone) return cudaSuccess;
    return allow_max_dynamic_smem(kern);
}

bool poisson_fast_size(int n) {
    return n == 48 || n == 64 || n == 80 || n == 96 || n == 128 || n == 256 || n == 512;
}
// the sizes of the split-y path's x rows and z transforms
static bool split_size(int n) { return n == 64 || n == 128 || n == 256 || n == 512; }

size_t zdst_rt_smem(int L, int tb, size_t rsize) {
    const int n = L / 2 - 1, nz = n + 2;
    return (size_t)(2 * tb + 1) * L * 2 * rsize + sizeof(double) * (size_t)(n + nz) +
           (size_t)tb * rsize + 16;
}

template <typename R, int N>
static cudaError_t rows_fwd_fast(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = per_block<N>();
    const size_t sm = sizeof(R2) * ((size_t)N + (size_t)TB * tstride<N>());
    cudaError_t e = set_smem(poisson_rows_fwd_fast<R, N>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.ny + 2 * TB - 1) / (2 * TB), a.nz - 2, a.ngrp);
    poisson_rows_fwd_fast<R, N><<<grid, 256, sm, s>>>((const R *)a.q, (R2 *)a.spec, a.rowsum,
                                                       (const R2 *)a.twx, a.qmean,
                                                       a.ny, a.nxh, a.pitch, a.eps, a.grp);
    return cudaGetLastError();
}
template <typename R, int N>
static cudaError_t rows_inv_fast(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = per_block<N>();
    const size_t sm = sizeof(R2) * ((size_t)N + (size_t)TB * tstride<N>());
    cudaError_t e = set_smem(poisson_rows_inv_fast<R, N>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.ny + 2 * TB - 1) / (2 * TB), a.nz - 2, a.ngrp);
    poisson_rows_inv_fast<R, N><<<grid, 256, sm, s>>>((const R2 *)a.spec, (R *)a.phip,
                                                       (const R2 *)a.twx, a.ny, a.nxh, a.pitch, a.grp);
    return cudaGetLastError();
}
template <typename R, int N, int S>
static cudaError_t cols_fast(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = per_block<N>();
    const size_t sm = sizeof(R2) * ((size_t)N + (size_t)TB * tstride<N>());
    cudaError_t e = set_smem(poisson_cols_fast<R, N, S>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nxh + TB - 1) / TB, a.nz - 2, a.ngrp);
    poisson_cols_fast<R, N, S><<<grid, 256, sm, s>>>((R2 *)a.spec, (const R2 *)a.twy, a.nxh,
                                                      a.pitch, a.rowsum, a.planesum, a.grp);
    return cudaGetLastError();
}

template <typename R>
static cudaError_t rows_fwd(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    switch (a.nx) {
        case 48: return rows_fwd_fast<R, 48>(a, s);
        case 64: return rows_fwd_fast<R, 64>(a, s);
        case 80: return rows_fwd_fast<R, 80>(a, s);
        case 96: return rows_fwd_fast<R, 96>(a, s);
        case 128: return rows_fwd_fast<R, 128>(a, s);
        case 256: return rows_fwd_fast<R, 256>(a, s);
        case 512: return rows_fwd_fast<R, 512>(a, s);
        default: break;
    }
    const int rows = a.rows_per_block;
    const size_t sm = (size_t)(2 * rows + 1) * a.nx * sizeof(R2);
    cudaError_t e = set_smem(poisson_rows_fwd<R>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.ny + 2 * rows - 1) / (2 * rows), a.nz - 2, a.ngrp);
    poisson_rows_fwd<R><<<grid, 256, sm, s>>>((const R *)a.q, (R2 *)a.spec, a.rowsum,
                                               (const R2 *)a.twx, a.qmean, a.px,
                                               a.nx, a.ny, a.nxh, a.pitch, rows, a.eps, a.grp);
    return cudaGetLastError();
}
template <typename R>
static cudaError_t rows_inv(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    switch (a.nx) {
        case 48: return rows_inv_fast<R, 48>(a, s);
        case 64: return rows_inv_fast<R, 64>(a, s);
        case 80: return rows_inv_fast<R, 80>(a, s);
        case 96: return rows_inv_fast<R, 96>(a, s);
        case 128: return rows_inv_fast<R, 128>(a, s);
        case 256: return rows_inv_fast<R, 256>(a, s);
        case 512: return rows_inv_fast<R, 512>(a, s);
        default: break;
    }
    const int rows = a.rows_per_block;
    const size_t sm = (size_t)(2 * rows + 1) * a.nx * sizeof(R2);
    cudaError_t e = set_smem(poisson_rows_inv<R>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.ny + 2 * rows - 1) / (2 * rows), a.nz - 2, a.ngrp);
    poisson_rows_inv<R><<<grid, 256, sm, s>>>((const R2 *)a.spec, (R *)a.phip,
                                               (const R2 *)a.twx, a.px, a.nx, a.ny, a.nxh,
                                               a.pitch, rows, a.grp);
    return cudaGetLastError();
}
template <typename R, int S>
static cudaError_t cols(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    switch (a.ny) {
        case 48: return cols_fast<R, 48, S>(a, s);
        case 64: return cols_fast<R, 64, S>(a, s);
        case 80: return cols_fast<R, 80, S>(a, s);
        case 96: return cols_fast<R, 96, S>(a, s);
        case 128: return cols_fast<R, 128, S>(a, s);
        case 256: return cols_fast<R, 256, S>(a, s);
        case 512: return cols_fast<R, 512, S>(a, s);
        default: break;
    }
    const int cc = a.cols_per_block;
    const size_t sm = (size_t)(2 * cc + 1) * a.ny * sizeof(R2);
    cudaError_t e = set_smem(poisson_cols<R>, sm, s);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nxh + cc - 1) / cc, a.nz - 2, a.ngrp);
    poisson_cols<R><<<grid, 256, sm, s>>>((R2 *)a.spec, (const R2 *)a.twy, a.py, a.ny, a.nxh,
                                           a.pitch, cc, (R)S, S < 0 ? a.rowsum : nullptr,
                                           S < 0 ? a.planesum : nullptr, a.grp);
    return cudaGetLastError();
}

template <typename R, int L>
static cudaError_t zdst(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = 256 / fft::WPlan<L>::G;  // modes per block, as poisson_zdst
    const size_t sm = sizeof(R2) * ((size_t)L + (size_t)TB * tstride<L>());
    cudaError_t e = set_smem(poisson_zdst<R, L>, sm, s);
    if (e != cudaSuccess) return e;
    const int modes = a.nxh * a.ny;
    const R2 *tw = (const R2 *)a.twz;
    poisson_zdst<R, L><<<dim3((modes + TB - 1) / TB, 1, a.ngrp), 256, sm, s>>>(
        (R2 *)a.spec, tw, (const R *)(tw + L), a.planesum, a.qmean, a.phi00, a.ez00, a.nx, a.ny,
        a.nxh, a.pitch, a.dz, a.eps, a.voltage, 2.0 * M_PI / a.lx, 2.0 * M_PI / a.ly, a.grp);
    return cudaGetLastError();
}

// ---- the fused y transform and z solve (poisson_yz) ----

template <typename R, int NY, int L>
static cudaError_t yz_nl(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr size_t sm = yz_smem<R, NY, L>();
    cudaError_t e = set_smem(poisson_yz<R, NY, L>, sm, s);
    if (e != cudaSuccess) return e;
    constexpr int TB = yz_cols<R, NY, L>();
    const R2 *tw = (const R2 *)a.twz;
    poisson_yz<R, NY, L><<<dim3((a.nxh + TB - 1) / TB, 1, a.ngrp), 256, sm, s>>>(
        (R2 *)a.spec, (const R2 *)a.twy, tw, (const R *)(tw + L), a.rowsum, a.planesum, a.qmean,
        a.phi00, a.ez00, a.nx, a.nxh, a.pitch, a.dz, a.eps, a.voltage, 2.0 * M_PI / a.lx,
        2.0 * M_PI / a.ly, a.grp);
    return cudaGetLastError();
}
template <typename R, int NY>
static cudaError_t yz_n(const PoissonArgs &a, cudaStream_t s) {
    switch (2 * (a.nz - 1)) {
        case 48: return yz_nl<R, NY, 48>(a, s);
        case 64: return yz_nl<R, NY, 64>(a, s);
        case 80: return yz_nl<R, NY, 80>(a, s);
        case 96: return yz_nl<R, NY, 96>(a, s);
        default: return yz_nl<R, NY, 128>(a, s);
    }
}
template <typename R>
static cudaError_t yz_all(const PoissonArgs &a, cudaStream_t s) {
    switch (a.ny) {
        case 48: return yz_n<R, 48>(a, s);
        case 80: return yz_n<R, 80>(a, s);
        default: return yz_n<R, 96>(a, s);
    }
}
// whether poisson_yz serves a grid: NY = 48, 80 or 96 (the widths the split-y
// path does not take), L = 2 (NZ - 1) = 48, 64, 80, 96 or 128, the sine
// transform z solve, and the split-y choice (ehd_tuning.poisson_path = 0)
template <typename R>
static bool yz_usable(const PoissonArgs &a) {
    const int L = 2 * (a.nz - 1);
    return a.split && a.twz && (a.ny == 48 || a.ny == 80 || a.ny == 96) &&
           (L == 48 || L == 64 || L == 80 || L == 96 || L == 128);
}
template <typename R, int NY>
static cudaError_t prepare_yz_n(int L) {
    switch (L) {
        case 48: return allow_max_dynamic_smem(poisson_yz<R, NY, 48>);
        case 64: return allow_max_dynamic_smem(poisson_yz<R, NY, 64>);
        case 80: return allow_max_dynamic_smem(poisson_yz<R, NY, 80>);
        case 96: return allow_max_dynamic_smem(poisson_yz<R, NY, 96>);
        default: return allow_max_dynamic_smem(poisson_yz<R, NY, 128>);
    }
}

// ---- split-y path ----

template <typename R, int N, int S>
constexpr size_t rows_inv_split_smem() {
    constexpr int TB = per_block<N>();
    return sizeof(typename Cplx<R>::T) * ((size_t)N + (size_t)TB * tstride<N>());
}

template <typename R, int N, int S>
static cudaError_t split_rows_fwd(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = per_block<N>(), NB = S == 1 ? 2 * TB : 2 * TB / S;
    const size_t sm = sizeof(R2) * ((size_t)N + (size_t)TB * tstride<N>());
    cudaError_t e = set_smem(poisson_rows_fwd_split<R, N, S>, sm, s);
    if (e != cudaSuccess) return e;
    poisson_rows_fwd_split<R, N, S><<<dim3(64 / NB, a.nz - 2, a.ngrp), 256, sm, s>>>(
        (const R *)a.q, (R2 *)a.spec, a.rowsum, (const R2 *)a.twx, (const R2 *)a.twy, a.qmean,
        a.nz - 2, a.nxh, a.eps, a.grp);
    return cudaGetLastError();
}
template <typename R, int N, int S>
static cudaError_t split_rows_inv(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr int TB = per_block<N>(), NB = S == 1 ? 2 * TB : 2 * TB / S;
    constexpr size_t sm = rows_inv_split_smem<R, N, S>();
    cudaError_t e = set_smem(poisson_rows_inv_split<R, N, S>, sm, s);
    if (e != cudaSuccess) return e;
    poisson_rows_inv_split<R, N, S><<<dim3(64 / NB, a.nz - 2, a.ngrp), 256, sm, s>>>(
        (const R2 *)a.spec, (R *)a.phip, (const R2 *)a.twx, (const R2 *)a.twy, a.nz - 2, a.nxh, a.grp);
    return cudaGetLastError();
}
template <typename R, int L, int S>
static cudaError_t split_slab(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    constexpr size_t sm = slab_smem<R, L>();
    cudaError_t e = set_smem(poisson_slab<R, L, S>, sm, s);
    if (e != cudaSuccess) return e;
    // one block more than kx columns: block x = 0 solves the mean mode
    poisson_slab<R, L, S><<<dim3(a.nxh + 1, S, a.ngrp), 256, sm, s>>>(
        (R2 *)a.spec, (const R2 *)a.twy, (const R *)a.cps, a.rowsum, a.planesum, a.qmean,
        a.phi00, a.ez00, a.nx, a.nxh, a.dz, a.eps, a.voltage, a.grp);
    return cudaGetLastError();
}

template <typename R, int N, int S>
static cudaError_t split_all_n(const PoissonArgs &a, cudaStream_t s) {
    cudaError_t e = split_rows_fwd<R, N, S>(a, s);
    if (e != cudaSuccess) return e;
    switch (2 * (a.nz - 1)) {
        case 64: e = split_slab<R, 64, S>(a, s); break;
        case 128: e = split_slab<R, 128, S>(a, s); break;
        case 256: e = split_slab<R, 256, S>(a, s); break;
        default: e = split_slab<R, 512, S>(a, s); break;
    }
    if (e != cudaSuccess) return e;
    return split_rows_inv<R, N, S>(a, s);
}
template <typename R, int S>
static cudaError_t split_all(const PoissonArgs &a, cudaStream_t s) {
    switch (a.nx) {
        case 64: return split_all_n<R, 64, S>(a, s);
        case 128: return split_all_n<R, 128, S>(a, s);
        case 256: return split_all_n<R, 256, S>(a, s);
        default: return split_all_n<R, 512, S>(a, s);
    }
}

template <typename R, int S>
static size_t split_slab_smem(int L) {
    switch (L) {
        case 64: return slab_smem<R, 64>();
        case 128: return slab_smem<R, 128>();
        case 256: return slab_smem<R, 256>();
        default: return slab_smem<R, 512>();
    }
}

// whether the split-y path serves a grid: NX a compile-time FFT size,
// NY = 64 S (S = 1, 2, 4, 8), 2 (NZ - 1) one of the slab kernel's sizes, and
// the slab with its pivots in shared memory
template <typename R>
static bool split_grid(int nx, int ny, int nz) {
    if (!split_size(nx) || !split_size(2 * (nz - 1))) return false;
    const int S = ny / 64;
    if (ny % 64 != 0 || (S != 1 && S != 2 && S != 4 && S != 8)) return false;
    const int L = 2 * (nz - 1);
    size_t sm = 0;
    switch (S) {
        case 1: sm = split_slab_smem<R, 1>(L); break;
        case 2: sm = split_slab_smem<R, 2>(L); break;
        case 4: sm = split_slab_smem<R, 4>(L); break;
        default: sm = split_slab_smem<R, 8>(L); break;
    }
    return sm + 4 * 1024 <= 227 * 1024;  // with the static shared arrays
}
bool poisson_split_grid(int nx, int ny, int nz, size_t rsize) {
    return rsize == 8 ? split_grid<double>(nx, ny, nz) : split_grid<float>(nx, ny, nz);
}
template <typename R>
bool poisson_split_usable(const PoissonArgs &a) {
    return a.cps && split_grid<R>(a.nx, a.ny, a.nz);
}

// The split path's shared-memory attributes, set before any stream capture
// (a launch inside a capture does not set them, see set_smem).
template <typename R, int N, int L, int S>
static cudaError_t prepare_split_nls() {
    cudaError_t e = allow_max_dynamic_smem(poisson_rows_fwd_split<R, N, S>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_slab<R, L, S>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_rows_inv_split<R, N, S>);
    return e;
}
template <typename R, int N, int S>
static cudaError_t prepare_split_ns(int L) {
    switch (L) {
        case 64: return prepare_split_nls<R, N, 64, S>();
        case 128: return prepare_split_nls<R, N, 128, S>();
        case 256: return prepare_split_nls<R, N, 256, S>();
        default: return prepare_split_nls<R, N, 512, S>();
    }
}
template <typename R, int S>
static cudaError_t prepare_split_s(int nx, int L) {
    switch (nx) {
        case 64: return prepare_split_ns<R, 64, S>(L);
        case 128: return prepare_split_ns<R, 128, S>(L);
        case 256: return prepare_split_ns<R, 256, S>(L);
        default: return prepare_split_ns<R, 512, S>(L);
    }
}
template <typename R, int N>
static cudaError_t prepare_fast_n() {
    cudaError_t e = allow_max_dynamic_smem(poisson_rows_fwd_fast<R, N>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_rows_inv_fast<R, N>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_cols_fast<R, N, -1>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_cols_fast<R, N, 1>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_zdst<R, N>);
    return e;
}
template <typename R>
static cudaError_t prepare_fast(int n) {
    switch (n) {
        case 48: return prepare_fast_n<R, 48>();
        case 64: return prepare_fast_n<R, 64>();
        case 80: return prepare_fast_n<R, 80>();
        case 96: return prepare_fast_n<R, 96>();
        case 128: return prepare_fast_n<R, 128>();
        case 256: return prepare_fast_n<R, 256>();
        case 512: return prepare_fast_n<R, 512>();
        default: return cudaSuccess;
    }
}
// Every Poisson kernel that a context of this grid can launch, under any
// tuning, may use the device's whole opt-in shared memory: the attribute
// cannot be set by a launch inside a stream capture (set_smem), and the
// batch graphs capture every launch.
template <typename R>
cudaError_t prepare_poisson(const PoissonArgs &a) {
    cudaError_t e = allow_max_dynamic_smem(poisson_rows_fwd<R>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_rows_inv<R>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_cols<R>);
    if (e == cudaSuccess) e = allow_max_dynamic_smem(poisson_zdst_rt<R>);
    if (e == cudaSuccess) e = prepare_fast<R>(a.nx);
    if (e == cudaSuccess) e = prepare_fast<R>(a.ny);
    if (e == cudaSuccess) e = prepare_fast<R>(2 * (a.nz - 1));
    if (e == cudaSuccess && a.twz && (a.ny == 48 || a.ny == 80 || a.ny == 96)) {
        const int L = 2 * (a.nz - 1);
        if (L == 48 || L == 64 || L == 80 || L == 96 || L == 128)
            e = a.ny == 48 ? prepare_yz_n<R, 48>(L)
                           : (a.ny == 80 ? prepare_yz_n<R, 80>(L) : prepare_yz_n<R, 96>(L));
    }
    if (e != cudaSuccess || !poisson_split_usable<R>(a)) return e;
    const int L = 2 * (a.nz - 1);
    switch (a.ny / 64) {
        case 1: return prepare_split_s<R, 1>(a.nx, L);
        case 2: return prepare_split_s<R, 2>(a.nx, L);
        case 4: return prepare_split_s<R, 4>(a.nx, L);
        default: return prepare_split_s<R, 8>(a.nx, L);
    }
}
template cudaError_t prepare_poisson<float>(const PoissonArgs &);
template cudaError_t prepare_poisson<double>(const PoissonArgs &);

template <typename R>
cudaError_t launch_poisson(const PoissonArgs &a, cudaStream_t s) {
    using R2 = typename Cplx<R>::T;
    cudaError_t e;
    if (a.split && poisson_split_usable<R>(a)) {
        switch (a.ny / 64) {
            case 1: return split_all<R, 1>(a, s);
            case 2: return split_all<R, 2>(a, s);
            case 4: return split_all<R, 4>(a, s);
            default: return split_all<R, 8>(a, s);
        }
    }
    if ((e = rows_fwd<R>(a, s)) != cudaSuccess) return e;
    if (yz_usable<R>(a)) {
        if ((e = yz_all<R>(a, s)) != cudaSuccess) return e;
        return rows_inv<R>(a, s);
    }
    if ((e = cols<R, -1>(a, s)) != cudaSuccess) return e;
    if (a.twz && poisson_fast_size(2 * (a.nz - 1))) {
        switch (2 * (a.nz - 1)) {
            case 48: e = zdst<R, 48>(a, s); break;
            case 64: e = zdst<R, 64>(a, s); break;
            case 80: e = zdst<R, 80>(a, s); break;
            case 96: e = zdst<R, 96>(a, s); break;
            case 128: e = zdst<R, 128>(a, s); break;
            case 256: e = zdst<R, 256>(a, s); break;
            default: e = zdst<R, 512>(a, s); break;
        }
        if (e != cudaSuccess) return e;
    } else if (a.twz && !(a.thomas && a.cpt)) {
        const int modes = a.nxh * a.ny;
        const int L = 2 * (a.nz - 1);
        const size_t sm = zdst_rt_smem(L, a.ztb, sizeof(R));
        if ((e = set_smem(poisson_zdst_rt<R>, sm, s)) != cudaSuccess) return e;
        const R2 *tw = (const R2 *)a.twz;
        poisson_zdst_rt<R><<<dim3((modes + a.ztb - 1) / a.ztb, 1, a.ngrp), 256, sm, s>>>(
            (R2 *)a.spec, tw, (const R *)(tw + L), a.pz, a.planesum, a.qmean, a.phi00, a.ez00,
            a.nx, a.ny, a.nxh, a.pitch, a.ztb, a.dz, a.eps, a.voltage, 2.0 * M_PI / a.lx,
            2.0 * M_PI / a.ly, a.grp);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    } else {
        const int modes = a.nxh * a.ny;
        poisson_zsolve<R><<<dim3((modes + 127) / 128, 1, a.ngrp), 128, 0, s>>>(
            (R2 *)a.spec, a.cpt, a.dpw, a.planesum, a.qmean, a.phi00, a.ez00, a.nx, a.ny, a.nz,
            a.nxh, a.pitch, a.dz, a.eps, a.voltage, a.grp);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = cols<R, 1>(a, s)) != cudaSuccess) return e;
    if ((e = rows_inv<R>(a, s)) != cudaSuccess) return e;
    return cudaSuccess;
}

template cudaError_t launch_poisson<float>(const PoissonArgs &, cudaStream_t);
template cudaError_t launch_poisson<double>(const PoissonArgs &, cudaStream_t);

}  // namespace ehd
