// noalloc.cu -- the Poisson solve and E field on caller-owned device buffers,
// for callers that cannot allocate device memory.
//
// Some callers of this library run where device allocation is not theirs to
// do: a host framework that owns every allocation on the GPU through its own
// pool, a process that must not grow its footprint after start-up, or code
// between the launches of another library's pipeline where a cudaMalloc would
// synchronise the device.  ehd_poisson_noalloc serves them: it solves the same
// discrete Poisson problem as the time step (FFT in x and y, FP64 tridiagonal
// solve in z, E = -grad(phi)) on device arrays the caller passes in, and keeps
// its working storage in one file-scope device array of fixed size instead of
// allocating.  It calls no cudaMalloc, cudaFree or other allocating routine,
// on the device or on the host.
//
// The array costs EHD_NOALLOC_SCRATCH_BYTES of device memory on each GPU the
// entry point is used on, until the process exits.  Under CUDA's lazy module
// loading (the default) the driver commits it when the first call on a device
// looks up its address, so that first call is itself a device allocation by
// the driver: make it at start-up, before any stream capture.  With
// CUDA_MODULE_LOADING=EAGER the array is committed on every GPU when the
// library's module loads.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "common.cuh"
#include "ehd.h"
#include "kernels.h"

namespace ehd {
namespace {

// The working storage.  In host code this name is a host-side stand-in, not a
// device address: host code obtains the address with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[EHD_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// per device: the array's address and the context it was looked up in (a
// cudaDeviceReset makes a new primary context, where the module reloads and
// the array may move)
void *g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};

// The calling thread's current driver context, through the runtime's driver
// entry point (the library links only the runtime).
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext *);
    static Fn fn = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult st{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &st) ==
                cudaSuccess && st == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<Fn>(p);
        looked_up = true;
    }
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

bool only_235(int n) {
    if (n < 1) return false;
    for (int f : {2, 3, 5})
        while (n % f == 0) n /= f;
    return n == 1;
}

FftPlan plan_of(int n) {
    FftPlan p{};
    p.n = n;
    while (n % 4 == 0) { p.rad[p.nrad++] = 4; n /= 4; }
    while (n % 2 == 0) { p.rad[p.nrad++] = 2; n /= 2; }
    while (n % 3 == 0) { p.rad[p.nrad++] = 3; n /= 3; }
    while (n % 5 == 0) { p.rad[p.nrad++] = 5; n /= 5; }
    return p;
}

// exp(-2 pi i k / n), FP64
__global__ void twiddle_kernel(double2 *tw, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)k / (double)n, &s, &c);
        tw[k] = make_double2(c, s);
    }
}

// Thomas pivots per mode, the same table as the context's (api.cu):
// beta = 2 + (kx^2 + ky^2) dz^2, cp_0 = -1/beta, cp_i = 1/(-beta - cp_{i-1}).
__global__ void pivot_kernel(double *cpt, int nx, int ny, int nz, double lx, double ly,
                             double dz) {
    const int nxh = nx / 2 + 1;
    const int modes = nxh * ny;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= modes) return;
    const int j = m / nxh, i = m - j * nxh;
    const double kx = (double)i * 2.0 * M_PI / lx;
    const double ky = (j <= ny / 2 ? (double)j : (double)j - ny) * 2.0 * M_PI / ly;
    const double beta = 2.0 + (kx * kx + ky * ky) * dz * dz;
    double prev = 0.0;
    for (int z = 0; z < nz - 2; ++z) {
        prev = 1.0 / (-beta - prev);
        cpt[(size_t)z * modes + m] = prev;
    }
}

// E = -grad(phi) from phi' (in phi) and phi00, central differences with the
// electrode copy of Ez (gpu_efield, gpu_bc, poisson.cu:44-73).
__global__ void efield_kernel(const double *__restrict__ phip, const double *__restrict__ phi00,
                              double *__restrict__ ex, double *__restrict__ ey,
                              double *__restrict__ ez, int nx, int ny, int nz, double dx,
                              double dy, double dz) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    auto idx = [&](int xx, int yy, int zz) {
        return (size_t)xx + (size_t)nx * ((size_t)yy + (size_t)ny * zz);
    };
    auto phi = [&](int xx, int yy, int zz) { return phi00[zz] + phip[idx(xx, yy, zz)]; };
    const int xm = (nx + x - 1) % nx, xp = (x + 1) % nx;
    const int ym = (ny + y - 1) % ny, yp = (y + 1) % ny;
    const int zc = z < 1 ? 1 : (z > nz - 2 ? nz - 2 : z);
    const size_t i = idx(x, y, z);
    ex[i] = 0.5 * (phi(xm, y, z) - phi(xp, y, z)) / dx;
    ey[i] = 0.5 * (phi(x, ym, z) - phi(x, yp, z)) / dy;
    ez[i] = 0.5 * (phi(x, y, zc - 1) - phi(x, y, zc + 1)) / dz;
}

// phi = phi00(z) + phi' in place (phi00 carries V and 0 on the electrodes).
__global__ void phi_kernel(double *__restrict__ phi, const double *__restrict__ phi00,
                           long long nxy, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) phi[i] = phi00[i / nxy] + phi[i];
}

}  // namespace
}  // namespace ehd

using namespace ehd;

extern "C" int ehd_poisson_noalloc(const ehd_params *p, const double *q, double *phi,
                                   double *ex, double *ey, double *ez, void *stream) {
    if (!p || !q || !phi || !ex || !ey || !ez)
        return set_error(EHD_ERR_INVALID, "ehd_poisson_noalloc: NULL argument");
    if (p->nx < 1 || p->ny < 1 || p->nz < 4 || !only_235(p->nx) || !only_235(p->ny) ||
        !(p->dx > 0) || !(p->dy > 0) || !(p->dz > 0) || !(p->lx > 0) || !(p->ly > 0) ||
        !(p->eps > 0))
        return set_error(EHD_ERR_INVALID, "ehd_poisson_noalloc: invalid grid or parameters");
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int nxh = nx / 2 + 1, pitch = (nxh + 15) / 16 * 16;
    const size_t modes = (size_t)nxh * ny;
    // scratch layout
    const size_t b_spec = align256(sizeof(double2) * (size_t)(nz - 2) * ny * pitch);
    const size_t b_cpt = align256(sizeof(double) * modes * (size_t)(nz - 2));
    const size_t b_dpw = align256(sizeof(double2) * modes * (size_t)(nz - 2));
    const size_t b_twx = align256(sizeof(double2) * nx), b_twy = align256(sizeof(double2) * ny);
    const size_t b_row = align256(sizeof(double) * (size_t)(nz - 2) * ny);
    const size_t b_z = align256(sizeof(double) * nz);
    const size_t b_qm = align256(sizeof(double) * 2 * nz);
    const size_t total = b_spec + b_cpt + b_dpw + b_twx + b_twy + b_row + 3 * b_z + b_qm;
    if (total > EHD_NOALLOC_SCRATCH_BYTES || (long long)nx * ny * nz > (1LL << 31))
        return set_error(EHD_ERR_INVALID,
                         "ehd_poisson_noalloc: the grid needs more working storage than the "
                         "EHD_NOALLOC_SCRATCH_BYTES (64 MiB) the entry point has; use ehd_poisson");
    // the shared-memory FFT limits of the context path apply as well
    if ((size_t)2 * nx * 16 > 200 * 1024 || (size_t)2 * ny * 16 > 200 * 1024)
        return set_error(EHD_ERR_INVALID, "ehd_poisson_noalloc: nx or ny too large");

    {
        // an error left pending by the caller's earlier work is reported as
        // such, and left pending (not consumed by this call's launch checks)
        const cudaError_t pending = cudaPeekAtLastError();
        if (pending != cudaSuccess)
            return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: a CUDA error from earlier work "
                                           "is pending; nothing was launched");
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: no usable current device");
    unsigned char *base = nullptr;
    {
        // first call on this device (in this context): the device address of
        // the array
        std::lock_guard<std::mutex> lk(g_mu);
        const CUcontext ctx = current_context();
        if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
            void *ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
                return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: cudaGetSymbolAddress failed");
            g_scratch_addr[dev] = ptr;
            g_scratch_ctx[dev] = ctx;
        }
        base = (unsigned char *)g_scratch_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    PoissonArgs a{};
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.nxh = nxh;
    a.pitch = pitch;
    {
        int rows = 16;
        while (rows > 1 && (size_t)2 * rows * nx * 16 > 64 * 1024) rows >>= 1;
        int cols = 8;
        while (cols > 1 && (size_t)2 * cols * ny * 16 > 160 * 1024) cols >>= 1;
        a.rows_per_block = rows;
        a.cols_per_block = cols;
    }
    a.px = plan_of(nx);
    a.py = plan_of(ny);
    unsigned char *cur = base;
    a.spec = cur;                       cur += b_spec;
    double *cpt = (double *)cur;        cur += b_cpt;
    a.dpw = (double2 *)cur;             cur += b_dpw;
    double2 *twx = (double2 *)cur;      cur += b_twx;
    double2 *twy = (double2 *)cur;      cur += b_twy;
    a.rowsum = (double *)cur;           cur += b_row;
    a.planesum = (double *)cur;         cur += b_z;
    a.phi00 = (double *)cur;            cur += b_z;
    a.ez00 = (double *)cur;             cur += b_z;
    double *qmean = (double *)cur;      cur += b_qm;
    a.cpt = cpt;
    a.twx = twx;
    a.twy = twy;
    a.q = q;
    a.qmean = qmean;
    a.phip = phi;  // phi' is built in the caller's phi array, then completed
    a.eps = p->eps;
    a.voltage = p->voltage;
    a.dz = p->dz;

    const size_t nxy = (size_t)nx * ny;
    // every region the solve reads before writing is set here: the tables,
    // the zero reference charge, and phi' = 0 on both electrodes
    twiddle_kernel<<<(nx + 255) / 256, 256, 0, s>>>(twx, nx);
    twiddle_kernel<<<(ny + 255) / 256, 256, 0, s>>>(twy, ny);
    pivot_kernel<<<(unsigned)((modes + 127) / 128), 128, 0, s>>>(cpt, nx, ny, nz, p->lx, p->ly,
                                                                  p->dz);
    if (cudaGetLastError() != cudaSuccess)
        return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: table kernels failed to launch");
    if (cudaMemsetAsync(qmean, 0, sizeof(double) * 2 * nz, s) != cudaSuccess ||
        cudaMemsetAsync(phi, 0, sizeof(double) * nxy, s) != cudaSuccess ||
        cudaMemsetAsync(phi + (size_t)(nz - 1) * nxy, 0, sizeof(double) * nxy, s) != cudaSuccess)
        return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: cudaMemsetAsync failed");
    if (launch_poisson<double>(a, s) != cudaSuccess)
        return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: Poisson kernels failed to launch");
    dim3 blk(nx >= 128 ? 128 : 32), grd((nx + blk.x - 1) / blk.x, ny, nz);
    efield_kernel<<<grd, blk, 0, s>>>(phi, a.phi00, ex, ey, ez, nx, ny, nz, p->dx, p->dy, p->dz);
    const long long n = (long long)nxy * nz;
    phi_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(phi, a.phi00, (long long)nxy, n);
    if (cudaGetLastError() != cudaSuccess)
        return set_error(EHD_ERR_CUDA, "ehd_poisson_noalloc: field kernels failed to launch");
    return EHD_OK;
}
