// common.cuh -- lattice tables, per-step constants and storage conversions
// shared by the step kernels.
//
// D3Q27 in the reference's numbering: population d at node x is pulled from
// x - e_d (gpu_stream, LBM.cu:1225-1250); opposite pairs are (2k-1, 2k);
// weights 8/27, 2/27, 1/54, 1/216 (LBM.h:73-76).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ehd {

constexpr int Q = 27;

__host__ __device__ constexpr int ex_of(int d) {
    constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1,
                          1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[d];
}
__host__ __device__ constexpr int ey_of(int d) {
    constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1,
                          0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[d];
}
__host__ __device__ constexpr int ez_of(int d) {
    constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0,
                          -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[d];
}
__host__ __device__ constexpr int opp_of(int d) { return d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1); }
__host__ __device__ constexpr double w_of(int d) {
    return d == 0 ? 8.0 / 27.0 : (d <= 6 ? 2.0 / 27.0 : (d <= 18 ? 1.0 / 54.0 : 1.0 / 216.0));
}
// sign of the moving upper wall term (LBM.cu:1145-1170); direction 3 gets +,
// direction 4 nothing, as the reference writes it.
__host__ __device__ constexpr int mw_sign_of(int d) {
    constexpr int t[Q] = {0, 1, -1, 1, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1,
                          1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[d];
}

// Everything a step kernel needs, derived once on the host in FP64 from
// ehd_params (formulas of LBM.cu:297-302, 688, 1017-1018, 1137-1139).
struct StepConst {
    int nx, ny, nz;
    int pad_;
    long long nxy, n;         // nodes per plane, nodes
    double dt, cfl, cs2;
    double cflinv, cflinv2;   // 1/CFL, 1/(CFL^2 cs^2)
    double tw0rp, tw0rm;      // omega_+ dt, omega_- dt for f
    double tw0cp, tw0cm;      // omega_c+ dt, omega_c- dt for g
    // The same four rates split as rate = hi - lo, applied as hi*X - lo*X:
    // hi = 2, lo = 2 - rate for an over-relaxed rate (rate >= 1), so that the
    // small complement 2 - rate, which sets the transport coefficient
    // (1/rate - 1/2), keeps full relative precision in FP32; hi = rate, lo = 0
    // otherwise.  Order: rp, rm, cp, cm.
    double rate_hi[4], rate_lo[4];
    double sp, sm;            // 1 - dt omega_+/2, 1 - dt omega_-/2
    double rho0, q0, K, exf;
    double inv2dx, inv2dy, inv2dz;  // 0.5/dx, 0.5/dy, 0.5/dz
    double mw[Q];             // moving-wall increment per direction at z=nz-1
};

// weight class: 0 rest, 1 axis (2/27), 2 face diagonal (1/54), 3 body diagonal (1/216)
__host__ __device__ constexpr int cls_of(int d) { return d == 0 ? 0 : (d <= 6 ? 1 : (d <= 18 ? 2 : 3)); }

// Storage tag of the mixed mode: flow populations f as FP16 deviations,
// charge populations g as FP32 deviations (the charge, the Poisson source,
// keeps FP32 storage; see PopT).
struct Mix16 {};

// The storage types of the two population sets for a storage tag T: both T,
// except for Mix16.
template <typename T> struct PopT {
    using F = T;
    using G = T;
};
template <> struct PopT<Mix16> {
    using F = __half;
    using G = float;
};

// Per-direction base pointers of the two population buffers, passed by value
// so each access is a 32-bit node offset from a kernel-parameter base.
template <typename T>
struct PopPtrs {
    const typename PopT<T>::F *fa[Q];
    typename PopT<T>::F *fb[Q];
    const typename PopT<T>::G *ha[Q];
    typename PopT<T>::G *hb[Q];
};

// The step constants in the compute type, with the per-weight-class factors
// of the collision precomputed (see lbm_step_kernel).
template <typename R>
struct KConst {
    int nx, ny, nz;
    unsigned nxy;
    R dt_half, cflinv, inv_cs2, inv_cs2cfl;
    R rate_hi[4], rate_lo[4];
    R q0, K, exf;
    R inv2dx, inv2dy, inv2dz;
    R w[4];
    R c1[4];  // dt sp w cflinv2 CFL   (times cu eF)
    R c2[4];  // dt sm (w/cs2) cflinv  (times eF)
    R c3[4];  // dt sp (w/cs2)         (times u.F)
    R mw[Q];
};

// ---- storage types ---------------------------------------------------------
// Opt a kernel in to the largest dynamic shared memory the device allows.
// The attribute belongs to the function, not to a context of this library, so
// it is never set to one context's size: a smaller value set for one grid
// would make another context's larger launch invalid.
template <typename K>
inline cudaError_t allow_max_dynamic_smem(K kern) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - (int)fa.sharedSizeBytes);
    return e;
}

template <typename T> struct Store;
template <> struct Store<double> {
    __device__ __forceinline__ static double ld(const double *p) { return __ldg(p); }
    __device__ __forceinline__ static double lds(const double *p) { return *p; }
    __device__ __forceinline__ static void st(double *p, double v) { *p = v; }
};
template <> struct Store<float> {
    __device__ __forceinline__ static float ld(const float *p) { return __ldg(p); }
    __device__ __forceinline__ static float lds(const float *p) { return *p; }
    __device__ __forceinline__ static void st(float *p, float v) { *p = v; }
};
template <> struct Store<__half> {
    __device__ __forceinline__ static float ld(const __half *p) { return __half2float(__ldg(p)); }
    __device__ __forceinline__ static float lds(const __half *p) { return __half2float(*p); }
    __device__ __forceinline__ static void st(__half *p, float v) { *p = __float2half_rn(v); }
};
template <> struct Store<__nv_bfloat16> {
    __device__ __forceinline__ static float ld(const __nv_bfloat16 *p) {
        return __bfloat162float(__ldg(p));
    }
    __device__ __forceinline__ static float lds(const __nv_bfloat16 *p) {
        return __bfloat162float(*p);
    }
    __device__ __forceinline__ static void st(__nv_bfloat16 *p, float v) {
        *p = __float2bfloat16_rn(v);
    }
};

// Population loads and stores by pointer type: pld from global memory
// (read-only path), plds from shared memory, pst to global memory; 16-bit
// values widen to FP32 and round to nearest even on the way back.
__device__ __forceinline__ double pld(const double *p) { return __ldg(p); }
__device__ __forceinline__ float pld(const float *p) { return __ldg(p); }
__device__ __forceinline__ float pld(const __half *p) { return __half2float(__ldg(p)); }
__device__ __forceinline__ float pld(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
__device__ __forceinline__ double plds(const double *p) { return *p; }
__device__ __forceinline__ float plds(const float *p) { return *p; }
__device__ __forceinline__ float plds(const __half *p) { return __half2float(*p); }
__device__ __forceinline__ float plds(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
__device__ __forceinline__ void pst(double *p, double v) { *p = v; }
__device__ __forceinline__ void pst(float *p, float v) { *p = v; }
__device__ __forceinline__ void pst(__half *p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ void pst(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }

template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };

template <typename R>
inline KConst<R> make_kconst(const StepConst &c) {
    KConst<R> k{};
    k.nx = c.nx;
    k.ny = c.ny;
    k.nz = c.nz;
    k.nxy = (unsigned)c.nxy;
    k.dt_half = (R)(0.5 * c.dt);
    k.cflinv = (R)c.cflinv;
    k.inv_cs2 = (R)(1.0 / c.cs2);
    k.inv_cs2cfl = (R)(1.0 / (c.cs2 * c.cfl));
    for (int i = 0; i < 4; ++i) {
        k.rate_hi[i] = (R)c.rate_hi[i];
        k.rate_lo[i] = (R)c.rate_lo[i];
    }
    k.q0 = (R)c.q0;
    k.K = (R)c.K;
    k.exf = (R)c.exf;
    k.inv2dx = (R)c.inv2dx;
    k.inv2dy = (R)c.inv2dy;
    k.inv2dz = (R)c.inv2dz;
    const int rep[4] = {0, 1, 7, 19};
    for (int i = 0; i < 4; ++i) {
        const double w = w_of(rep[i]);
        k.w[i] = (R)w;
        k.c1[i] = (R)(c.dt * c.sp * w * c.cflinv2 * c.cfl);
        k.c2[i] = (R)(c.dt * c.sm * (w / c.cs2) * c.cflinv);
        k.c3[i] = (R)(c.dt * c.sp * (w / c.cs2));
    }
    for (int d = 0; d < Q; ++d) k.mw[d] = (R)c.mw[d];
    return k;
}

}  // namespace ehd
