// lbm.cu -- the fused D3Q27 TRT stream-collide for the flow populations f and
// the charge populations g, with the electrode and injection rules, in one
// pass per time step.
//
// The reference runs four kernels per step (stream_collide_save,
// LBM.cu:278-293): collide (LBM.cu:295-1091), wall bounce-back
// (LBM.cu:1093-1203), pull streaming periodic in x, y and z (LBM.cu:1205-1279)
// and injection anti-bounce-back (LBM.cu:1281-1353).  Here the populations are
// kept in the post-collision, post-wall-rule state P; one kernel pulls P from
// the neighbours (the reference's stream), applies the injection rule while
// loading (the reference's bc_charge), collides, applies the wall rules while
// storing (the reference's boundary), and writes the new P into the other
// buffer.  Each population set is read once and written once per step.
//
// Storage: SoA, pop[d][z][y][x] with d = 0..26 in one array (d = 0 is the rest
// population).  Flow populations are stored as deviations f_d - w_d rho0; the
// charge populations as they are.  Where the reference's boundary kernel
// replaces a value with another node's or another direction's, the same value
// is written here by the thread that owns it:
//   z = 0      f: P_d = f_opp(d) pulled this step, rest f unchanged
//                 (LBM.cu:1103-1131 with f0bc, LBM.cu:309)
//              g: pulled as -P_opp(d)(own node) + 2 q0 w_d (LBM.cu:1320-1348);
//                 rest g stored already as -g0' + 2 q0 w0
//   z = NZ-1   f: P_d = f_opp(d) + moving-wall term (LBM.cu:1143-1170)
//              g: P = post-collision g of z = NZ-2 (LBM.cu:1173-1200), written
//                 by the z = NZ-2 thread
//   z = 0 velocity: minus the z = 1 velocity built from z = 1 pre-collision
//                 populations, z = 1 charge and E, and the LOCAL 1/rho
//                 (LBM.cu:417-492).  The reference reads z = 1's rest
//                 populations while z = 1 threads overwrite them; here the
//                 rest populations are double-buffered, so the z = 0 node
//                 always sees the pre-collision value.
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "kernels.h"

namespace ehd {

namespace {

struct PullIdx {
    unsigned row[3][3];  // [e_y+1][e_z+1] -> NX*(ys + NY*zs) for source (y - e_y, z - e_z)
    int xs[3];           // [e_x+1] -> source x - e_x
};

__device__ __forceinline__ void make_pull(PullIdx &P, int x, int y, int z, int NX, int NY,
                                          int NZ) {
    const int xm = x == 0 ? NX - 1 : x - 1, xp = x == NX - 1 ? 0 : x + 1;
    const int ym = y == 0 ? NY - 1 : y - 1, yp = y == NY - 1 ? 0 : y + 1;
    const int zm = z == 0 ? NZ - 1 : z - 1, zp = z == NZ - 1 ? 0 : z + 1;
    P.xs[0] = xp;  // e_x = -1: source x + 1
    P.xs[1] = x;
    P.xs[2] = xm;  // e_x = +1: source x - 1
    const int ys[3] = {yp, y, ym};
    const int zs[3] = {zp, z, zm};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            P.row[a][b] = (unsigned)NX * ((unsigned)ys[a] + (unsigned)NY * (unsigned)zs[b]);
}

__device__ __forceinline__ unsigned pull_src(const PullIdx &P, int d) {
    return P.row[ey_of(d) + 1][ez_of(d) + 1] + (unsigned)P.xs[ex_of(d) + 1];
}

// e_d . (a, b, c) with the components of e_d in {-1, 0, 1}
template <typename R>
__device__ __forceinline__ R dot_e(int d, R a, R b, R c) {
    R s = 0;
    if (ex_of(d)) s = ex_of(d) > 0 ? a : -a;
    if (ey_of(d)) s = ey_of(d) > 0 ? s + b : s - b;
    if (ez_of(d)) s = ez_of(d) > 0 ? s + c : s - c;
    return s;
}

// Per-plane reference state.  Populations are stored as deviations
// f_d - w_d rho_w(z), g_d - w_d q_w(z) from the reference (rho_w, q_w) of the
// step that wrote them and of the plane z they are stored in.  A step reads
// populations written against the previous step's references (rho_r, q_r) and
// writes against its own, so a population pulled from plane z - e_z is moved
// to this step's reference of plane z by adding w_d (rho_r(z - e_z) -
// rho_w(z)).  The kernel table holds per plane, in the compute type:
// {rho_w, q_w, drho[e_z = -1, 0, +1], dq[e_z = -1, 0, +1], q_w(z) - q_w(z+1),
// unused} with drho[e] = rho_r(z - e) - rho_w(z), z - e periodic.
constexpr int kZRefStride = 10;

template <typename R>
struct ZRef {
    R rref, qref, drm, dr0, drp, dqm, dq0, dqp, up;
    // offset for a population with z-velocity e (source plane z - e)
    __device__ __forceinline__ R dr(int e) const { return e > 0 ? drm : (e < 0 ? drp : dr0); }
    __device__ __forceinline__ R dq(int e) const { return e > 0 ? dqm : (e < 0 ? dqp : dq0); }
};

// rate * x with rate = hi - lo (see StepConst::rate_hi)
template <typename R>
__device__ __forceinline__ R relax(R hi, R lo, R x) {
    return hi * x - lo * x;
}

template <typename R>
__device__ __forceinline__ ZRef<R> load_zref(const R *__restrict__ t, int z) {
    const R *p = t + kZRefStride * z;
    return ZRef<R>{__ldg(p),     __ldg(p + 1), __ldg(p + 2), __ldg(p + 3), __ldg(p + 4),
                   __ldg(p + 5), __ldg(p + 6), __ldg(p + 7), __ldg(p + 8)};
}

}  // namespace

// Kernel arguments shared by both step kernels.
template <typename T, typename R>
struct StepArgs {
    PopPtrs<T> pp;
    const R *phip;                    // phi', zero on both electrodes
    const double *ez00;               // mean-field Ez per plane
    const double *exa, *eya, *eza;    // uploaded E (first step after set_fields)
    R *qout, *rout, *uout, *vout, *wout;
    const R *zref;                    // reference table (load_zref)
    float2 *psum;                     // per-warp plane sums
    int *err;                         // set to 1 if a bounded wait gives up
};

// Pull of node (x, y, z) from global memory (the reference's stream and
// injection rule), as deviations ft_d = f_d - w_d rho_w(z), ht_d = g_d -
// w_d q_w(z).  local: the buffers hold each node's own pre-collision values.
template <typename T, typename R>
__device__ __forceinline__ void pull_global(R (&f)[Q], R (&h)[Q], const PopPtrs<T> &pp,
                                            const PullIdx &P, unsigned node, int z,
                                            const ZRef<R> &zr, const KConst<R> &c, bool local) {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        f[d] = pld(pp.fa[d] + (local ? node : pull_src(P, d))) +
               c.w[cls_of(d)] * zr.dr(local ? 0 : ez_of(d));
    }
    if (local) {
#pragma unroll
        for (int d = 0; d < Q; ++d) h[d] = pld(pp.ha[d] + node) + c.w[cls_of(d)] * zr.dq0;
    } else if (z == 0) {
        // g_d = -g_opp(d) + 2 q0 w_d (LBM.cu:1320-1348), on deviations
        h[0] = pld(pp.ha[0] + node) + c.w[0] * zr.dq0;
        const R inj = (R)2 * (c.q0 - zr.qref) - zr.dq0;
#pragma unroll
        for (int d = 1; d < Q; ++d)
            h[d] = -pld(pp.ha[opp_of(d)] + node) + inj * c.w[cls_of(d)];
    } else {
#pragma unroll
        for (int d = 0; d < Q; ++d)
            h[d] = pld(pp.ha[d] + pull_src(P, d)) + c.w[cls_of(d)] * zr.dq(ez_of(d));
    }
}

template <typename R>
struct Moments {
    R drho, dq, mx, my, mz, rho, charge;
};

template <typename R>
__device__ __forceinline__ Moments<R> moments(const R (&f)[Q], const R (&h)[Q], const ZRef<R> &zr) {
    Moments<R> m{0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        m.drho += f[d];
        m.dq += h[d];
        if (ex_of(d)) m.mx += ex_of(d) > 0 ? f[d] : -f[d];
        if (ey_of(d)) m.my += ey_of(d) > 0 ? f[d] : -f[d];
        if (ez_of(d)) m.mz += ez_of(d) > 0 ? f[d] : -f[d];
    }
    m.rho = zr.rref + m.drho;
    m.charge = zr.qref + m.dq;
    return m;
}

// Warp sum of rho and q into psum[slot] (fixed order; all 32 lanes take part).
__device__ __forceinline__ void warp_plane_sum(float rho, float charge, float2 *psum, size_t slot) {
    float2 v = make_float2(rho, charge);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if ((threadIdx.x & 31) == 0) psum[slot] = v;
}

// ---- packed FP32x2 collision (sm_100 FFMA2): two opposite pairs of one weight
// class at once, the same algebra as the scalar loops of finish_node ----
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

struct PackF {
    float2 rp_hi, nrp_lo, rm_hi, nrm_lo, half, mone;
    float2 PK[4], QK[4], nhWR[4], nWR[4], nc1[4], nc2[4];
    float tux, tuy, tuz, fx, fy, fz;
};

template <int D1, int D2, typename T>
__device__ __forceinline__ void f_pair2(const float (&f)[Q], const PackF &p,
                                        const PopPtrs<T> &pp, unsigned node) {
    constexpr int K = cls_of(D1);
    static_assert(cls_of(D2) == K, "pairs of one weight class");
    const float2 fd = f2(f[D1], f[D2]), fo = f2(f[D1 + 1], f[D2 + 1]);
    const float2 cu = f2(dot_e(D1, p.tux, p.tuy, p.tuz), dot_e(D2, p.tux, p.tuy, p.tuz));
    const float2 eF = f2(dot_e(D1, p.fx, p.fy, p.fz), dot_e(D2, p.fx, p.fy, p.fz));
    float2 X = __ffma2_rn(p.half, __fadd2_rn(fd, fo), p.PK[K]);
    X = __ffma2_rn(__fmul2_rn(p.nhWR[K], cu), cu, X);
    float2 A = __ffma2_rn(p.nrp_lo, X, p.QK[K]);
    A = __ffma2_rn(p.rp_hi, X, A);
    A = __ffma2_rn(p.nc1[K], __fmul2_rn(cu, eF), A);
    const float2 D = __ffma2_rn(p.mone, fo, fd);
    const float2 Y = __ffma2_rn(p.half, D, __fmul2_rn(p.nWR[K], cu));
    float2 B = __ffma2_rn(p.nrm_lo, Y, __fmul2_rn(p.nc2[K], eF));
    B = __ffma2_rn(p.rm_hi, Y, B);
    const float2 od = __ffma2_rn(p.mone, __fadd2_rn(A, B), fd);
    const float2 oo = __ffma2_rn(p.mone, A, __fadd2_rn(fo, B));
    pst(pp.fb[D1] + node, od.x);
    pst(pp.fb[D2] + node, od.y);
    pst(pp.fb[D1 + 1] + node, oo.x);
    pst(pp.fb[D2 + 1] + node, oo.y);
}

struct PackG {
    float2 cp_hi, ncp_lo, cm_hi, ncm_lo, cm_lo, half, mone;
    float2 PQ[4], nhWQ[4], nWQ[4], twoWQ[4], wup[4];
    float tux, tuy, tuz;
    bool over;  // antisymmetric rate over-relaxed: hi = 2 exactly
};

template <int D1, int D2, typename T>
__device__ __forceinline__ void g_pair2(const float (&h)[Q], const PackG &p,
                                        const PopPtrs<T> &pp, unsigned node, unsigned nodeup,
                                        bool dup) {
    constexpr int K = cls_of(D1);
    static_assert(cls_of(D2) == K, "pairs of one weight class");
    const float2 hd = f2(h[D1], h[D2]), ho = f2(h[D1 + 1], h[D2 + 1]);
    const float2 cu = f2(dot_e(D1, p.tux, p.tuy, p.tuz), dot_e(D2, p.tux, p.tuy, p.tuz));
    float2 X = __ffma2_rn(p.half, __fadd2_rn(hd, ho), p.PQ[K]);
    X = __ffma2_rn(__fmul2_rn(p.nhWQ[K], cu), cu, X);
    const float2 Dd = __ffma2_rn(p.mone, ho, hd);
    const float2 Y = __ffma2_rn(p.half, Dd, __fmul2_rn(p.nWQ[K], cu));
    const float2 A = __ffma2_rn(p.cp_hi, X, __fmul2_rn(p.ncp_lo, X));
    float2 od, oo;
    if (p.over) {
        // with B = 2 Y - lo Y: hd - 2 Y = ho + 2 WQ cu and ho + 2 Y = hd - 2 WQ cu
        // exactly, so the outputs never form hd - B, which cancels when the
        // rate is close to 2
        const float2 t = __fmul2_rn(p.twoWQ[K], cu);
        od = __ffma2_rn(p.cm_lo, Y, __ffma2_rn(p.mone, A, __fadd2_rn(ho, t)));
        oo = __ffma2_rn(p.ncm_lo, Y, __ffma2_rn(p.mone, A, __ffma2_rn(p.mone, t, hd)));
    } else {
        const float2 B = __ffma2_rn(p.cm_hi, Y, __fmul2_rn(p.ncm_lo, Y));
        od = __ffma2_rn(p.mone, __fadd2_rn(A, B), hd);
        oo = __ffma2_rn(p.mone, A, __fadd2_rn(ho, B));
    }
    pst(pp.hb[D1] + node, od.x);
    pst(pp.hb[D2] + node, od.y);
    pst(pp.hb[D1 + 1] + node, oo.x);
    pst(pp.hb[D2 + 1] + node, oo.y);
    if (dup) {
        const float2 ud = __fadd2_rn(od, p.wup[K]), uo = __fadd2_rn(oo, p.wup[K]);
        pst(pp.hb[D1] + nodeup, ud.x);
        pst(pp.hb[D2] + nodeup, ud.y);
        pst(pp.hb[D1 + 1] + nodeup, uo.x);
        pst(pp.hb[D2 + 1] + nodeup, uo.y);
    }
}

// Everything after the moments: E, the injector override, the macroscopic
// outputs, the TRT collisions of f and g and the wall rules on store.
//
// Collision algebra (LBM.cu:519-1089 rewritten on deviations, per opposite
// pair d, o = d+1 of weight class k, s = f_d + f_o):
//   fp - feq+  = s/2 + P_k - (w_k rho / 2) cu^2,  P_k = w_k rho usq - w_k drho
//   fm - feq-  = (f_d - f_o)/2 - w_k rho cu
//   A = rate+ (fp - feq+) + dt sp (w_k/cs2) uF - dt sp w_k cflinv2 CFL cu eF
//   B = rate- (fm - feq-) - dt sm (w_k/cs2) cflinv eF
//   f_d' = f_d - A - B,  f_o' = f_o - A + B
// (e.u = cu cs2 CFL); the same with q, u + K E and no source for g.
template <typename T, typename R, bool MACROS>
__device__ __forceinline__ void finish_node(R (&f)[Q], R (&h)[Q], const Moments<R> &mo, int x,
                                            int y, int z, unsigned node, const ZRef<R> &zr,
                                            const StepArgs<T, R> &a, const KConst<R> &c,
                                            bool local, bool earr) {
    const int NX = c.nx, NY = c.ny, NZ = c.nz;
    const R drho = mo.drho, dq = mo.dq, mx = mo.mx, my = mo.my, mz = mo.mz;
    const R rho = mo.rho, charge = mo.charge;
    // ---- E at this node (and at z = 1 for the injector override) ----
    R Ex, Ey, Ez;
    const unsigned row = (unsigned)NX * ((unsigned)y + (unsigned)NY * z);
    const int xm = x == 0 ? NX - 1 : x - 1, xp = x == NX - 1 ? 0 : x + 1;
    const int ym = y == 0 ? NY - 1 : y - 1, yp = y == NY - 1 ? 0 : y + 1;
    const unsigned rym = (unsigned)NX * ((unsigned)ym + (unsigned)NY * z);
    const unsigned ryp = (unsigned)NX * ((unsigned)yp + (unsigned)NY * z);
    if (!earr) {
        // E = -grad(phi), central differences (gpu_efield, poisson.cu:44-60);
        // phi = phi00(z) + phi'(x,y,z) with phi' = 0 on both electrodes, and
        // Ez on the electrodes copied from the planes inside (gpu_bc,
        // poisson.cu:61-73).
        Ex = (__ldg(a.phip + row + xm) - __ldg(a.phip + row + xp)) * c.inv2dx;
        Ey = (__ldg(a.phip + rym + x) - __ldg(a.phip + ryp + x)) * c.inv2dy;
        const int zc = z < 1 ? 1 : (z > NZ - 2 ? NZ - 2 : z);
        const unsigned rzc = (unsigned)NX * ((unsigned)y + (unsigned)NY * zc);
        Ez = (R)__ldg(a.ez00 + zc) +
             (__ldg(a.phip + rzc - c.nxy + x) - __ldg(a.phip + rzc + c.nxy + x)) * c.inv2dz;
    } else {
        Ex = (R)__ldg(a.exa + node);
        Ey = (R)__ldg(a.eya + node);
        Ez = (R)__ldg(a.eza + node);
    }

    const R fx = charge * Ex + c.exf, fy = charge * Ey, fz = charge * Ez;
    const R rhoinv = (R)1 / rho;
    R ux = rhoinv * (mx * c.cflinv + fx * c.dt_half);
    R uy = rhoinv * (my * c.cflinv + fy * c.dt_half);
    R uz = rhoinv * (mz * c.cflinv + fz * c.dt_half);

    if (z == 0) {
        // LBM.cu:417-492
        const ZRef<R> z1 = load_zref(a.zref, 1);
        PullIdx P1;
        make_pull(P1, x, y, 1, NX, NY, NZ);
        const unsigned node1 = node + c.nxy;
        R dqm = pld(a.pp.ha[0] + node1) + c.w[0] * z1.dq0;
        R mxm = 0, mym = 0, mzm = 0;
#pragma unroll
        for (int d = 1; d < Q; ++d) {
            const unsigned s1 = local ? node1 : pull_src(P1, d);
            const int e = local ? 0 : ez_of(d);
            const R fm = pld(a.pp.fa[d] + s1) + c.w[cls_of(d)] * z1.dr(e);
            const R hm = pld(a.pp.ha[d] + s1) + c.w[cls_of(d)] * z1.dq(e);
            dqm += hm;
            if (ex_of(d)) mxm += ex_of(d) > 0 ? fm : -fm;
            if (ey_of(d)) mym += ey_of(d) > 0 ? fm : -fm;
            if (ez_of(d)) mzm += ez_of(d) > 0 ? fm : -fm;
        }
        const R chargem = z1.qref + dqm;
        R Exm, Eym, Ezm;
        if (!earr) {
            const unsigned row1 = row + c.nxy;
            Exm = (__ldg(a.phip + row1 + xm) - __ldg(a.phip + row1 + xp)) * c.inv2dx;
            Eym = (__ldg(a.phip + rym + c.nxy + x) - __ldg(a.phip + ryp + c.nxy + x)) * c.inv2dy;
            Ezm = (R)__ldg(a.ez00 + 1) +
                  (__ldg(a.phip + row + x) - __ldg(a.phip + row + 2 * c.nxy + x)) * c.inv2dz;
        } else {
            Exm = (R)__ldg(a.exa + node1);
            Eym = (R)__ldg(a.eya + node1);
            Ezm = (R)__ldg(a.eza + node1);
        }
        const R fxm = chargem * Exm + c.exf, fym = chargem * Eym, fzm = chargem * Ezm;
        ux = -rhoinv * (mxm * c.cflinv + fxm * c.dt_half);
        uy = -rhoinv * (mym * c.cflinv + fym * c.dt_half);
        uz = -rhoinv * (mzm * c.cflinv + fzm * c.dt_half);
    }

    a.qout[node] = charge;
    if (MACROS) {
        a.rout[node] = rho;
        a.uout[node] = ux;
        a.vout[node] = uy;
        a.wout[node] = uz;
    }

    // ---- f: collide (interior) or wall rule ----
    if (z == 0 || z == NZ - 1) {
        pst(a.pp.fb[0] + node, f[0]);
#pragma unroll
        for (int d = 1; d < Q; ++d) {
            R v = f[opp_of(d)];
            if (z == NZ - 1 && mw_sign_of(d) != 0) v += c.mw[d];
            pst(a.pp.fb[d] + node, v);
        }
    } else {
        const R rp_hi = c.rate_hi[0], rp_lo = c.rate_lo[0];
        const R rm_hi = c.rate_hi[1], rm_lo = c.rate_lo[1];
        const R usq = (R)0.5 * (ux * ux + uy * uy + uz * uz) * c.inv_cs2;
        const R tux = ux * c.inv_cs2cfl, tuy = uy * c.inv_cs2cfl, tuz = uz * c.inv_cs2cfl;
        const R uF = ux * fx + uy * fy + uz * fz;
        R WR[4], PK[4], QK[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            WR[k] = c.w[k] * rho;
            PK[k] = WR[k] * usq - c.w[k] * drho;
            QK[k] = c.c3[k] * uF;
        }
        pst(a.pp.fb[0] + node, f[0] - relax(rp_hi, rp_lo, f[0] + PK[0]) - QK[0]);
        if constexpr (sizeof(R) == 4) {
            PackF pk;
            pk.rp_hi = f2(rp_hi);
            pk.nrp_lo = f2(-rp_lo);
            pk.rm_hi = f2(rm_hi);
            pk.nrm_lo = f2(-rm_lo);
            pk.half = f2(0.5f);
            pk.mone = f2(-1.f);
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                pk.PK[k] = f2(PK[k]);
                pk.QK[k] = f2(QK[k]);
                pk.nhWR[k] = f2(-0.5f * WR[k]);
                pk.nWR[k] = f2(-WR[k]);
                pk.nc1[k] = f2(-c.c1[k]);
                pk.nc2[k] = f2(-c.c2[k]);
            }
            pk.tux = tux;
            pk.tuy = tuy;
            pk.tuz = tuz;
            pk.fx = fx;
            pk.fy = fy;
            pk.fz = fz;
            f_pair2<1, 3>(f, pk, a.pp, node);
            f_pair2<7, 9>(f, pk, a.pp, node);
            f_pair2<11, 13>(f, pk, a.pp, node);
            f_pair2<15, 17>(f, pk, a.pp, node);
            f_pair2<19, 21>(f, pk, a.pp, node);
            f_pair2<23, 25>(f, pk, a.pp, node);
            {  // the fifth pair of class 1 alone
                constexpr int d = 5, o = 6, k = 1;
                const R cu = dot_e(d, tux, tuy, tuz);
                const R eF = dot_e(d, fx, fy, fz);
                const R X = (R)0.5 * (f[d] + f[o]) + PK[k] - (R)0.5 * WR[k] * cu * cu;
                const R A = relax(rp_hi, rp_lo, X) + QK[k] - c.c1[k] * cu * eF;
                const R Y = (R)0.5 * (f[d] - f[o]) - WR[k] * cu;
                const R B = relax(rm_hi, rm_lo, Y) - c.c2[k] * eF;
                pst(a.pp.fb[d] + node, f[d] - A - B);
                pst(a.pp.fb[o] + node, f[o] - A + B);
            }
        } else {
#pragma unroll
        for (int d = 1; d < Q; d += 2) {
            const int o = d + 1, k = cls_of(d);
            const R cu = dot_e(d, tux, tuy, tuz);
            const R eF = dot_e(d, fx, fy, fz);
            const R X = (R)0.5 * (f[d] + f[o]) + PK[k] - (R)0.5 * WR[k] * cu * cu;
            const R A = relax(rp_hi, rp_lo, X) + QK[k] - c.c1[k] * cu * eF;
            const R Y = (R)0.5 * (f[d] - f[o]) - WR[k] * cu;
            const R B = relax(rm_hi, rm_lo, Y) - c.c2[k] * eF;
            pst(a.pp.fb[d] + node, f[d] - A - B);
            pst(a.pp.fb[o] + node, f[o] - A + B);
        }
        }
    }

    // ---- g: collide (z <= NZ-2); the NZ-1 plane is written by z = NZ-2,
    // relative to q_ref(NZ-1) ----
    if (z != NZ - 1) {
        const R cp_hi = c.rate_hi[2], cp_lo = c.rate_lo[2];
        const R cm_hi = c.rate_hi[3], cm_lo = c.rate_lo[3];
        const R ucx = ux + c.K * Ex, ucy = uy + c.K * Ey, ucz = uz + c.K * Ez;
        const R usq = (R)0.5 * (ucx * ucx + ucy * ucy + ucz * ucz) * c.inv_cs2;
        const R tux = ucx * c.inv_cs2cfl, tuy = ucy * c.inv_cs2cfl, tuz = ucz * c.inv_cs2cfl;
        const bool dup = (z == NZ - 2);
        const unsigned nodeup = node + c.nxy;
        const R up = zr.up;  // q_w(z) - q_w(z+1)
        R WQ[4], PQ[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            WQ[k] = c.w[k] * charge;
            PQ[k] = WQ[k] * usq - c.w[k] * dq;
        }
        {
            const R out = h[0] - relax(cp_hi, cp_lo, h[0] + PQ[0]);
            pst(a.pp.hb[0] + node, z == 0 ? -out + (R)2 * (c.q0 - zr.qref) * c.w[0] : out);
            if (dup) pst(a.pp.hb[0] + nodeup, out + c.w[0] * up);
        }
        auto g_one = [&](auto dc) {
            constexpr int d = decltype(dc)::value, o = d + 1, k = cls_of(d);
            const R cu = dot_e(d, tux, tuy, tuz);
            const R X = (R)0.5 * (h[d] + h[o]) + PQ[k] - (R)0.5 * WQ[k] * cu * cu;
            const R Y = (R)0.5 * (h[d] - h[o]) - WQ[k] * cu;
            const R A = relax(cp_hi, cp_lo, X);
            R outd, outo;
            if (sizeof(R) == 4 && cm_hi == (R)2) {  // cancellation-free form, see g_pair2
                const R t = (R)2 * WQ[k] * cu;
                outd = (h[o] + t) - A + cm_lo * Y;
                outo = (h[d] - t) - A - cm_lo * Y;
            } else {
                const R B = relax(cm_hi, cm_lo, Y);
                outd = h[d] - A - B;
                outo = h[o] - A + B;
            }
            pst(a.pp.hb[d] + node, outd);
            pst(a.pp.hb[o] + node, outo);
            if (dup) {
                pst(a.pp.hb[d] + nodeup, outd + c.w[k] * up);
                pst(a.pp.hb[o] + nodeup, outo + c.w[k] * up);
            }
        };
        if constexpr (sizeof(R) == 4) {
            PackG pg;
            pg.cp_hi = f2(cp_hi);
            pg.ncp_lo = f2(-cp_lo);
            pg.cm_hi = f2(cm_hi);
            pg.ncm_lo = f2(-cm_lo);
            pg.cm_lo = f2(cm_lo);
            pg.over = cm_hi == 2.f;
            pg.half = f2(0.5f);
            pg.mone = f2(-1.f);
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                pg.PQ[k] = f2(PQ[k]);
                pg.nhWQ[k] = f2(-0.5f * WQ[k]);
                pg.nWQ[k] = f2(-WQ[k]);
                pg.twoWQ[k] = f2(2.f * WQ[k]);
                pg.wup[k] = f2(c.w[k] * up);
            }
            pg.tux = tux;
            pg.tuy = tuy;
            pg.tuz = tuz;
            g_pair2<1, 3>(h, pg, a.pp, node, nodeup, dup);
            g_pair2<7, 9>(h, pg, a.pp, node, nodeup, dup);
            g_pair2<11, 13>(h, pg, a.pp, node, nodeup, dup);
            g_pair2<15, 17>(h, pg, a.pp, node, nodeup, dup);
            g_pair2<19, 21>(h, pg, a.pp, node, nodeup, dup);
            g_pair2<23, 25>(h, pg, a.pp, node, nodeup, dup);
            g_one(std::integral_constant<int, 5>{});
        } else {
#pragma unroll
            for (int d = 1; d < Q; d += 2) {
                const int o = d + 1, k = cls_of(d);
                const R cu = dot_e(d, tux, tuy, tuz);
                const R X = (R)0.5 * (h[d] + h[o]) + PQ[k] - (R)0.5 * WQ[k] * cu * cu;
                const R Y = (R)0.5 * (h[d] - h[o]) - WQ[k] * cu;
                const R A = relax(cp_hi, cp_lo, X);
                R outd, outo;
                if (sizeof(R) == 4 && cm_hi == (R)2) {  // cancellation-free form, see g_pair2
                    const R t = (R)2 * WQ[k] * cu;
                    outd = (h[o] + t) - A + cm_lo * Y;
                    outo = (h[d] - t) - A - cm_lo * Y;
                } else {
                    const R B = relax(cm_hi, cm_lo, Y);
                    outd = h[d] - A - B;
                    outo = h[o] - A + B;
                }
                pst(a.pp.hb[d] + node, outd);
                pst(a.pp.hb[o] + node, outo);
                if (dup) {
                    pst(a.pp.hb[d] + nodeup, outd + c.w[k] * up);
                    pst(a.pp.hb[o] + nodeup, outo + c.w[k] * up);
                }
            }
        }
    }
}

// GENERAL = false: the steady-state step (pull, E from phi).  GENERAL = true
// adds two run-time switches used right after ehd_set_fields:
//   local_pops: the buffers hold the pre-collision populations of each node
//               (the reference's f1/h1 after init_equilibrium), so they are
//               read in place, without pull or injection rule;
//   e_arrays:   E comes from the uploaded FP64 arrays instead of phi.
// One thread per node, 128-thread blocks.
// One block of the per-node step: block (bxi, byi) of a gx x gy tiling of
// plane z (the grid indices are arguments so that a launch over several
// instances can map its blocks).
template <typename T, typename R, bool GENERAL, bool MACROS>
__device__ __forceinline__ void node_block(const StepArgs<T, R> &a, const KConst<R> &c, int bxi,
                                           int byi, int z, int gx, int gy, int local_pops,
                                           int e_arrays) {
    const bool local = GENERAL && local_pops;
    const bool earr = GENERAL && e_arrays;
    int x = bxi * blockDim.x + threadIdx.x;
    int y = byi * blockDim.y + threadIdx.y;
    const bool inside = x < c.nx && y < c.ny;
    // lanes outside the grid work on a valid node so that the whole warp can
    // take part in the plane sums; they store nothing
    if (!inside) {
        x = x < c.nx ? x : c.nx - 1;
        y = y < c.ny ? y : c.ny - 1;
    }
    const unsigned node = (unsigned)x + (unsigned)c.nx * ((unsigned)y + (unsigned)c.ny * z);
    const ZRef<R> zr = load_zref(a.zref, z);
    PullIdx P;
    make_pull(P, x, y, z, c.nx, c.ny, c.nz);
    R f[Q], h[Q];
    pull_global<T, R>(f, h, a.pp, P, node, z, zr, c, local);
    const Moments<R> mo = moments(f, h, zr);
    {
        const int tid = threadIdx.x + blockDim.x * threadIdx.y;
        const int wpb = (blockDim.x * blockDim.y) >> 5;
        warp_plane_sum(inside ? (float)mo.rho : 0.f, inside ? (float)mo.charge : 0.f, a.psum,
                       (((size_t)z * gy + byi) * gx + bxi) * wpb + (tid >> 5));
    }
    if (!inside) return;
    finish_node<T, R, MACROS>(f, h, mo, x, y, z, node, zr, a, c, local, earr);
}

template <typename T, typename R, bool GENERAL, bool MACROS>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 2 : 4)
lbm_step_kernel(const StepArgs<T, R> a, const KConst<R> c, int local_pops, int e_arrays) {
    node_block<T, R, GENERAL, MACROS>(a, c, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x,
                                      gridDim.y, local_pops, e_arrays);
}

// ---- bulk-copy row kernel ------------------------------------------------------

namespace {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// one contiguous global -> shared copy completing on the barrier; both
// addresses 16-byte aligned and the size a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

constexpr unsigned kWaitLimit = 1u << 24;  // try_wait polls before giving up

// e_y + 1 and e_z + 1 of all directions, 2 bits per direction, for lookups
// with a run-time d (a constexpr table indexed at run time lands in local
// memory)
constexpr unsigned long long pack_e(int comp) {
    unsigned long long v = 0;
    for (int d = 0; d < Q; ++d)
        v |= (unsigned long long)((comp == 1 ? ey_of(d) : ez_of(d)) + 1) << (2 * d);
    return v;
}
constexpr unsigned long long kEyPack = pack_e(1), kEzPack = pack_e(2);
__device__ __forceinline__ int ey_rt(int d) { return (int)((kEyPack >> (2 * d)) & 3u) - 1; }
__device__ __forceinline__ int ez_rt(int d) { return (int)((kEzPack >> (2 * d)) & 3u) - 1; }

}  // namespace

// Persistent variant of the steady-state step for rows of NX nodes: one CTA
// of NX threads walks the x-rows (y, z) of the planes z >= 1, and the source
// rows (y - e_y, z - e_z) of f_d and g_d of each row arrive in shared memory
// by bulk copies, two rows ahead (two stages).  The x shift -e_x and its
// periodic wrap are applied when reading shared memory.
//
// No block-wide barrier in the loop: each warp waits for its stage on the
// stage's mbarrier, reads its 54 values into registers and counts itself out
// of the stage (shared counter); the warp that counts last refills the stage
// with the row two iterations ahead while the others compute.  The injector
// plane z = 0 (own-node g and z = 1 populations) is left to the per-node
// kernel, launched for that plane alone.  A wait that does not complete within
// kWaitLimit polls sets *err, waits (bounded) for the copies that may still
// be landing, and ends the warp.
//
// rows_run is the loop of CTA blk of nblk; lbm_rows_kernel runs one instance,
// lbm_rows_group_kernel several instances of the same NX (blockIdx.y) with
// their arguments from a device table.
template <typename T, typename R, bool MACROS, bool PART>
__device__ __forceinline__ void rows_run(const StepArgs<T, R> &a, const KConst<R> &c, int blk,
                                         int nblk) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ unsigned long long bar[2];
    __shared__ unsigned cnt[2];
    const int NX = c.nx, NY = c.ny, NZ = c.nz;
    using F = typename PopT<T>::F;
    using G = typename PopT<T>::G;
    // stage s: the 27 f rows, then the 27 g rows
    const size_t stage_bytes = (size_t)Q * NX * (sizeof(F) + sizeof(G));
    auto stage_f = [&](int st) { return reinterpret_cast<F *>(smem_raw + (size_t)st * stage_bytes); };
    auto stage_g = [&](int st) {
        return reinterpret_cast<G *>(smem_raw + (size_t)st * stage_bytes + (size_t)Q * NX * sizeof(F));
    };
    const unsigned row_bytes_f = (unsigned)(NX * sizeof(F)), row_bytes_g = (unsigned)(NX * sizeof(G));
    // blockDim.x = NX rounded up to whole warps: with PART (NX not a multiple
    // of 32), lanes past the row work on its last node (so that the whole warp
    // takes part in the plane sums) and store nothing
    const bool inside = !PART || (int)threadIdx.x < NX;
    const int x = inside ? (int)threadIdx.x : NX - 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned nw = blockDim.x / 32u;

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        cnt[0] = 0u;
        cnt[1] = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // the calling warp issues the 54 row copies of row (yy, zz) into stage s;
    // lane d < 27 copies direction d
    auto issue = [&](int yy, int zz, int s) {
        if (lane == 0) mbar_expect_tx(&bar[s], (unsigned)Q * (row_bytes_f + row_bytes_g));
        __syncwarp();
        if (lane < Q) {
            int ys = yy - ey_rt(lane), zs = zz - ez_rt(lane);
            ys += ys < 0 ? NY : (ys >= NY ? -NY : 0);
            zs += zs < 0 ? NZ : (zs >= NZ ? -NZ : 0);
            // direction d's array starts d * NX * NY * NZ after direction 0's
            const size_t off = (size_t)lane * NX * NY * NZ + (size_t)NX * ((size_t)ys + (size_t)NY * zs);
            bulk_g2s(stage_f(s) + (size_t)lane * NX, a.pp.fa[0] + off, row_bytes_f, &bar[s]);
            bulk_g2s(stage_g(s) + (size_t)lane * NX, a.pp.ha[0] + off, row_bytes_g, &bar[s]);
        }
    };
    // bounded wait of the calling thread for the phase `parity` of bar[s]
    auto wait_stage = [&](int s, unsigned parity) {
        unsigned n = 0;
        while (!mbar_try_wait(&bar[s], parity) && ++n < kWaitLimit) {
        }
        return n < kWaitLimit;
    };
    // rows r = NY + blk + k nblk, r < NY NZ, as (y, z); a step of nblk rows
    // advances y by gy and z by gz (plus the carry)
    const int g = nblk, gy = g % NY, gz = g / NY;
    auto advance = [&](int &yy, int &zz) {
        yy += gy;
        zz += gz;
        if (yy >= NY) {
            yy -= NY;
            ++zz;
        }
    };

    unsigned phases = 0u;  // bit s: parity of the next phase of bar[s]
    int y = blk % NY, z = 1 + blk / NY;
    if (warp == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        int y1 = y, z1 = z;
        advance(y1, z1);
        if (z < NZ) issue(y, z, 0);
        if (z1 < NZ) issue(y1, z1, 1);
    }
    for (int it = 0; z < NZ; ++it) {
        const int s = it & 1;
        const unsigned node = (unsigned)x + (unsigned)NX * ((unsigned)y + (unsigned)NY * z);
        const ZRef<R> zr = load_zref(a.zref, z);
        PullIdx P;
        make_pull(P, x, y, z, NX, NY, NZ);
        R f[Q], h[Q];
        const unsigned par = (phases >> s) & 1u;
        if (!__all_sync(0xffffffffu, wait_stage(s, par))) {
            if (lane == 0) {
                atomicExch(a.err, 1);
                // this stage's copies and the other stage's (the next row)
                // may still be landing: bounded waits for both
                (void)wait_stage(s, par);
                int y1 = y, z1 = z;
                advance(y1, z1);
                if (z1 < NZ) (void)wait_stage(s ^ 1, (phases >> (s ^ 1)) & 1u);
            }
            __syncwarp();
            return;
        }
        phases ^= 1u << s;
        {
            const F *sf = stage_f(s);
            const G *sh = stage_g(s);
#pragma unroll
            for (int d = 0; d < Q; ++d) {
                const int xs = P.xs[ex_of(d) + 1];
                f[d] = plds(sf + (size_t)d * NX + xs) + c.w[cls_of(d)] * zr.dr(ez_of(d));
                h[d] = plds(sh + (size_t)d * NX + xs) + c.w[cls_of(d)] * zr.dq(ez_of(d));
            }
        }
        const Moments<R> mo = moments(f, h, zr);
        warp_plane_sum(inside ? (float)mo.rho : 0.f, inside ? (float)mo.charge : 0.f, a.psum,
                       ((size_t)z * NY + y) * nw + warp);
        if (inside) finish_node<T, R, MACROS>(f, h, mo, x, y, z, node, zr, a, c, false, false);
        // this warp is done with the stage; the last of the nw warps refills it
        __syncwarp();
        unsigned last = 0u;
        if (lane == 0) {
            __threadfence_block();
            last = atomicAdd(&cnt[s], 1u) == nw - 1u;
            if (last) atomicExch(&cnt[s], 0u);
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        advance(y, z);  // the next row of this block
        if (last) {
            int y2 = y, z2 = z;
            advance(y2, z2);
            if (z2 < NZ) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(y2, z2, s);
            }
        }
    }
}

template <typename T, typename R, bool MACROS, bool PART>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 1 : 2)
lbm_rows_kernel(const StepArgs<T, R> a, const KConst<R> c) {
    rows_run<T, R, MACROS, PART>(a, c, (int)blockIdx.x, (int)gridDim.x);
}

template <typename T, typename R>
struct LbmGroupDesc {
    StepArgs<T, R> a;
    KConst<R> k;
};

// A copy of the instance's descriptor in shared memory, as 8-byte words.
template <typename T, typename R>
__device__ __forceinline__ void load_group_desc(LbmGroupDesc<T, R> &sd,
                                                const LbmGroupDesc<T, R> *__restrict__ desc,
                                                int inst) {
    static_assert(sizeof(LbmGroupDesc<T, R>) % 8 == 0, "copied as 8-byte words");
    constexpr int W = sizeof(LbmGroupDesc<T, R>) / 8;
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(desc + inst);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sd);
    const int nt = blockDim.x * blockDim.y;
    for (int i = threadIdx.x + blockDim.x * threadIdx.y; i < W; i += nt) dst[i] = src[i];
}

template <typename T, typename R, bool MACROS, bool PART>
__global__ void __launch_bounds__(256, sizeof(R) == 8 ? 1 : 2)
lbm_rows_group_kernel(const LbmGroupDesc<T, R> *__restrict__ desc) {
    __shared__ LbmGroupDesc<T, R> sd;
    load_group_desc(sd, desc, (int)blockIdx.y);
    __syncthreads();
    rows_run<T, R, MACROS, PART>(sd.a, sd.k, (int)blockIdx.x, (int)gridDim.x);
}

// the row kernels for (macro output, row ending inside a warp)
template <typename T, typename R>
using RowsKern = void (*)(const StepArgs<T, R>, const KConst<R>);
template <typename T, typename R>
RowsKern<T, R> rows_kernel(bool macros, bool part) {
    return macros ? (part ? lbm_rows_kernel<T, R, true, true> : lbm_rows_kernel<T, R, true, false>)
                  : (part ? lbm_rows_kernel<T, R, false, true> : lbm_rows_kernel<T, R, false, false>);
}
template <typename T, typename R>
using RowsGroupKern = void (*)(const LbmGroupDesc<T, R> *);
template <typename T, typename R>
RowsGroupKern<T, R> rows_group_kernel(bool macros, bool part) {
    return macros ? (part ? lbm_rows_group_kernel<T, R, true, true>
                          : lbm_rows_group_kernel<T, R, true, false>)
                  : (part ? lbm_rows_group_kernel<T, R, false, true>
                          : lbm_rows_group_kernel<T, R, false, false>);
}

// Equilibrium populations from the FP64 fields (gpu_init_equilibrium,
// LBM.cu:110-276), computed in FP64 and stored as deviations from the plane's
// reference state.
template <typename T>
__global__ void init_equilibrium_kernel(typename PopT<T>::F *__restrict__ f,
                                        typename PopT<T>::G *__restrict__ h,
                                        const double *__restrict__ r,
                                        const double *__restrict__ u,
                                        const double *__restrict__ v,
                                        const double *__restrict__ w,
                                        const double *__restrict__ q,
                                        const double *__restrict__ ex,
                                        const double *__restrict__ ey,
                                        const double *__restrict__ ez,
                                        const double *__restrict__ ref, StepConst c) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int z = (int)(i / c.nxy);
    const double rref = ref[2 * z], qref = ref[2 * z + 1];
    const double cs2 = c.cs2;
    const double rho = r[i], ux = u[i], uy = v[i], uz = w[i], ch = q[i];
    const double ucx = ux + c.K * ex[i], ucy = uy + c.K * ey[i], ucz = uz + c.K * ez[i];
    const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy + uz * uz) / cs2;
    const double omusq_c = 1.0 - 0.5 * (ucx * ucx + ucy * ucy + ucz * ucz) / cs2;
    const double tux = ux / cs2 / c.cfl, tuy = uy / cs2 / c.cfl, tuz = uz / cs2 / c.cfl;
    const double tcx = ucx / cs2 / c.cfl, tcy = ucy / cs2 / c.cfl, tcz = ucz / cs2 / c.cfl;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const double cu = ex_of(d) * tux + ey_of(d) * tuy + ez_of(d) * tuz;
        const double cc = ex_of(d) * tcx + ey_of(d) * tcy + ez_of(d) * tcz;
        const double fe = w_of(d) * rho * (omusq + cu * (1.0 + 0.5 * cu));
        const double he = w_of(d) * ch * (omusq_c + cc * (1.0 + 0.5 * cc));
        pst(f + d * c.n + i, (decltype(pld(f)))(fe - w_of(d) * rref));
        pst(h + d * c.n + i, (decltype(pld(h)))(he - w_of(d) * qref));
    }
}

// Driver-visible FP64 fields from the step's working buffers.  mask bit 1:
// rho, u, v, w, q widened; bit 2: phi = phi00(z) + phi' and E = -grad(phi)
// with the electrode copy of Ez (poisson.cu:44-73, 154-167).
template <typename R>
__global__ void materialize_kernel(const R *__restrict__ rho, const R *__restrict__ u,
                                   const R *__restrict__ v, const R *__restrict__ w,
                                   const R *__restrict__ q, const R *__restrict__ phip,
                                   const double *__restrict__ phi00, double *__restrict__ o_rho,
                                   double *__restrict__ o_u, double *__restrict__ o_v,
                                   double *__restrict__ o_w, double *__restrict__ o_q,
                                   double *__restrict__ o_phi, double *__restrict__ o_ex,
                                   double *__restrict__ o_ey, double *__restrict__ o_ez,
                                   int mask, StepConst c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= c.nx) return;
    const int NX = c.nx, NY = c.ny, NZ = c.nz;
    auto idx = [&](int xx, int yy, int zz) {
        return (long long)xx + (long long)NX * ((long long)yy + (long long)NY * zz);
    };
    auto phi = [&](int xx, int yy, int zz) { return phi00[zz] + (double)phip[idx(xx, yy, zz)]; };
    const long long i = idx(x, y, z);
    if (mask & 1) {
        o_rho[i] = rho[i];
        o_u[i] = u[i];
        o_v[i] = v[i];
        o_w[i] = w[i];
        o_q[i] = q[i];
    }
    if (!(mask & 2)) return;
    o_phi[i] = phi(x, y, z);
    const int xm = (NX + x - 1) % NX, xp = (x + 1) % NX;
    const int ym = (NY + y - 1) % NY, yp = (y + 1) % NY;
    o_ex[i] = 0.5 * (phi(xm, y, z) - phi(xp, y, z)) * (2.0 * c.inv2dx);
    o_ey[i] = 0.5 * (phi(x, ym, z) - phi(x, yp, z)) * (2.0 * c.inv2dy);
    const int zc = z < 1 ? 1 : (z > NZ - 2 ? NZ - 2 : z);
    o_ez[i] = 0.5 * (phi(x, y, zc - 1) - phi(x, y, zc + 1)) * (2.0 * c.inv2dz);
}

// The reference's start, gpu_initialization (LBM.cu:81-96): rho = rho0, q = 0,
// phi = V (Lz - dz z)/Lz, u = E = 0, into the FP64 field arrays.
__global__ void reference_init_kernel(double *const *out, StepConst c, double voltage,
                                      double lz, double dz) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int z = (int)(i / c.nxy);
    out[0][i] = c.rho0;
    out[1][i] = 0.0;
    out[2][i] = 0.0;
    out[3][i] = 0.0;
    out[4][i] = 0.0;
    out[5][i] = voltage * (lz - dz * z) / lz;
    out[6][i] = 0.0;
    out[7][i] = 0.0;
    out[8][i] = 0.0;
}

// FP64 fields -> the step's compute-type macroscopic buffers.
template <typename R>
__global__ void fields_to_compute_kernel(const double *const *out, R *rho, R *u, R *v, R *w,
                                         R *q, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rho[i] = (R)out[0][i];
    u[i] = (R)out[1][i];
    v[i] = (R)out[2][i];
    w[i] = (R)out[3][i];
    q[i] = (R)out[4][i];
}

// ---- launchers ---------------------------------------------------------------

// Block width of the per-node launch of the injector plane beside the row
// kernel: whole warps along x, so that its plane sums land in the row
// kernel's slots [y][x / 32] (the widest of 128, 96, 64 that divides NX, else
// 32 with a partial last block).
static int z0_block_x(int nx) {
    for (int bx = 128; bx > 32; bx -= 32)
        if (nx % bx == 0) return bx;
    return 32;
}
// CTA width of the row kernel: NX rounded up to whole warps
static int rows_block_x(int nx) { return (nx + 31) / 32 * 32; }

size_t lbm_rows_smem(int nx, size_t fsize, size_t gsize) {
    return (size_t)2 * Q * nx * (fsize + gsize);
}

// FP32 and FP64 charge populations only: with both sets in 2 bytes the
// per-node kernel measured faster (0.73 vs 0.76 ms at 256 x 256 x 129, FP16);
// the mixed storage (2-byte f, 4-byte g) runs on it.  Rows are whole bulk
// copies, so their bytes are multiples of 16.
bool lbm_rows_usable(int nx, size_t fsize, size_t gsize) {
    return gsize >= 4 && nx >= 32 && nx <= 256 && (nx * fsize) % 16 == 0 &&
           (nx * gsize) % 16 == 0 && lbm_rows_smem(nx, fsize, gsize) <= 220 * 1024;
}

template <typename T, typename R>
cudaError_t prepare_lbm_rows(int nx, int ny, int nz, int *grid) {
    *grid = 0;
    using F = typename PopT<T>::F;
    using G = typename PopT<T>::G;
    if (!lbm_rows_usable(nx, sizeof(F), sizeof(G))) return cudaSuccess;
    const int sm = (int)lbm_rows_smem(nx, sizeof(F), sizeof(G));
    cudaError_t e;
    for (int v = 0; v < 4; ++v)
        if ((e = allow_max_dynamic_smem(rows_kernel<T, R>(v & 1, v & 2))) != cudaSuccess ||
            (e = allow_max_dynamic_smem(rows_group_kernel<T, R>(v & 1, v & 2))) != cudaSuccess)
            return e;
    const bool part = nx % 32 != 0;
    int dev = 0, nsm = 0, occ_a = 0, occ_b = 0;
    const int tx = rows_block_x(nx);
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, rows_kernel<T, R>(true, part),
                                                           tx, sm)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, rows_kernel<T, R>(false, part),
                                                           tx, sm)) != cudaSuccess)
        return e;
    const long long rows = (long long)ny * (nz - 1);
    *grid = (int)std::min<long long>(rows, (long long)nsm * std::min(occ_a, occ_b));
    return cudaSuccess;
}

template cudaError_t prepare_lbm_rows<double, double>(int, int, int, int *);
template cudaError_t prepare_lbm_rows<float, float>(int, int, int, int *);
template cudaError_t prepare_lbm_rows<__half, float>(int, int, int, int *);
template cudaError_t prepare_lbm_rows<__nv_bfloat16, float>(int, int, int, int *);
template cudaError_t prepare_lbm_rows<Mix16, float>(int, int, int, int *);

template <typename T, typename R>
static StepArgs<T, R> make_step_args(const LbmArgs &la, const StepConst &c) {
    StepArgs<T, R> a;
    for (int d = 0; d < Q; ++d) {
        a.pp.fa[d] = (const typename PopT<T>::F *)la.fa + (size_t)d * c.n;
        a.pp.ha[d] = (const typename PopT<T>::G *)la.ha + (size_t)d * c.n;
        a.pp.fb[d] = (typename PopT<T>::F *)la.fb + (size_t)d * c.n;
        a.pp.hb[d] = (typename PopT<T>::G *)la.hb + (size_t)d * c.n;
    }
    a.phip = (const R *)la.phip;
    a.ez00 = la.ez00;
    a.exa = la.exa;
    a.eya = la.eya;
    a.eza = la.eza;
    a.qout = (R *)la.q;
    a.rout = (R *)la.rho;
    a.uout = (R *)la.u;
    a.vout = (R *)la.v;
    a.wout = (R *)la.w;
    a.zref = (const R *)la.zref;
    a.psum = la.psum;
    a.err = la.err;
    return a;
}

// ---- launches over a group of instances with the same grid ----------------
//
// One launch of the per-node step covers every instance of the group: block
// z = instance * NZ + plane.  Each block copies its instance's arguments and
// constants (about 1.3 KB) into shared memory and runs the same node_block as
// lbm_step_kernel, so an instance's result is bitwise that of a lone context
// on the per-node kernel with the default block shape.
// planes per block of the per-node group kernel
constexpr int kGroupPlanes = 4;

template <typename T, typename R, bool MACROS>
__global__ void __launch_bounds__(128, sizeof(R) == 8 ? 2 : 4)
lbm_group_kernel(const LbmGroupDesc<T, R> *__restrict__ desc, int nz, int zpb) {
    // blockIdx.z: instance and a run of zpb consecutive planes, so that a
    // block's copy of the instance's arguments serves several planes
    __shared__ LbmGroupDesc<T, R> sd;
    const int runs = (nz + zpb - 1) / zpb;
    const int inst = blockIdx.z / runs, z0 = (blockIdx.z - inst * runs) * zpb;
    load_group_desc(sd, desc, inst);
    __syncthreads();
    const int z1 = z0 + zpb < nz ? z0 + zpb : nz;
#pragma unroll 1
    for (int z = z0; z < z1; ++z)
        node_block<T, R, false, MACROS>(sd.a, sd.k, blockIdx.x, blockIdx.y, z, gridDim.x,
                                        gridDim.y, 0, 0);
}

template <typename T, typename R>
size_t lbm_group_desc_bytes(int n) {
    return sizeof(LbmGroupDesc<T, R>) * (size_t)n;
}
template <typename T, typename R>
void build_lbm_group_desc(const LbmArgs *la, const StepConst *c, int n, void *host) {
    LbmGroupDesc<T, R> *d = reinterpret_cast<LbmGroupDesc<T, R> *>(host);
    for (int i = 0; i < n; ++i) {
        d[i].a = make_step_args<T, R>(la[i], c[i]);
        d[i].k = make_kconst<R>(c[i]);
    }
}
template <typename T, typename R>
cudaError_t launch_lbm_group(const void *desc_dev, int n, int nx, int ny, int nz, int bx,
                             bool macros, cudaStream_t s) {
    const dim3 block(bx, 128 / bx, 1);
    const dim3 grid((nx + bx - 1) / bx, (ny + block.y - 1) / block.y,
                    (nz + kGroupPlanes - 1) / kGroupPlanes * n);
    const auto *d = reinterpret_cast<const LbmGroupDesc<T, R> *>(desc_dev);
    if (macros) lbm_group_kernel<T, R, true><<<grid, block, 0, s>>>(d, nz, kGroupPlanes);
    else lbm_group_kernel<T, R, false><<<grid, block, 0, s>>>(d, nz, kGroupPlanes);
    return cudaGetLastError();
}

// The steady-state step of a group on the row kernel: plane z = 0 of every
// instance on the per-node kernel (z0_block_x), then the planes z >= 1 on
// per_inst CTAs of the row kernel per instance.
template <typename T, typename R>
cudaError_t launch_lbm_rows_group(const void *desc_dev, int n, int nx, int ny, int per_inst,
                                  bool macros, cudaStream_t s) {
    const auto *d = reinterpret_cast<const LbmGroupDesc<T, R> *>(desc_dev);
    const int bx = z0_block_x(nx);
    const dim3 g0((nx + bx - 1) / bx, ny, n);
    if (macros) lbm_group_kernel<T, R, true><<<g0, bx, 0, s>>>(d, 1, 1);
    else lbm_group_kernel<T, R, false><<<g0, bx, 0, s>>>(d, 1, 1);
    const size_t sm = lbm_rows_smem(nx, sizeof(typename PopT<T>::F), sizeof(typename PopT<T>::G));
    const dim3 g1(per_inst, n, 1);
    rows_group_kernel<T, R>(macros, nx % 32 != 0)<<<g1, rows_block_x(nx), sm, s>>>(d);
    return cudaGetLastError();
}

template <typename T, typename R>
cudaError_t launch_lbm_step(const LbmArgs &la, const StepConst &c, int local_pops, int e_arrays,
                            bool macros, cudaStream_t s) {
    StepArgs<T, R> a = make_step_args<T, R>(la, c);
    const KConst<R> k = make_kconst<R>(c);
    const bool general = local_pops || e_arrays;
    if (!general && la.rows_grid > 0) {
        // plane z = 0 on the per-node kernel, in blocks of whole warps along
        // x so that its plane sums land in the row kernel's slots
        // [y][x / 32]; then the planes z >= 1 on the row kernel (its
        // shared-memory attribute was set by prepare_lbm_rows)
        const int bx = z0_block_x(c.nx);
        const dim3 g0((c.nx + bx - 1) / bx, c.ny, 1);
        if (macros) lbm_step_kernel<T, R, false, true><<<g0, bx, 0, s>>>(a, k, 0, 0);
        else lbm_step_kernel<T, R, false, false><<<g0, bx, 0, s>>>(a, k, 0, 0);
        const size_t sm = lbm_rows_smem(c.nx, sizeof(typename PopT<T>::F), sizeof(typename PopT<T>::G));
        const int tx = rows_block_x(c.nx);
        rows_kernel<T, R>(macros, c.nx % 32 != 0)<<<la.rows_grid, tx, sm, s>>>(a, k);
        return cudaGetLastError();
    }
    const int bx = la.node_bx > 0 ? la.node_bx : lbm_default_block_x(c.nx);
    dim3 block(bx, 128 / bx, 1);
    dim3 grid((c.nx + block.x - 1) / block.x, (c.ny + block.y - 1) / block.y, c.nz);
#define EHD_LAUNCH(G, M) lbm_step_kernel<T, R, G, M><<<grid, block, 0, s>>>(a, k, local_pops, e_arrays)
    if (general) {
        if (macros) EHD_LAUNCH(true, true);
        else EHD_LAUNCH(true, false);
    } else {
        if (macros) EHD_LAUNCH(false, true);
        else EHD_LAUNCH(false, false);
    }
#undef EHD_LAUNCH
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_init_equilibrium(void *f, void *h, const double *const fields[9],
                                    const double *ref, const StepConst &c, cudaStream_t s) {
    const int bs = 128;
    const long long nb = (c.n + bs - 1) / bs;
    init_equilibrium_kernel<T><<<(unsigned)nb, bs, 0, s>>>(
        (typename PopT<T>::F *)f, (typename PopT<T>::G *)h, fields[0], fields[1], fields[2], fields[3], fields[4], fields[6],
        fields[7], fields[8], ref, c);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_materialize(const void *rho, const void *u, const void *v, const void *w,
                               const void *q, const void *phip, const double *phi00,
                               double *const out[9], int mask, const StepConst &c,
                               cudaStream_t s) {
    dim3 block(c.nx >= 128 ? 128 : 32);
    dim3 grid((c.nx + block.x - 1) / block.x, c.ny, c.nz);
    materialize_kernel<R><<<grid, block, 0, s>>>(
        (const R *)rho, (const R *)u, (const R *)v, (const R *)w, (const R *)q,
        (const R *)phip, phi00, out[0], out[1], out[2], out[3], out[4], out[5], out[6],
        out[7], out[8], mask, c);
    return cudaGetLastError();
}

#define EHD_INST_LBM(T, R) template cudaError_t launch_lbm_step<T, R>(const LbmArgs &, \
    const StepConst &, int, int, bool, cudaStream_t); \
    template size_t lbm_group_desc_bytes<T, R>(int); \
    template void build_lbm_group_desc<T, R>(const LbmArgs *, const StepConst *, int, void *); \
    template cudaError_t launch_lbm_group<T, R>(const void *, int, int, int, int, int, bool, \
                                                cudaStream_t); \
    template cudaError_t launch_lbm_rows_group<T, R>(const void *, int, int, int, int, bool, \
                                                     cudaStream_t);
EHD_INST_LBM(double, double)
EHD_INST_LBM(float, float)
EHD_INST_LBM(__half, float)
EHD_INST_LBM(__nv_bfloat16, float)
EHD_INST_LBM(Mix16, float)
template cudaError_t launch_init_equilibrium<double>(void *, void *, const double *const[9],
                                                    const double *, const StepConst &, cudaStream_t);
template cudaError_t launch_init_equilibrium<float>(void *, void *, const double *const[9],
                                                   const double *, const StepConst &, cudaStream_t);
template cudaError_t launch_init_equilibrium<__half>(void *, void *, const double *const[9],
                                                    const double *, const StepConst &, cudaStream_t);
template cudaError_t launch_init_equilibrium<__nv_bfloat16>(void *, void *,
                                                           const double *const[9],
                                                           const double *, const StepConst &,
                                                           cudaStream_t);
template cudaError_t launch_init_equilibrium<Mix16>(void *, void *, const double *const[9],
                                                   const double *, const StepConst &, cudaStream_t);
template cudaError_t launch_materialize<double>(const void *, const void *, const void *,
                                               const void *, const void *, const void *,
                                               const double *, double *const[9], int,
                                               const StepConst &, cudaStream_t);
template cudaError_t launch_materialize<float>(const void *, const void *, const void *,
                                              const void *, const void *, const void *,
                                              const double *, double *const[9], int,
                                              const StepConst &, cudaStream_t);

cudaError_t launch_reference_init(double *const *out_dev, const StepConst &c, double voltage,
                                  double lz, double dz, cudaStream_t s) {
    const int bs = 256;
    reference_init_kernel<<<(unsigned)((c.n + bs - 1) / bs), bs, 0, s>>>(out_dev, c, voltage,
                                                                         lz, dz);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_fields_to_compute(double *const *out_dev, void *rho, void *u, void *v,
                                     void *w, void *q, long long n, cudaStream_t s) {
    const int bs = 256;
    fields_to_compute_kernel<R><<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(
        out_dev, (R *)rho, (R *)u, (R *)v, (R *)w, (R *)q, n);
    return cudaGetLastError();
}
template cudaError_t launch_fields_to_compute<float>(double *const *, void *, void *, void *,
                                                     void *, void *, long long, cudaStream_t);
template cudaError_t launch_fields_to_compute<double>(double *const *, void *, void *, void *,
                                                      void *, void *, long long, cudaStream_t);

// ---- reference tables -------------------------------------------------------

// Plane means of rho and q from the FP64 fields: m[2z] = mean rho, m[2z+1] =
// mean q (one block per plane, fixed-order FP64 reduction).
__global__ void fields_plane_mean_kernel(const double *__restrict__ rho,
                                         const double *__restrict__ q, double *__restrict__ m,
                                         long long nxy) {
    __shared__ double sr[256], sq[256];
    const int z = blockIdx.x;
    double a = 0.0, b = 0.0;
    for (long long i = threadIdx.x; i < nxy; i += blockDim.x) {
        a += rho[z * nxy + i];
        b += q[z * nxy + i];
    }
    sr[threadIdx.x] = a;
    sq[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sr[threadIdx.x] += sr[threadIdx.x + o];
            sq[threadIdx.x] += sq[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        m[2 * z] = sr[0] / (double)nxy;
        m[2 * z + 1] = sq[0] / (double)nxy;
    }
}

// Plane means from the step kernel's per-block sums (fixed order).
// Plane z's sums of rho and q over its nblk per-warp slots, as means, into
// m[2z], m[2z+1]; fixed summation order.  One block of 256 threads.
__device__ __forceinline__ void psum_reduce_block(const float2 *__restrict__ psum,
                                                  double *__restrict__ m, int nblk, long long nxy,
                                                  int z) {
    __shared__ double wr[8], wq[8];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nblk; i += 256) {
        const float2 v = psum[(size_t)z * nblk + i];
        a += v.x;
        b += v.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        wr[threadIdx.x >> 5] = a;
        wq[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sr = 0.0, sq = 0.0;
        for (int w = 0; w < 8; ++w) {
            sr += wr[w];
            sq += wq[w];
        }
        m[2 * z] = sr / (double)nxy;
        m[2 * z + 1] = sq / (double)nxy;
    }
}

// wdst := the plane means msrc, except that the collector plane takes the
// values of the plane below it, whose g it holds as copies (LBM.cu:1173-1200);
// then the step kernel's table for reading against wread and writing against
// wdst (layout of load_zref).  The references only choose what the stored
// deviations are relative to; any choice is exact in exact arithmetic.
template <typename R>
__device__ __forceinline__ void build_tables_block(const double *__restrict__ msrc, double *wdst,
                                                   const double *wread, R *__restrict__ ktab,
                                                   int nz) {
    for (int z = threadIdx.x; z < nz; z += blockDim.x) {
        const int zs = z == nz - 1 ? nz - 2 : z;
        wdst[2 * z] = msrc[2 * zs];
        wdst[2 * z + 1] = msrc[2 * zs + 1];
    }
    __syncthreads();
    for (int z = threadIdx.x; z < nz; z += blockDim.x) {
        const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;
        const double rw = wdst[2 * z], qw = wdst[2 * z + 1];
        R *k = ktab + 10 * z;
        k[0] = (R)rw;
        k[1] = (R)qw;
        k[2] = (R)(wread[2 * zm] - rw);      // e_z = +1: source z - 1
        k[3] = (R)(wread[2 * z] - rw);       // e_z = 0
        k[4] = (R)(wread[2 * zp] - rw);      // e_z = -1: source z + 1
        k[5] = (R)(wread[2 * zm + 1] - qw);
        k[6] = (R)(wread[2 * z + 1] - qw);
        k[7] = (R)(wread[2 * zp + 1] - qw);
        k[8] = (R)(qw - wdst[2 * zp + 1]);   // copy of g into the plane above
        k[9] = (R)0;
    }
}

template <typename R>
__global__ void build_tables_kernel(const double *__restrict__ msrc, double *wdst,
                                    const double *wread, R *__restrict__ ktab, int nz) {
    build_tables_block<R>(msrc, wdst, wread, ktab, nz);
}

// Blocks 0..nz-1: psum_reduce of plane z; block nz: build_tables (which reads
// the previous means, not the ones reduced here).  One launch per step.
template <typename R>
__global__ void __launch_bounds__(256)
reduce_tables_kernel(const float2 *__restrict__ psum, double *__restrict__ m, int nblk,
                     long long nxy, const double *__restrict__ msrc, double *wdst,
                     const double *wread, R *__restrict__ ktab, int nz) {
    if ((int)blockIdx.x < nz) psum_reduce_block(psum, m, nblk, nxy, blockIdx.x);
    else build_tables_block<R>(msrc, wdst, wread, ktab, nz);
}

// reduce_tables_kernel over a group of instances with the same NZ: block
// (b, i) is block b of instance i's reduction.
template <typename R>
__global__ void __launch_bounds__(256)
reduce_tables_group_kernel(const ReduceDesc *__restrict__ desc) {
    const ReduceDesc &r = desc[blockIdx.y];
    if ((int)blockIdx.x < r.nz) psum_reduce_block(r.psum, r.m, r.nblk, r.nxy, blockIdx.x);
    else build_tables_block<R>(r.msrc, r.wdst, r.wread, (R *)r.ktab, r.nz);
}
template <typename R>
cudaError_t launch_reduce_tables_group(const ReduceDesc *desc_dev, int n, int nz, cudaStream_t s) {
    reduce_tables_group_kernel<R><<<dim3(nz + 1, n), 256, 0, s>>>(desc_dev);
    return cudaGetLastError();
}
template cudaError_t launch_reduce_tables_group<float>(const ReduceDesc *, int, int, cudaStream_t);
template cudaError_t launch_reduce_tables_group<double>(const ReduceDesc *, int, int, cudaStream_t);

cudaError_t launch_fields_plane_mean(const double *rho, const double *q, double *m,
                                     const StepConst &c, cudaStream_t s) {
    fields_plane_mean_kernel<<<c.nz, 256, 0, s>>>(rho, q, m, c.nxy);
    return cudaGetLastError();
}


template <typename R>
cudaError_t launch_build_tables(const double *msrc, double *wdst, const double *wread,
                                void *ktab, const StepConst &c, cudaStream_t s) {
    build_tables_kernel<R><<<1, 256, 0, s>>>(msrc, wdst, wread, (R *)ktab, c.nz);
    return cudaGetLastError();
}
template <typename R>
cudaError_t launch_reduce_tables(const float2 *psum, double *m, int nblk, const double *msrc,
                                 double *wdst, const double *wread, void *ktab,
                                 const StepConst &c, cudaStream_t s) {
    reduce_tables_kernel<R><<<c.nz + 1, 256, 0, s>>>(psum, m, nblk, c.nxy, msrc, wdst, wread,
                                                     (R *)ktab, c.nz);
    return cudaGetLastError();
}
template cudaError_t launch_reduce_tables<float>(const float2 *, double *, int, const double *,
                                                 double *, const double *, void *,
                                                 const StepConst &, cudaStream_t);
template cudaError_t launch_reduce_tables<double>(const float2 *, double *, int, const double *,
                                                  double *, const double *, void *,
                                                  const StepConst &, cudaStream_t);
template cudaError_t launch_build_tables<float>(const double *, double *, const double *, void *,
                                                const StepConst &, cudaStream_t);
template cudaError_t launch_build_tables<double>(const double *, double *, const double *,
                                                 void *, const StepConst &, cudaStream_t);

// number of per-warp partial sums per plane written by the step kernel
// the widest of 64, 32, 16 that leaves the fewest idle lanes at the row end
// (96 -> 32, 80 and 48 -> 16, 256 and 122 -> 64)
int lbm_default_block_x(int nx) {
    int best = 64, waste = 1 << 30;
    for (int bx : {64, 32, 16}) {
        const int w = (nx + bx - 1) / bx * bx - nx;
        if (w < waste) {
            waste = w;
            best = bx;
        }
    }
    return best;
}

int lbm_blocks_per_plane(int nx, int ny, int bx) {
    const int by = 128 / bx;
    return ((nx + bx - 1) / bx) * ((ny + by - 1) / by) * 4;
}

int lbm_rows_slots_per_plane(int nx, int ny) { return ny * ((nx + 31) / 32); }

// ---- seeded initial state ------------------------------------------------------

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    unsigned long long z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// out[k][i] = prof[k][z]; u, v, w at rest plus amp (2 r - 1) on the interior
// planes, r = splitmix64(seed * 2^32 + 3 i + c) / 2^64 (53 bits).
__global__ void seeded_state_kernel(double *const *out, const double *__restrict__ prof,
                                    unsigned long long seed, double amp, StepConst c) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int z = (int)(i / c.nxy);
    const int nz = c.nz;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        double v = prof[k * nz + z];
        if (k >= 1 && k <= 3) {
            v = 0.0;
            if (z > 0 && z < nz - 1 && amp != 0.0) {
                const unsigned long long ctr =
                    (seed << 32) + 3ULL * (unsigned long long)i + (unsigned long long)(k - 1);
                const double r = (double)(splitmix64(ctr) >> 11) * (1.0 / 9007199254740992.0);
                v = amp * (2.0 * r - 1.0);
            }
        }
        out[k][i] = v;
    }
}

// Equilibrium of population d of f (density rho, velocity u) and of g
// (charge ch, advection velocity uc = u + K E): the formulas of
// init_equilibrium_kernel (LBM.cu:110-276), FP64.
__device__ __forceinline__ void eq_pair(int d, double rho, double ux, double uy, double uz,
                                        double ch, double ucx, double ucy, double ucz,
                                        const StepConst &c, double &fe, double &he) {
    const double cs2 = c.cs2;
    const double omusq = 1.0 - 0.5 * (ux * ux + uy * uy + uz * uz) / cs2;
    const double omusq_c = 1.0 - 0.5 * (ucx * ucx + ucy * ucy + ucz * ucz) / cs2;
    const double tux = ux / cs2 / c.cfl, tuy = uy / cs2 / c.cfl, tuz = uz / cs2 / c.cfl;
    const double tcx = ucx / cs2 / c.cfl, tcy = ucy / cs2 / c.cfl, tcz = ucz / cs2 / c.cfl;
    const double cu = ex_of(d) * tux + ey_of(d) * tuy + ez_of(d) * tuz;
    const double cc = ex_of(d) * tcx + ey_of(d) * tcy + ez_of(d) * tcz;
    fe = w_of(d) * rho * (omusq + cu * (1.0 + 0.5 * cu));
    he = w_of(d) * ch * (omusq_c + cc * (1.0 + 0.5 * cc));
}

// A 3D state from a 1 x 1 x NZ column's: on every node of plane z the
// column's populations colv[(s Q + d) nz + z] (s = 0: f, 1: g; the values,
// not deviations), plus the change of their equilibrium that the seeded
// velocity perturbation makes (u0 -> u0 + du with the plane's rho, q and E
// from prof, the column's fields [k][z]), stored against the plane's
// reference ref.  out[1..3] hold du on entry and u0 + du on exit.  The
// potential's non-mean part phi' is the column's, phi - phi00 per plane.
template <typename T, typename R>
__global__ void column_state_kernel(typename PopT<T>::F *__restrict__ f,
                                    typename PopT<T>::G *__restrict__ h, double *const *out,
                                    const double *__restrict__ prof,
                                    const double *__restrict__ colv,
                                    const double *__restrict__ ref, R *__restrict__ phip,
                                    const double *__restrict__ phi00, StepConst c) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const int nz = c.nz, z = (int)(i / c.nxy);
    const double rho = prof[z], ch = prof[4 * nz + z];
    const double u0 = prof[nz + z], v0 = prof[2 * nz + z], w0 = prof[3 * nz + z];
    const double kex = c.K * prof[6 * nz + z], key = c.K * prof[7 * nz + z],
                 kez = c.K * prof[8 * nz + z];
    const double u1 = u0 + out[1][i], v1 = v0 + out[2][i], w1 = w0 + out[3][i];
    out[1][i] = u1;
    out[2][i] = v1;
    out[3][i] = w1;
    phip[i] = (R)(prof[5 * nz + z] - phi00[z]);
    const double rref = ref[2 * z], qref = ref[2 * z + 1];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        double fe0, he0, fe1, he1;
        eq_pair(d, rho, u0, v0, w0, ch, u0 + kex, v0 + key, w0 + kez, c, fe0, he0);
        eq_pair(d, rho, u1, v1, w1, ch, u1 + kex, v1 + key, w1 + kez, c, fe1, he1);
        const double fv = colv[(size_t)d * nz + z] + (fe1 - fe0);
        const double hv = colv[(size_t)(Q + d) * nz + z] + (he1 - he0);
        pst(f + d * c.n + i, (decltype(pld(f)))(fv - w_of(d) * rref));
        pst(h + d * c.n + i, (decltype(pld(h)))(hv - w_of(d) * qref));
    }
}

template <typename T, typename R>
cudaError_t launch_column_state(void *f, void *h, double *const *out_dev, const double *prof_dev,
                                const double *colv_dev, const double *ref, void *phip,
                                const double *phi00, const StepConst &c, cudaStream_t s) {
    const int bs = 128;
    column_state_kernel<T, R><<<(unsigned)((c.n + bs - 1) / bs), bs, 0, s>>>(
        (typename PopT<T>::F *)f, (typename PopT<T>::G *)h, out_dev, prof_dev, colv_dev, ref,
        (R *)phip, phi00, c);
    return cudaGetLastError();
}
#define EHD_INST_COLUMN(T, R)                                                                  \
    template cudaError_t launch_column_state<T, R>(void *, void *, double *const *,           \
                                                   const double *, const double *,            \
                                                   const double *, void *, const double *,    \
                                                   const StepConst &, cudaStream_t);
EHD_INST_COLUMN(double, double)
EHD_INST_COLUMN(float, float)
EHD_INST_COLUMN(__half, float)
EHD_INST_COLUMN(__nv_bfloat16, float)
EHD_INST_COLUMN(Mix16, float)

cudaError_t launch_seeded_state(double *const *out_dev, const double *prof_dev,
                                unsigned long long seed, double amp, const StepConst &c,
                                cudaStream_t s) {
    const int bs = 256;
    seeded_state_kernel<<<(unsigned)((c.n + bs - 1) / bs), bs, 0, s>>>(out_dev, prof_dev, seed,
                                                                       amp, c);
    return cudaGetLastError();
}

}  // namespace ehd
