/*
 * ehd_oracle.c -- CPU FP64 restatement of the reference EHD time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the
 * smoke() check and bench.py's cpu_baseline leg may load it, only as the
 * checker or the timed CPU baseline.  Nothing in the product library links,
 * loads or calls it.
 *
 * It restates, in plain C with OpenMP, the reference's per-step algorithm
 * (gyf135/EHD-convection-3D), one pass per reference kernel, in the same order
 * and with the same FP64 arithmetic:
 *
 *   collide   LBM.cu:295-1091  (gpu_collide_save)
 *   boundary  LBM.cu:1093-1203 (gpu_boundary)
 *   stream    LBM.cu:1205-1279 (gpu_stream)
 *   injection LBM.cu:1281-1353 (gpu_bc_charge)
 *   Poisson   poisson.cu:87-121 (odd_extension), main.cu:194 (forward 3D DFT),
 *             poisson.cu:132-143 (gpu_derivative) with the wavenumbers of
 *             main.cu:110-136, main.cu:200 (inverse 3D DFT),
 *             poisson.cu:154-167 (odd_extract)
 *   E field   poisson.cu:44-73 (gpu_efield, gpu_bc)
 *   equilibrium init LBM.cu:110-276, current LBM.cu:1647-1671.
 *
 * The 3D DFT that the reference takes from cuFFT (closed library) is restated
 * here as a plain mixed-radix complex FFT (any length; radices 2,3,4,5 and a
 * direct DFT for other prime factors), unnormalised forward exp(-2 pi i jk/N)
 * and inverse exp(+2 pi i jk/N), which is cuFFT's documented Z2Z convention.
 *
 * One documented choice: in the reference, threads of the z=0 plane read the
 * rest populations f0/h0 of the z=1 plane (LBM.cu:418-419) while the z=1
 * threads overwrite them in place (LBM.cu:1035-1036), a read/write race.  The
 * oracle reads the pre-collision values (the order in which the hardware
 * schedules the z=0 blocks first).
 *
 * Layout is the reference's: scalars [z][y][x] (x fastest), non-rest
 * populations [d-1][z][y][x] for d = 1..26, rest populations separate
 * (LBM.cu:21-34).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Physical and scheme parameters: the reference's LBM.h:30-80 constants and
 * __device__ scalars, as a runtime struct.  Field order matches ehd_params in
 * include/ehd.h so one ctypes structure serves both. */
typedef struct {
    int32_t nx, ny, nz;       /* nodes; z has electrodes at 0 and nz-1        */
    int32_t pad_;
    double lx, ly, lz;        /* Lx, Ly, Lz                                   */
    double dx, dy, dz;        /* grid spacings                                */
    double dt, cfl;           /* time step and CFL = dt/dx                    */
    double rho0, charge0;     /* reference density, injected charge q0        */
    double voltage, eps;      /* electrode voltage V, permittivity            */
    double diffu, nu, K;      /* charge diffusivity, viscosity, mobility      */
    double uw, exf;           /* moving-wall speed, external x force          */
    double lambda_f;          /* TRT magic parameter for f (reference V)      */
    double lambda_g;          /* TRT magic parameter for g (reference VC)     */
} orc_params;

/* D3Q27 directions in the reference's numbering (stream offsets of
 * LBM.cu:1225-1250: population d at x comes from x - e_d). */
static const int EV[27][3] = {
    {0, 0, 0},
    {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
    {1, 1, 0},  {-1, -1, 0}, {1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, -1},
    {1, -1, 0}, {-1, 1, 0}, {1, 0, -1}, {-1, 0, 1}, {0, 1, -1}, {0, -1, 1},
    {1, 1, 1},  {-1, -1, -1}, {1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {-1, 1, -1},
    {-1, 1, 1}, {1, -1, -1}};

static double WT(int d) { /* LBM.h:73-76 */
    if (d == 0) return 8.0 / 27.0;
    if (d <= 6) return 2.0 / 27.0;
    if (d <= 18) return 1.0 / 54.0;
    return 1.0 / 216.0;
}
static int OPP(int d) { return d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1); }

/* Sign pattern of the moving-upper-wall term, LBM.cu:1145-1170.  Direction 3
 * receives +multis while direction 4 receives nothing (kept as written). */
static const int MW_SIGN[27] = {0, 1, -1, 1, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1,
                                1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};

typedef struct {
    orc_params p;
    size_t n;   /* nodes                                */
    double *f0, *f1, *f2, *h0, *h1, *h2;
    double *f0pre, *h0pre; /* pre-collision rest populations (race choice) */
    double *rho, *q, *u, *v, *w, *phi, *ex, *ey, *ez;
    double *f0bc;          /* LBM.cu:309-311                              */
    double *kx, *ky, *kz;  /* main.cu:110-136                             */
    double *ext;           /* interleaved complex NX*NY*NE                */
    double *ext2;
    int ne;
} orc_ctx;

static inline size_t SIDX(const orc_ctx *c, int x, int y, int z) {
    return (size_t)c->p.nx * ((size_t)c->p.ny * z + y) + x;
}
static inline size_t PIDX(const orc_ctx *c, int x, int y, int z, int d) {
    return (size_t)(d - 1) * c->n + SIDX(c, x, y, z);
}

/* ------------------------------------------------------------------------ */
/* complex FFT (mixed radix, recursive, out of place)                      */
/* ------------------------------------------------------------------------ */

/* Recursive decimation-in-time step.  `in` has element stride `stride`
 * (complex units); `out` is contiguous; `tmp` is scratch of the same length.
 * `w` holds exp(sign 2 pi i k / ntot) for k < ntot, and n divides ntot. */
static void fft_rec(const double *in, double *out, int n, int stride, const double *w,
                    int ntot, double *tmp) {
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    int r = 0;
    if (n % 4 == 0) r = 4;
    else if (n % 2 == 0) r = 2;
    else if (n % 3 == 0) r = 3;
    else if (n % 5 == 0) r = 5;
    else {
        for (int f = 7; f * f <= n; f += 2)
            if (n % f == 0) { r = f; break; }
        if (r == 0) r = n; /* prime: direct DFT */
    }
    const int m = n / r;
    const long step_n = ntot / n; /* w index of exp(sign 2 pi i / n) */
    const long step_r = ntot / r; /* w index of exp(sign 2 pi i / r) */
    if (m > 1)
        for (int j = 0; j < r; ++j)
            fft_rec(in + 2 * (size_t)j * stride, tmp + 2 * (size_t)j * m, m, stride * r, w,
                    ntot, out);
    double sbr[16], sbi[16];
    double *br = sbr, *bi = sbi;
    if (r > 16) {
        br = (double *)malloc(sizeof(double) * r);
        bi = (double *)malloc(sizeof(double) * r);
    }
    for (int k = 0; k < m; ++k) {
        for (int j = 0; j < r; ++j) {
            double xr, xi;
            if (m > 1) {
                xr = tmp[2 * ((size_t)j * m + k)];
                xi = tmp[2 * ((size_t)j * m + k) + 1];
            } else {
                xr = in[2 * (size_t)j * stride];
                xi = in[2 * (size_t)j * stride + 1];
            }
            long t = ((long)j * k % n) * step_n;
            double c = w[2 * t], s = w[2 * t + 1];
            br[j] = xr * c - xi * s;
            bi[j] = xr * s + xi * c;
        }
        for (int q = 0; q < r; ++q) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < r; ++j) {
                long t = ((long)j * q % r) * step_r;
                double c = w[2 * t], s = w[2 * t + 1];
                sr += br[j] * c - bi[j] * s;
                si += br[j] * s + bi[j] * c;
            }
            out[2 * ((size_t)q * m + k)] = sr;
            out[2 * ((size_t)q * m + k) + 1] = si;
        }
    }
    if (r > 16) { free(br); free(bi); }
}

/* In-place 1D FFT of `count` lines of length n, element stride `es`, line
 * stride `ls` (complex units), over an interleaved complex array. */
static void fft_lines(double *a, int n, size_t es, size_t ls, size_t count, int sign) {
    if (n == 1) return;
    double *w = (double *)malloc(sizeof(double) * 2 * n);
    for (int k = 0; k < n; ++k) {
        double ang = sign * 2.0 * M_PI * (double)k / (double)n;
        w[2 * k] = cos(ang);
        w[2 * k + 1] = sin(ang);
    }
#pragma omp parallel
    {
        double *line = (double *)malloc(sizeof(double) * 2 * n);
        double *out = (double *)malloc(sizeof(double) * 2 * n);
        double *tmp = (double *)malloc(sizeof(double) * 2 * n);
#pragma omp for schedule(static)
        for (long l = 0; l < (long)count; ++l) {
            double *base = a + 2 * (size_t)l * ls;
            for (int j = 0; j < n; ++j) {
                line[2 * j] = base[2 * j * es];
                line[2 * j + 1] = base[2 * j * es + 1];
            }
            fft_rec(line, out, n, 1, w, n, tmp);
            for (int j = 0; j < n; ++j) {
                base[2 * j * es] = out[2 * j];
                base[2 * j * es + 1] = out[2 * j + 1];
            }
        }
        free(line);
        free(out);
        free(tmp);
    }
    free(w);
}

/* 3D complex FFT on (NE, NY, NX), x fastest: cufftPlan3d(NE, NY, NX) of
 * main.cu:104.  sign -1 forward, +1 inverse, unnormalised. */
static void fft3d(double *a, int nx, int ny, int ne, int sign) {
    fft_lines(a, nx, 1, nx, (size_t)ny * ne, sign);          /* x lines */
    for (int z = 0; z < ne; ++z)                             /* y lines */
        fft_lines(a + 2 * (size_t)z * nx * ny, ny, nx, 1, nx, sign);
    fft_lines(a, ne, (size_t)nx * ny, 1, (size_t)nx * ny, sign); /* z lines */
}

/* public: 1D FFT for tests */
void orc_fft1d(double *a, int n, int sign) { fft_lines(a, n, 1, n, 1, sign); }

/* ------------------------------------------------------------------------ */
/* context                                                                  */
/* ------------------------------------------------------------------------ */

void orc_destroy(orc_ctx *c);

orc_ctx *orc_create(const orc_params *p) {
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
    c->p = *p;
    c->n = (size_t)p->nx * p->ny * p->nz;
    c->ne = 2 * (p->nz - 1);
    size_t n = c->n;
    c->f0 = calloc(n, sizeof(double));
    c->h0 = calloc(n, sizeof(double));
    c->f0pre = calloc(n, sizeof(double));
    c->h0pre = calloc(n, sizeof(double));
    c->f1 = calloc(26 * n, sizeof(double));
    c->f2 = calloc(26 * n, sizeof(double));
    c->h1 = calloc(26 * n, sizeof(double));
    c->h2 = calloc(26 * n, sizeof(double));
    double **fs[] = {&c->rho, &c->q, &c->u, &c->v, &c->w, &c->phi, &c->ex, &c->ey, &c->ez};
    for (int i = 0; i < 9; ++i) *fs[i] = calloc(n, sizeof(double));
    c->f0bc = calloc(2 * (size_t)p->nx * p->ny, sizeof(double));
    c->kx = calloc(p->nx, sizeof(double));
    c->ky = calloc(p->ny, sizeof(double));
    c->kz = calloc(c->ne, sizeof(double));
    size_t ns = (size_t)p->nx * p->ny * c->ne;
    c->ext = calloc(2 * ns, sizeof(double));
    c->ext2 = calloc(2 * ns, sizeof(double));
    {
        double *all[] = {c->f0, c->h0, c->f0pre, c->h0pre, c->f1, c->f2, c->h1, c->h2,
                         c->rho, c->q, c->u, c->v, c->w, c->phi, c->ex, c->ey, c->ez,
                         c->f0bc, c->kx, c->ky, c->kz, c->ext, c->ext2};
        for (size_t i = 0; i < sizeof(all) / sizeof(all[0]); ++i)
            if (!all[i]) {
                orc_destroy(c);
                return NULL;
            }
    }
    /* wavenumbers, main.cu:110-136 */
    for (int i = 0; i < p->nx; ++i)
        c->kx[i] = (i <= p->nx / 2 ? (double)i : (double)i - p->nx) * 2.0 * M_PI / p->lx;
    for (int i = 0; i < p->ny; ++i)
        c->ky[i] = (i <= p->ny / 2 ? (double)i : (double)i - p->ny) * 2.0 * M_PI / p->ly;
    for (int i = 0; i < c->ne; ++i)
        c->kz[i] = (i <= c->ne / 2 ? (double)i : (double)i - c->ne) * 2.0 * M_PI /
                   (c->ne * p->dz);
    return c;
}

void orc_destroy(orc_ctx *c) {
    if (!c) return;
    double *ps[] = {c->f0, c->h0, c->f0pre, c->h0pre, c->f1, c->f2, c->h1, c->h2,
                    c->rho, c->q, c->u, c->v, c->w, c->phi, c->ex, c->ey, c->ez,
                    c->f0bc, c->kx, c->ky, c->kz, c->ext, c->ext2};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    free(c);
}

static double cs2_of(const orc_params *p) { return 1.0 / 3.0 / (p->cfl * p->cfl); }

/* Equilibrium populations of a node: feq_i = w_i rho (omusq + cu (1 + cu/2)),
 * LBM.cu:143-274 (same polynomial in the collide, LBM.cu:519-660). */
static void equilibrium(const orc_params *p, double dens, double ux, double uy, double uz,
                        double *fe) {
    double cs2 = cs2_of(p);
    double omusq = 1.0 - 0.5 * (ux * ux + uy * uy + uz * uz) / cs2;
    double tux = ux / cs2 / p->cfl, tuy = uy / cs2 / p->cfl, tuz = uz / cs2 / p->cfl;
    fe[0] = WT(0) * dens * omusq;
    for (int d = 1; d < 27; ++d) {
        double cu = EV[d][0] * tux + EV[d][1] * tuy + EV[d][2] * tuz;
        fe[d] = WT(d) * dens * (omusq + cu * (1.0 + 0.5 * cu));
    }
}

/* init_equilibrium, LBM.cu:110-276 */
void orc_init_equilibrium(orc_ctx *c) {
    const orc_params *p = &c->p;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)c->n; ++i) {
        double fe[27], he[27];
        equilibrium(p, c->rho[i], c->u[i], c->v[i], c->w[i], fe);
        equilibrium(p, c->q[i], c->u[i] + p->K * c->ex[i], c->v[i] + p->K * c->ey[i],
                    c->w[i] + p->K * c->ez[i], he);
        c->f0[i] = fe[0];
        c->h0[i] = he[0];
        for (int d = 1; d < 27; ++d) {
            c->f1[(size_t)(d - 1) * c->n + i] = fe[d];
            c->h1[(size_t)(d - 1) * c->n + i] = he[d];
        }
    }
}

void orc_set_fields(orc_ctx *c, const double *rho, const double *u, const double *v,
                    const double *w, const double *q, const double *phi, const double *ex,
                    const double *ey, const double *ez) {
    size_t b = c->n * sizeof(double);
    memcpy(c->rho, rho, b);
    memcpy(c->u, u, b);
    memcpy(c->v, v, b);
    memcpy(c->w, w, b);
    memcpy(c->q, q, b);
    memcpy(c->phi, phi, b);
    memcpy(c->ex, ex, b);
    memcpy(c->ey, ey, b);
    memcpy(c->ez, ez, b);
    orc_init_equilibrium(c);
}

void orc_get_fields(const orc_ctx *c, double *rho, double *u, double *v, double *w,
                    double *q, double *phi, double *ex, double *ey, double *ez) {
    size_t b = c->n * sizeof(double);
    memcpy(rho, c->rho, b);
    memcpy(u, c->u, b);
    memcpy(v, c->v, b);
    memcpy(w, c->w, b);
    memcpy(q, c->q, b);
    memcpy(phi, c->phi, b);
    memcpy(ex, c->ex, b);
    memcpy(ey, c->ey, b);
    memcpy(ez, c->ez, b);
}

/* populations in the reference layout (f0[n], f1[26n], h0[n], h1[26n]) */
void orc_get_pops(const orc_ctx *c, double *f0, double *f1, double *h0, double *h1) {
    memcpy(f0, c->f0, c->n * sizeof(double));
    memcpy(h0, c->h0, c->n * sizeof(double));
    memcpy(f1, c->f1, 26 * c->n * sizeof(double));
    memcpy(h1, c->h1, 26 * c->n * sizeof(double));
}
void orc_set_pops(orc_ctx *c, const double *f0, const double *f1, const double *h0,
                  const double *h1) {
    memcpy(c->f0, f0, c->n * sizeof(double));
    memcpy(c->h0, h0, c->n * sizeof(double));
    memcpy(c->f1, f1, 26 * c->n * sizeof(double));
    memcpy(c->h1, h1, 26 * c->n * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* the LBM part of the step                                                  */
/* ------------------------------------------------------------------------ */

/* gpu_collide_save, LBM.cu:295-1091 (perturb == 0, the only reachable branch:
 * gpu_boundary resets it every step, LBM.cu:1100). */
static void collide(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz;
    const double cs2 = cs2_of(p), dt = p->dt, CFL = p->cfl;
    const double omega_plus = 1.0 / (p->nu / cs2 / dt + 1.0 / 2.0) / dt;
    const double omega_minus = 1.0 / (p->lambda_f / (p->nu / cs2 / dt) + 1.0 / 2.0) / dt;
    const double omega_c_minus = 1.0 / (p->diffu / cs2 / dt + 1.0 / 2.0) / dt;
    const double omega_c_plus = 1.0 / (p->lambda_g / (p->diffu / cs2 / dt) + 1.0 / 2.0) / dt;
    const double tw0rp = omega_plus * dt, tw0rm = omega_minus * dt;
    const double tw0cp = omega_c_plus * dt, tw0cm = omega_c_minus * dt;
    const double sp = 1.0 - 0.5 * dt * omega_plus;
    const double sm = 1.0 - 0.5 * dt * omega_minus;
    const double cflinv = 1.0 / CFL;
    const double cflinv2 = cflinv * cflinv / cs2;

    memcpy(c->f0pre, c->f0, c->n * sizeof(double));
    memcpy(c->h0pre, c->h0, c->n * sizeof(double));

#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t s = SIDX(c, x, y, z);
                if (z == 0) c->f0bc[(size_t)x + (size_t)NX * y] = c->f0pre[s];
                if (z == NZ - 1) c->f0bc[(size_t)NX * NY + x + (size_t)NX * y] = c->f0pre[s];
                double ft[27], ht[27];
                ft[0] = c->f0pre[s];
                ht[0] = c->h0pre[s];
                for (int d = 1; d < 27; ++d) {
                    ft[d] = c->f1[PIDX(c, x, y, z, d)];
                    ht[d] = c->h1[PIDX(c, x, y, z, d)];
                }
                double rho = 0.0, charge = 0.0;
                for (int d = 0; d < 27; ++d) { rho += ft[d]; charge += ht[d]; }
                double rhoinv = 1.0 / rho;
                double Ex = c->ex[s], Ey = c->ey[s], Ez = c->ez[s];
                double fx = charge * Ex + p->exf, fy = charge * Ey, fz = charge * Ez;
                double mx = 0, my = 0, mz = 0;
                for (int d = 1; d < 27; ++d) {
                    mx += EV[d][0] * ft[d];
                    my += EV[d][1] * ft[d];
                    mz += EV[d][2] * ft[d];
                }
                double ux = rhoinv * (mx / CFL + fx * dt * 0.5);
                double uy = rhoinv * (my / CFL + fy * dt * 0.5);
                double uz = rhoinv * (mz / CFL + fz * dt * 0.5);
                if (z == 0) {
                    /* LBM.cu:417-492: velocity of the injector node is the
                     * negated velocity of the z=1 node, rebuilt from z=1
                     * pre-collision populations, z=1 charge and E, but the
                     * LOCAL 1/rho (LBM.cu:477). */
                    size_t s1 = SIDX(c, x, y, 1);
                    double chargem = c->h0pre[s1];
                    double mxm = 0, mym = 0, mzm = 0;
                    for (int d = 1; d < 27; ++d) {
                        double fm = c->f1[PIDX(c, x, y, 1, d)];
                        chargem += c->h1[PIDX(c, x, y, 1, d)];
                        mxm += EV[d][0] * fm;
                        mym += EV[d][1] * fm;
                        mzm += EV[d][2] * fm;
                    }
                    double rhoinvm = 1.0 / rho;
                    double fxm = chargem * c->ex[s1] + p->exf;
                    double fym = chargem * c->ey[s1];
                    double fzm = chargem * c->ez[s1];
                    ux = -rhoinvm * (mxm / CFL + fxm * dt * 0.5);
                    uy = -rhoinvm * (mym / CFL + fym * dt * 0.5);
                    uz = -rhoinvm * (mzm / CFL + fzm * dt * 0.5);
                }
                c->rho[s] = rho;
                c->u[s] = ux;
                c->v[s] = uy;
                c->w[s] = uz;
                c->q[s] = charge;

                double fe[27], he[27];
                equilibrium(p, rho, ux, uy, uz, fe);
                equilibrium(p, charge, ux + p->K * Ex, uy + p->K * Ey, uz + p->K * Ez, he);

                /* Guo force populations, LBM.cu:662-702 */
                double fpop[27];
                double uF = ux * fx + uy * fy + uz * fz;
                fpop[0] = -(WT(0) / cs2) * uF;
                for (int d = 1; d < 27; ++d) {
                    double eu = EV[d][0] * ux + EV[d][1] * uy + EV[d][2] * uz;
                    double acc = 0.0;
                    const double F[3] = {fx, fy, fz}, U[3] = {ux, uy, uz};
                    for (int a = 0; a < 3; ++a)
                        acc += ((EV[d][a] * cflinv - U[a]) + EV[d][a] * eu * cflinv2) * F[a];
                    fpop[d] = (WT(d) / cs2) * acc;
                }
                /* TRT, LBM.cu:704-1089 */
                double f0n = ft[0] - (tw0rp * (ft[0] - fe[0])) + dt * sp * fpop[0];
                double h0n = ht[0] - (tw0cp * (ht[0] - he[0]));
                c->f0[s] = f0n;
                c->h0[s] = h0n;
                for (int d = 1; d < 27; d += 2) {
                    int o = d + 1;
                    double fp = 0.5 * (ft[d] + ft[o]), fmn = 0.5 * (ft[d] - ft[o]);
                    double fep = 0.5 * (fe[d] + fe[o]), fem = 0.5 * (fe[d] - fe[o]);
                    double hp = 0.5 * (ht[d] + ht[o]), hmn = 0.5 * (ht[d] - ht[o]);
                    double hep = 0.5 * (he[d] + he[o]), hem = 0.5 * (he[d] - he[o]);
                    double frp = 0.5 * (fpop[d] + fpop[o]), frm = 0.5 * (fpop[d] - fpop[o]);
                    double src_d = sp * frp + sm * frm;
                    double src_o = sp * frp - sm * frm;
                    c->f2[PIDX(c, x, y, z, d)] =
                        ft[d] - (tw0rp * (fp - fep) + tw0rm * (fmn - fem)) + dt * src_d;
                    c->f2[PIDX(c, x, y, z, o)] =
                        ft[o] - (tw0rp * (fp - fep) + tw0rm * (-fmn + fem)) + dt * src_o;
                    c->h2[PIDX(c, x, y, z, d)] =
                        ht[d] - (tw0cp * (hp - hep) + tw0cm * (hmn - hem));
                    c->h2[PIDX(c, x, y, z, o)] =
                        ht[o] - (tw0cp * (hp - hep) + tw0cm * (-hmn + hem));
                }
            }
}

/* gpu_boundary, LBM.cu:1093-1203 */
static void boundary(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz;
    const double cs2 = cs2_of(p);
    const double multis = 2.0 * p->rho0 * p->uw / cs2 * WT(1) / p->cfl;
    const double multia = 2.0 * p->rho0 * p->uw / cs2 * WT(7) / p->cfl;
    const double multid = 2.0 * p->rho0 * p->uw / cs2 * WT(19) / p->cfl;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            size_t s0 = SIDX(c, x, y, 0), st = SIDX(c, x, y, NZ - 1), sb = SIDX(c, x, y, NZ - 2);
            c->f0[s0] = c->f0bc[(size_t)x + (size_t)NX * y];
            for (int d = 1; d < 27; ++d)
                c->f2[PIDX(c, x, y, 0, d)] = c->f1[PIDX(c, x, y, 0, OPP(d))];
            c->f0[st] = c->f0bc[(size_t)NX * NY + x + (size_t)NX * y];
            for (int d = 1; d < 27; ++d) {
                double m = d <= 6 ? multis : (d <= 18 ? multia : multid);
                c->f2[PIDX(c, x, y, NZ - 1, d)] =
                    c->f1[PIDX(c, x, y, NZ - 1, OPP(d))] + MW_SIGN[d] * m;
            }
            c->h0[st] = c->h0[sb];
            for (int d = 1; d < 27; ++d)
                c->h2[PIDX(c, x, y, NZ - 1, d)] = c->h2[PIDX(c, x, y, NZ - 2, d)];
        }
}

/* gpu_stream, LBM.cu:1205-1279: pull, periodic in x, y and z */
static void stream(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x)
                for (int d = 1; d < 27; ++d) {
                    int xs = (x - EV[d][0] + NX) % NX;
                    int ys = (y - EV[d][1] + NY) % NY;
                    int zs = (z - EV[d][2] + NZ) % NZ;
                    c->f1[PIDX(c, x, y, z, d)] = c->f2[PIDX(c, xs, ys, zs, d)];
                    c->h1[PIDX(c, x, y, z, d)] = c->h2[PIDX(c, xs, ys, zs, d)];
                }
}

/* gpu_bc_charge, LBM.cu:1281-1353: anti-bounce-back injection at z=0 */
static void bc_charge(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            size_t s0 = SIDX(c, x, y, 0);
            c->h0[s0] = -c->h0[s0] + 2.0 * p->charge0 * WT(0);
            for (int d = 1; d < 27; ++d)
                c->h1[PIDX(c, x, y, 0, d)] =
                    -c->h2[PIDX(c, x, y, 0, OPP(d))] + 2.0 * p->charge0 * WT(d);
        }
}

/* ------------------------------------------------------------------------ */
/* Poisson solve and E field                                                  */
/* ------------------------------------------------------------------------ */

/* odd_extension (poisson.cu:87-121) -> forward DFT -> gpu_derivative
 * (poisson.cu:132-143) -> inverse DFT -> odd_extract (poisson.cu:154-167). */
void orc_poisson(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz, NE = c->ne;
    const double V = p->voltage, eps = p->eps, dz = p->dz;
    double *ext = c->ext;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NE; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t e = (size_t)NX * ((size_t)NY * z + y) + x;
                double val;
                if (z == 0) val = 0.0;
                else if (z == 1) val = -c->q[SIDX(c, x, y, z)] / eps - V / dz / dz;
                else if (z < NZ - 1) val = -c->q[SIDX(c, x, y, z)] / eps;
                else if (z == NZ - 1) val = 0.0;
                else if (z < NE - 1) val = c->q[SIDX(c, x, y, NE - z)] / eps;
                else val = c->q[SIDX(c, x, y, 1)] / eps + V / dz / dz;
                ext[2 * e] = val;
                ext[2 * e + 1] = 0.0;
            }
    fft3d(ext, NX, NY, NE, -1);
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NE; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t e = (size_t)NX * ((size_t)NY * z + y) + x;
                double I = c->kx[x], J = c->ky[y], K = c->kz[z];
                double mu = (4.0 / dz / dz) * (sin(K * dz * 0.5) * sin(K * dz * 0.5)) + I * I + J * J;
                if (y == 0 && x == 0 && z == 0) mu = 1.0;
                ext[2 * e] = -ext[2 * e] / mu;
                ext[2 * e + 1] = -ext[2 * e + 1] / mu;
            }
    fft3d(ext, NX, NY, NE, +1);
    const double size = (double)NX * NY * NE;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                size_t s = SIDX(c, x, y, z);
                if (z == 0) c->phi[s] = V;
                else if (z == NZ - 1) c->phi[s] = 0.0;
                else c->phi[s] = ext[2 * s] / size;
            }
}

/* gpu_efield + gpu_bc, poisson.cu:44-73 */
void orc_efield(orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz;
    const double *fi = c->phi;
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < NZ; ++z)
        for (int y = 0; y < NY; ++y)
            for (int x = 0; x < NX; ++x) {
                int xp1 = (x + 1) % NX, yp1 = (y + 1) % NY, zp1 = (z + 1) % NZ;
                int xm1 = (NX + x - 1) % NX, ym1 = (NY + y - 1) % NY, zm1 = (NZ + z - 1) % NZ;
                size_t s = SIDX(c, x, y, z);
                c->ex[s] = 0.5 * (fi[SIDX(c, xm1, y, z)] - fi[SIDX(c, xp1, y, z)]) / p->dx;
                c->ey[s] = 0.5 * (fi[SIDX(c, x, ym1, z)] - fi[SIDX(c, x, yp1, z)]) / p->dy;
                c->ez[s] = 0.5 * (fi[SIDX(c, x, y, zm1)] - fi[SIDX(c, x, y, zp1)]) / p->dz;
            }
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            c->ez[SIDX(c, x, y, 0)] = c->ez[SIDX(c, x, y, 1)];
            c->ez[SIDX(c, x, y, NZ - 1)] = c->ez[SIDX(c, x, y, NZ - 2)];
        }
}

/* One pass of each reference kernel per step, in main.cu:184-206's order. */
void orc_step(orc_ctx *c, int nsteps) {
    for (int i = 0; i < nsteps; ++i) {
        collide(c);
        boundary(c);
        stream(c);
        bc_charge(c);
        orc_poisson(c);
        orc_efield(c);
    }
}

/* Only the LBM part (collide, boundary, stream, injection) -- for tests that
 * feed E from elsewhere. */
void orc_step_lbm(orc_ctx *c) {
    collide(c);
    boundary(c);
    stream(c);
    bc_charge(c);
}

/* Test hooks: the collide pass alone, and the post-collision / post-wall
 * populations f2, h2 (with the in-place rest populations f0, h0). */
void orc_collide_only(orc_ctx *c) { collide(c); }
void orc_get_post(const orc_ctx *c, double *f0, double *f2, double *h0, double *h2) {
    memcpy(f0, c->f0, c->n * sizeof(double));
    memcpy(h0, c->h0, c->n * sizeof(double));
    memcpy(f2, c->f2, 26 * c->n * sizeof(double));
    memcpy(h2, c->h2, 26 * c->n * sizeof(double));
}

/* current(), LBM.cu:1647-1671: q at the collector extrapolated linearly from
 * the two planes below, I = K dy^2 sum_xy q(NZ-1) Ez(NZ-1). */
double orc_current(const orc_ctx *c) {
    const orc_params *p = &c->p;
    const int NX = p->nx, NY = p->ny, NZ = p->nz;
    double I = 0.0;
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            double qt = 2.0 * c->q[SIDX(c, x, y, NZ - 2)] - c->q[SIDX(c, x, y, NZ - 3)];
            I += qt * c->ez[SIDX(c, x, y, NZ - 1)];
        }
    return I * p->K * p->dy * p->dy;
}

/* Set-up helpers used to build identical inputs for the oracle and for the
 * product: the reference's own initialization (LBM.cu:81-96). */
void orc_initialization(orc_ctx *c) {
    const orc_params *p = &c->p;
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                size_t s = SIDX(c, x, y, z);
                c->rho[s] = p->rho0;
                c->q[s] = 0.0;
                c->phi[s] = p->voltage * (p->lz - p->dz * z) / p->lz;
                c->u[s] = c->v[s] = c->w[s] = 0.0;
                c->ex[s] = c->ey[s] = c->ez[s] = 0.0;
            }
    orc_init_equilibrium(c);
}

size_t orc_nodes(const orc_ctx *c) { return c->n; }

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
