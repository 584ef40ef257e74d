// api.cu -- the C ABI (include/ehd.h): context, buffers, the time step, graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ehd.h"
#include "common.cuh"
#include "kernels.h"

using namespace ehd;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define EHD_CK(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(EHD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                              \
    } while (0)

// Makes the context's device current for the scope of one API call.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

FftPlan make_plan(int n) {
    FftPlan p{};
    p.n = n;
    p.nrad = 0;
    while (n % 4 == 0) { p.rad[p.nrad++] = 4; n /= 4; }
    while (n % 2 == 0) { p.rad[p.nrad++] = 2; n /= 2; }
    while (n % 3 == 0) { p.rad[p.nrad++] = 3; n /= 3; }
    while (n % 5 == 0) { p.rad[p.nrad++] = 5; n /= 5; }
    for (int f = 7; n > 1; f += 2)  // remaining odd primes: direct radix-f passes
        while (n % f == 0) { p.rad[p.nrad++] = f; n /= f; }
    return p;
}

}  // namespace

namespace ehd {
// The thread's last-error message, for entry points outside this file.
int set_error(int code, const char *msg) { return fail(code, "%s", msg); }
}  // namespace ehd

struct ehd_ctx;
namespace ehd {
const ehd_params *ctx_params(const ehd_ctx *c);
double *ctx_time(ehd_ctx *c);
}  // namespace ehd

struct ehd_ctx {
    ehd_params p{};
    ehd_config cfg{};
    int prec = EHD_PREC_FP64;
    int device = 0;
    StepConst sc{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t fsize = 8, gsize = 8, rsize = 8;  // f and g storage, compute bytes
    std::vector<void *> allocs;
    size_t bytes = 0;

    void *f[2] = {nullptr, nullptr}, *h[2] = {nullptr, nullptr};
    int cur = 0;  // buffer holding the populations read by the next step
    void *q = nullptr, *rho = nullptr, *u = nullptr, *v = nullptr, *w = nullptr;
    void *phip = nullptr;
    double *phi00 = nullptr, *ez00 = nullptr;
    // Reference tables, indexed by buffer parity (see lbm.cu): populations in
    // buffer p are stored against wref[p]; mean[p] holds the plane means of
    // the state in buffer p; ktab[p] is the step kernel's table for reading
    // buffer p and writing buffer p^1.
    double *wref[2] = {nullptr, nullptr};
    double *mean[2] = {nullptr, nullptr};
    void *ktab[2] = {nullptr, nullptr};
    float2 *psum = nullptr;
    int psum_blocks = 0;   // psum slots per plane of the per-node kernel
    int rows_grid = 0;     // CTAs of the bulk-copy row kernel, 0: not available
    ehd_tuning tune{};     // launch shapes (ehd_set_tuning)
    unsigned generation = 0;  // bumped by ehd_set_tuning
    int *err = nullptr;    // device flag set by a row-kernel wait that gave up
    double *out[9] = {};
    double **out_dev = nullptr;
    double *prof_dev = nullptr;  // 9 x NZ profile for ehd_set_state_seeded
    PoissonArgs pa{};
    double *diag_partial = nullptr, *diag_result = nullptr, *host_diag = nullptr;
    int diag_blocks = 0;

    bool have_state = false;
    bool pops_local = false;  // populations are pre-collision, in place
    bool e_arrays = false;    // E still comes from the uploaded arrays
    bool out_valid = false;   // FP64 field arrays match the state
    long long step = 0;
    double t = 0.0;
    double i0 = 0.0;

    bool use_graphs = true;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [cur][macros]
};

namespace ehd {
const ehd_params *ctx_params(const ehd_ctx *c) { return &c->p; }
double *ctx_time(ehd_ctx *c) { return &c->t; }
}  // namespace ehd

namespace {

int dalloc(ehd_ctx *c, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(EHD_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    c->allocs.push_back(*p);
    c->bytes += bytes;
    return EHD_OK;
}

int validate(const ehd_params *p) {
    if (!p) return fail(EHD_ERR_INVALID, "params is NULL");
    if (p->nx < 1 || p->ny < 1) return fail(EHD_ERR_INVALID, "nx, ny must be >= 1");
    if (p->nz < 4) return fail(EHD_ERR_INVALID, "nz must be >= 4 (got %d)", p->nz);
    if ((long long)p->nx * p->ny * p->nz > (1LL << 31))
        return fail(EHD_ERR_INVALID, "grid too large: nx*ny*nz must be <= 2^31");
    const double pos[] = {p->lx, p->ly, p->lz, p->dx, p->dy, p->dz, p->dt, p->cfl,
                          p->rho0, p->eps, p->diffu, p->nu, p->lambda_f, p->lambda_g};
    const char *names[] = {"lx", "ly", "lz", "dx", "dy", "dz", "dt", "cfl",
                           "rho0", "eps", "diffu", "nu", "lambda_f", "lambda_g"};
    for (int i = 0; i < 14; ++i)
        if (!(pos[i] > 0.0) || !std::isfinite(pos[i]))
            return fail(EHD_ERR_INVALID, "%s must be positive and finite", names[i]);
    const double other[] = {p->charge0, p->voltage, p->K, p->uw, p->exf};
    for (double x : other)
        if (!std::isfinite(x)) return fail(EHD_ERR_INVALID, "non-finite parameter");
    if (p->pad_ != 0) return fail(EHD_ERR_INVALID, "pad_ must be 0");
    return EHD_OK;
}

StepConst make_const(const ehd_params *p) {
    StepConst c{};
    c.nx = p->nx;
    c.ny = p->ny;
    c.nz = p->nz;
    c.nxy = (long long)p->nx * p->ny;
    c.n = c.nxy * p->nz;
    c.dt = p->dt;
    c.cfl = p->cfl;
    c.cs2 = 1.0 / 3.0 / (p->cfl * p->cfl);
    c.cflinv = 1.0 / p->cfl;
    c.cflinv2 = c.cflinv * c.cflinv / c.cs2;
    const double dt = p->dt, cs2 = c.cs2;
    // LBM.cu:297-302
    const double omega_plus = 1.0 / (p->nu / cs2 / dt + 1.0 / 2.0) / dt;
    const double omega_minus = 1.0 / (p->lambda_f / (p->nu / cs2 / dt) + 1.0 / 2.0) / dt;
    const double omega_c_minus = 1.0 / (p->diffu / cs2 / dt + 1.0 / 2.0) / dt;
    const double omega_c_plus = 1.0 / (p->lambda_g / (p->diffu / cs2 / dt) + 1.0 / 2.0) / dt;
    c.tw0rp = omega_plus * dt;
    c.tw0rm = omega_minus * dt;
    c.tw0cp = omega_c_plus * dt;
    c.tw0cm = omega_c_minus * dt;
    const double rates[4] = {c.tw0rp, c.tw0rm, c.tw0cp, c.tw0cm};
    for (int i = 0; i < 4; ++i) {
        c.rate_hi[i] = rates[i] >= 1.0 ? 2.0 : rates[i];
        c.rate_lo[i] = rates[i] >= 1.0 ? 2.0 - rates[i] : 0.0;
    }
    c.sp = 1.0 - 0.5 * dt * omega_plus;  // LBM.cu:987-988
    c.sm = 1.0 - 0.5 * dt * omega_minus;
    c.rho0 = p->rho0;
    c.q0 = p->charge0;
    c.K = p->K;
    c.exf = p->exf;
    c.inv2dx = 0.5 / p->dx;
    c.inv2dy = 0.5 / p->dy;
    c.inv2dz = 0.5 / p->dz;
    // LBM.cu:1137-1139
    const double multis = 2.0 * p->rho0 * p->uw / cs2 * w_of(1) / p->cfl;
    const double multia = 2.0 * p->rho0 * p->uw / cs2 * w_of(7) / p->cfl;
    const double multid = 2.0 * p->rho0 * p->uw / cs2 * w_of(19) / p->cfl;
    for (int d = 0; d < Q; ++d) {
        const double m = d <= 6 ? multis : (d <= 18 ? multia : multid);
        c.mw[d] = mw_sign_of(d) * m;
    }
    return c;
}

int lbm(ehd_ctx *c, bool macros) {
    LbmArgs a{};
    a.fa = c->f[c->cur];
    a.ha = c->h[c->cur];
    a.fb = c->f[c->cur ^ 1];
    a.hb = c->h[c->cur ^ 1];
    a.phip = c->phip;
    a.ez00 = c->ez00;
    a.exa = c->out[6];
    a.eya = c->out[7];
    a.eza = c->out[8];
    a.q = c->q;
    a.rho = c->rho;
    a.u = c->u;
    a.v = c->v;
    a.w = c->w;
    a.zref = c->ktab[c->cur];
    a.psum = c->psum;
    a.err = c->err;
    const int loc = c->pops_local ? 1 : 0, ea = c->e_arrays ? 1 : 0;
    const bool rows = c->rows_grid > 0 && c->tune.lbm_kernel == 0 && !loc && !ea;
    a.rows_grid = rows ? c->rows_grid : 0;
    a.node_bx = c->tune.node_block_x;
    cudaError_t e = cudaErrorInvalidValue;
    switch (c->prec) {
        case EHD_PREC_FP64: e = launch_lbm_step<double, double>(a, c->sc, loc, ea, macros, c->stream); break;
        case EHD_PREC_FP32: e = launch_lbm_step<float, float>(a, c->sc, loc, ea, macros, c->stream); break;
        case EHD_PREC_FP16: e = launch_lbm_step<__half, float>(a, c->sc, loc, ea, macros, c->stream); break;
        case EHD_PREC_BF16: e = launch_lbm_step<__nv_bfloat16, float>(a, c->sc, loc, ea, macros, c->stream); break;
        case EHD_PREC_MIXED: e = launch_lbm_step<Mix16, float>(a, c->sc, loc, ea, macros, c->stream); break;
    }
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "LBM step launch: %s", cudaGetErrorString(e));
    // plane means of the new state, then the references of the next step:
    // buffer p will next be written against the means of the state it holds
    // now (the same phase of the injector's two-step alternation)
    const int p = c->cur;
    const int nblk = rows ? lbm_rows_slots_per_plane(c->p.nx, c->p.ny) : c->psum_blocks;
    // (psum_blocks follows the node kernel's block shape, see ehd_set_tuning)
    e = c->rsize == 8
            ? launch_reduce_tables<double>(c->psum, c->mean[p ^ 1], nblk, c->mean[p], c->wref[p], c->wref[p ^ 1], c->ktab[p ^ 1], c->sc, c->stream)
            : launch_reduce_tables<float>(c->psum, c->mean[p ^ 1], nblk, c->mean[p], c->wref[p], c->wref[p ^ 1], c->ktab[p ^ 1], c->sc, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "reference tables: %s", cudaGetErrorString(e));
    c->cur ^= 1;
    c->pops_local = false;
    return EHD_OK;
}

int poisson(ehd_ctx *c) {
    c->pa.qmean = c->mean[c->cur];
    cudaError_t e = c->prec == EHD_PREC_FP64 ? launch_poisson<double>(c->pa, c->stream)
                                             : launch_poisson<float>(c->pa, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "Poisson launch: %s", cudaGetErrorString(e));
    c->e_arrays = false;
    return EHD_OK;
}

void drop_graphs(ehd_ctx *c) {
    for (auto &row : c->graph)
        for (auto &g : row)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
}

// After a stream synchronisation: a row-kernel wait that gave up leaves the
// state invalid; report it on every later call that returns results.
int check_device_error(ehd_ctx *c) {
    int flag = 0;
    EHD_CK(cudaMemcpy(&flag, c->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag)
        return fail(EHD_ERR_CUDA,
                    "LBM row kernel: a bulk-copy wait did not complete; the state is invalid");
    return EHD_OK;
}

// One steady-state step (pull, E from phi) as a CUDA graph, captured once per
// (buffer parity, macro output) pair.
int step_graph(ehd_ctx *c, bool macros) {
    cudaGraphExec_t &ge = c->graph[c->cur][macros ? 1 : 0];
    if (!ge) {
        cudaGraph_t g = nullptr;
        EHD_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int cur0 = c->cur;
        int r1 = lbm(c, macros);
        int r2 = r1 == EHD_OK ? poisson(c) : r1;
        c->cur = cur0;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (r1 != EHD_OK || r2 != EHD_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            c->use_graphs = false;  // fall back to direct launches for good
            return 1;
        }
        e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            ge = nullptr;
            cudaGetLastError();
            c->use_graphs = false;
            return 1;
        }
    }
    EHD_CK(cudaGraphLaunch(ge, c->stream));
    c->cur ^= 1;
    return EHD_OK;
}

int after_upload(ehd_ctx *c) {
    // references of the uploaded state: its plane means, for both buffers
    const int p = c->cur;
    cudaError_t e = launch_fields_plane_mean(c->out[0], c->out[4], c->mean[p], c->sc, c->stream);
    if (e == cudaSuccess)
        e = c->rsize == 8 ? launch_build_tables<double>(c->mean[p], c->wref[p], c->wref[p], c->ktab[p ^ 1], c->sc, c->stream)
                          : launch_build_tables<float>(c->mean[p], c->wref[p], c->wref[p], c->ktab[p ^ 1], c->sc, c->stream);
    if (e == cudaSuccess)
        e = c->rsize == 8 ? launch_build_tables<double>(c->mean[p], c->wref[p ^ 1], c->wref[p], c->ktab[p], c->sc, c->stream)
                          : launch_build_tables<float>(c->mean[p], c->wref[p ^ 1], c->wref[p], c->ktab[p], c->sc, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "reference tables: %s", cudaGetErrorString(e));
    switch (c->prec) {
        case EHD_PREC_FP64: e = launch_init_equilibrium<double>(c->f[c->cur], c->h[c->cur], c->out, c->wref[p], c->sc, c->stream); break;
        case EHD_PREC_FP32: e = launch_init_equilibrium<float>(c->f[c->cur], c->h[c->cur], c->out, c->wref[p], c->sc, c->stream); break;
        case EHD_PREC_FP16: e = launch_init_equilibrium<__half>(c->f[c->cur], c->h[c->cur], c->out, c->wref[p], c->sc, c->stream); break;
        case EHD_PREC_MIXED: e = launch_init_equilibrium<Mix16>(c->f[c->cur], c->h[c->cur], c->out, c->wref[p], c->sc, c->stream); break;
        default: e = launch_init_equilibrium<__nv_bfloat16>(c->f[c->cur], c->h[c->cur], c->out, c->wref[p], c->sc, c->stream); break;
    }
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "init_equilibrium: %s", cudaGetErrorString(e));
    e = c->prec == EHD_PREC_FP64
            ? launch_fields_to_compute<double>(c->out_dev, c->rho, c->u, c->v, c->w, c->q, c->sc.n, c->stream)
            : launch_fields_to_compute<float>(c->out_dev, c->rho, c->u, c->v, c->w, c->q, c->sc.n, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "fields_to_compute: %s", cudaGetErrorString(e));
    EHD_CK(cudaStreamSynchronize(c->stream));
    c->have_state = true;
    c->pops_local = true;
    c->e_arrays = true;
    c->out_valid = true;
    c->step = 0;
    c->t = 0.0;
    return EHD_OK;
}

int materialize(ehd_ctx *c) {
    if (c->out_valid) return EHD_OK;
    // phi and E stay as uploaded until the first Poisson solve
    const int mask = c->e_arrays ? 1 : 3;
    cudaError_t e =
        c->prec == EHD_PREC_FP64
            ? launch_materialize<double>(c->rho, c->u, c->v, c->w, c->q, c->phip, c->phi00, c->out, mask, c->sc, c->stream)
            : launch_materialize<float>(c->rho, c->u, c->v, c->w, c->q, c->phip, c->phi00, c->out, mask, c->sc, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "materialize: %s", cudaGetErrorString(e));
    c->out_valid = true;
    return EHD_OK;
}

}  // namespace

namespace ehd {
cudaStream_t ctx_stream(const ehd_ctx *c) { return c->stream; }
int ctx_device(const ehd_ctx *c) { return c->device; }
int ctx_precision(const ehd_ctx *c) { return c->prec; }
bool ctx_steady(const ehd_ctx *c) { return c->have_state && !c->pops_local && !c->e_arrays; }
int ctx_parity(const ehd_ctx *c) { return c->cur; }
int ctx_launch_step(ehd_ctx *c, bool macros) {
    const int cur0 = c->cur;
    int r = lbm(c, macros);
    if (r == EHD_OK) r = poisson(c);
    c->cur = cur0;
    return r;
}
unsigned ctx_generation(const ehd_ctx *c) { return c->generation; }
void ctx_tuning(const ehd_ctx *c, ehd_tuning *t) { *t = c->tune; }
int ctx_step_args(ehd_ctx *c, bool macros, LbmArgs *la, StepConst *sc, ReduceDesc *rd,
                  PoissonArgs *pa) {
    (void)macros;
    const int p = c->cur;
    LbmArgs a{};
    a.fa = c->f[p];
    a.ha = c->h[p];
    a.fb = c->f[p ^ 1];
    a.hb = c->h[p ^ 1];
    a.phip = c->phip;
    a.ez00 = c->ez00;
    a.exa = c->out[6];
    a.eya = c->out[7];
    a.eza = c->out[8];
    a.q = c->q;
    a.rho = c->rho;
    a.u = c->u;
    a.v = c->v;
    a.w = c->w;
    a.zref = c->ktab[p];
    a.psum = c->psum;
    a.err = c->err;
    // the steady-state step's kernel, as in lbm(): the row kernel where it is
    // available and chosen, else the per-node kernel
    const bool rows = c->rows_grid > 0 && c->tune.lbm_kernel == 0;
    a.rows_grid = rows ? c->rows_grid : 0;
    a.node_bx = c->tune.node_block_x;
    *la = a;
    *sc = c->sc;
    // the reduction of lbm() for that kernel's plane-sum slots
    rd->psum = c->psum;
    rd->m = c->mean[p ^ 1];
    rd->msrc = c->mean[p];
    rd->wdst = c->wref[p];
    rd->wread = c->wref[p ^ 1];
    rd->ktab = c->ktab[p ^ 1];
    rd->nxy = c->sc.nxy;
    rd->nblk = rows ? lbm_rows_slots_per_plane(c->p.nx, c->p.ny)
                    : lbm_blocks_per_plane(c->p.nx, c->p.ny, c->tune.node_block_x);
    rd->nz = c->p.nz;
    // poisson() after lbm() reads the plane means of the new state
    *pa = c->pa;
    pa->qmean = c->mean[p ^ 1];
    return EHD_OK;
}
double ctx_reference_current(const ehd_ctx *c) { return c->i0; }
void ctx_commit_step(ehd_ctx *c) {
    c->cur ^= 1;
    c->step += 1;
    c->t += c->p.dt;
    c->out_valid = false;
}
}  // namespace ehd

extern "C" {


int ehd_abi_version(void) { return EHD_ABI_VERSION; }

const char *ehd_last_error(void) { return g_err.c_str(); }

int ehd_params_from_groups(ehd_params *p, double T, double M, double C, double Fe) {
    if (!p) return fail(EHD_ERR_INVALID, "params is NULL");
    if (!(T > 0) || !(M > 0) || !(C > 0) || !(Fe > 0))
        return fail(EHD_ERR_INVALID, "T, M, C, Fe must be positive");
    if (!(p->eps > 0) || !(p->rho0 > 0) || !(p->lz > 0) || p->voltage == 0.0)
        return fail(EHD_ERR_INVALID, "eps, rho0, lz, voltage must be set");
    // inverse of LBM.cu:1375-1378
    p->K = std::sqrt(p->eps / p->rho0) / M;
    p->nu = p->eps * p->voltage / (p->K * T * p->rho0);
    p->charge0 = C * p->voltage * p->eps / (p->lz * p->lz);
    p->diffu = p->K * p->voltage / Fe;
    return EHD_OK;
}

int ehd_groups_from_params(const ehd_params *p, double *T, double *M, double *C, double *Fe) {
    if (!p) return fail(EHD_ERR_INVALID, "params is NULL");
    if (M) *M = std::sqrt(p->eps / p->rho0) / p->K;
    if (T) *T = p->eps * p->voltage / p->K / p->nu / p->rho0;
    if (C) *C = p->charge0 * p->lz * p->lz / (p->voltage * p->eps);
    if (Fe) *Fe = p->K * p->voltage / p->diffu;
    return EHD_OK;
}

int ehd_create(const ehd_params *params, const ehd_config *config, ehd_ctx **out) {
    if (!out) return fail(EHD_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int r = validate(params);
    if (r != EHD_OK) return r;
    ehd_config cfg{};
    if (config) cfg = *config;
    if (cfg.precision < EHD_PREC_FP64 || cfg.precision > EHD_PREC_MIXED)
        return fail(EHD_ERR_INVALID, "unknown precision %d", cfg.precision);
    int ndev = 0;
    EHD_CK(cudaGetDeviceCount(&ndev));
    if (cfg.device < 0 || cfg.device >= ndev)
        return fail(EHD_ERR_INVALID, "device %d out of range (%d devices)", cfg.device, ndev);
    DeviceGuard dg(cfg.device);
    if (!dg.ok) return fail(EHD_ERR_CUDA, "cudaSetDevice(%d) failed", cfg.device);

    ehd_ctx *c = new ehd_ctx();
    c->p = *params;
    c->cfg = cfg;
    c->prec = cfg.precision;
    c->device = cfg.device;
    c->sc = make_const(params);
    c->use_graphs = !(cfg.flags & EHD_FLAG_NO_GRAPH);
    c->fsize = c->prec == EHD_PREC_FP64 ? 8 : (c->prec == EHD_PREC_FP32 ? 4 : 2);
    c->gsize = c->prec == EHD_PREC_FP64 ? 8 : (c->prec == EHD_PREC_FP32 || c->prec == EHD_PREC_MIXED ? 4 : 2);
    c->rsize = c->prec == EHD_PREC_FP64 ? 8 : 4;
    auto bail = [&](int code) {
        ehd_destroy(c);
        return code;
    };
    if (cfg.stream) {
        c->stream = (cudaStream_t)cfg.stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            return fail(EHD_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        }
        c->own_stream = true;
    }
    const size_t n = (size_t)c->sc.n;
    const int nx = params->nx, ny = params->ny, nz = params->nz;
    for (int i = 0; i < 2; ++i) {
        if ((r = dalloc(c, &c->f[i], (size_t)Q * n * c->fsize))) return bail(r);
        if ((r = dalloc(c, &c->h[i], (size_t)Q * n * c->gsize))) return bail(r);
    }
    void **macro[] = {&c->q, &c->rho, &c->u, &c->v, &c->w, &c->phip};
    for (void **m : macro)
        if ((r = dalloc(c, m, n * c->rsize))) return bail(r);
    if ((r = dalloc(c, (void **)&c->phi00, sizeof(double) * nz))) return bail(r);
    if ((r = dalloc(c, (void **)&c->ez00, sizeof(double) * nz))) return bail(r);
    for (int i = 0; i < 2; ++i) {
        if ((r = dalloc(c, (void **)&c->wref[i], sizeof(double) * 2 * nz))) return bail(r);
        if ((r = dalloc(c, (void **)&c->mean[i], sizeof(double) * 2 * nz))) return bail(r);
        if ((r = dalloc(c, &c->ktab[i], c->rsize * 10 * nz))) return bail(r);
    }
    c->tune.lbm_kernel = (cfg.flags & EHD_FLAG_NODE_KERNEL) ? 1 : 0;
    c->tune.node_block_x = lbm_default_block_x(nx);
    c->psum_blocks = lbm_blocks_per_plane(nx, ny, c->tune.node_block_x);
    {
        // the bulk-copy row kernel for steady-state steps, where it applies
        cudaError_t e = cudaSuccess;
        switch (c->prec) {
            case EHD_PREC_FP64: e = prepare_lbm_rows<double, double>(nx, ny, nz, &c->rows_grid); break;
            case EHD_PREC_FP32: e = prepare_lbm_rows<float, float>(nx, ny, nz, &c->rows_grid); break;
            case EHD_PREC_FP16: e = prepare_lbm_rows<__half, float>(nx, ny, nz, &c->rows_grid); break;
            case EHD_PREC_MIXED: e = prepare_lbm_rows<Mix16, float>(nx, ny, nz, &c->rows_grid); break;
            default: e = prepare_lbm_rows<__nv_bfloat16, float>(nx, ny, nz, &c->rows_grid); break;
        }
        if (e != cudaSuccess) return bail(fail(EHD_ERR_CUDA, "row kernel set-up: %s", cudaGetErrorString(e)));
    }
    {
        // room for the plane sums of every launch shape ehd_set_tuning allows
        int slots = c->rows_grid > 0 ? lbm_rows_slots_per_plane(nx, ny) : 0;
        for (int bx = 16; bx <= 128; bx *= 2) slots = std::max(slots, lbm_blocks_per_plane(nx, ny, bx));
        if ((r = dalloc(c, (void **)&c->psum, sizeof(float2) * (size_t)slots * nz))) return bail(r);
    }
    if ((r = dalloc(c, (void **)&c->err, sizeof(int)))) return bail(r);
    for (int i = 0; i < 9; ++i)
        if ((r = dalloc(c, (void **)&c->out[i], sizeof(double) * n))) return bail(r);
    if ((r = dalloc(c, (void **)&c->out_dev, sizeof(double *) * 9))) return bail(r);
    if ((r = dalloc(c, (void **)&c->prof_dev, sizeof(double) * 9 * nz))) return bail(r);

    // Poisson solver set-up: replaces cufftPlan3d and the wavenumber tables
    // (main.cu:104-143)
    PoissonArgs &pa = c->pa;
    pa.nx = nx;
    pa.ny = ny;
    pa.nz = nz;
    pa.nxh = nx / 2 + 1;
    pa.split = 1;
    pa.pitch = (pa.nxh + 15) / 16 * 16;
    const size_t c2 = 2 * c->rsize;  // complex compute type
    {
        int rows = 16;
        while (rows > 1 && (size_t)2 * rows * nx * c2 > 64 * 1024) rows >>= 1;
        pa.rows_per_block = rows;
        int cols = (int)(128 / c2);
        while (cols > 1 && (size_t)2 * cols * ny * c2 > 160 * 1024) cols >>= 1;
        pa.cols_per_block = cols;
        if ((size_t)2 * rows * nx * c2 > 200 * 1024 || (size_t)2 * cols * ny * c2 > 200 * 1024)
            return bail(fail(EHD_ERR_INVALID, "nx or ny too large for the in-shared-memory FFT"));
        c->tune.fft_rows = rows;
        c->tune.fft_cols = cols;
    }
    pa.px = make_plan(nx);
    pa.py = make_plan(ny);
    const size_t nspec = (size_t)(nz - 2) * ny * pa.pitch;
    if ((r = dalloc(c, &pa.spec, nspec * c2))) return bail(r);
    if ((r = dalloc(c, (void **)&pa.rowsum, sizeof(double) * (size_t)(nz - 2) * ny))) return bail(r);
    if ((r = dalloc(c, (void **)&pa.planesum, sizeof(double) * nz))) return bail(r);
    void *twx = nullptr, *twy = nullptr;
    if ((r = dalloc(c, &twx, (size_t)nx * c2))) return bail(r);
    if ((r = dalloc(c, &twy, (size_t)ny * c2))) return bail(r);
    const size_t nmodes = (size_t)pa.nxh * ny;
    // z solve: sine transform, with compile-time FFT passes where 2 (nz - 1)
    // is one of their sizes and run-time ones where the transforms of a few
    // modes fit in shared memory; else the Thomas solve with its pivot table
    // and sweep scratch
    const int lz2 = 2 * (nz - 1);
    bool zdst = poisson_fast_size(lz2);
    if (!zdst) {
        int tb = 16;
        while (tb > 1 && zdst_rt_smem(lz2, tb, c->rsize) > 160 * 1024) tb >>= 1;
        if (zdst_rt_smem(lz2, tb, c->rsize) <= 160 * 1024) {
            zdst = true;
            pa.ztb = tb;
            pa.pz = make_plan(lz2);
        }
    }
    // where 2 (nz - 1) is not a compile-time size, the Thomas solve stays
    // available beside the run-time sine transform (ehd_tuning.z_solve)
    const bool thomas = !poisson_fast_size(lz2);
    double *cpt = nullptr;
    void *twz = nullptr, *cps = nullptr;
    const bool split = poisson_split_grid(nx, ny, nz, c->rsize);
    if (split) {
        if ((r = dalloc(c, &cps, c->rsize * nmodes * (size_t)((nz - 1) / 2)))) return bail(r);
    }
    if (zdst) {
        if ((r = dalloc(c, &twz, c->rsize * (size_t)(2 * lz2 + lz2 / 2 + 1)))) return bail(r);
    }
    if (thomas) {
        if ((r = dalloc(c, (void **)&cpt, sizeof(double) * nmodes * (size_t)(nz - 2)))) return bail(r);
        if ((r = dalloc(c, (void **)&pa.dpw, sizeof(double2) * nmodes * (size_t)(nz - 2)))) return bail(r);
    }
    pa.twx = twx;
    pa.twy = twy;
    pa.twz = twz;
    pa.lx = params->lx;
    pa.ly = params->ly;
    pa.cpt = cpt;
    pa.cps = cps;
    pa.phi00 = c->phi00;
    pa.ez00 = c->ez00;
    pa.q = c->q;
    pa.phip = c->phip;
    pa.eps = params->eps;
    pa.voltage = params->voltage;
    pa.dz = params->dz;
    {
        cudaError_t e = c->rsize == 8 ? prepare_poisson<double>(pa) : prepare_poisson<float>(pa);
        if (e != cudaSuccess)
            return bail(fail(EHD_ERR_CUDA, "Poisson set-up: %s", cudaGetErrorString(e)));
    }
    {
        auto table = [&](int N, void *dst) -> cudaError_t {
            std::vector<double> t(2 * (size_t)N);
            for (int k = 0; k < N; ++k) {
                const double a = -2.0 * M_PI * (double)k / (double)N;
                t[2 * k] = std::cos(a);
                t[2 * k + 1] = std::sin(a);
            }
            if (c->rsize == 8)
                return cudaMemcpy(dst, t.data(), sizeof(double) * 2 * N, cudaMemcpyHostToDevice);
            std::vector<float> tf(t.begin(), t.end());
            return cudaMemcpy(dst, tf.data(), sizeof(float) * 2 * N, cudaMemcpyHostToDevice);
        };
        EHD_CK(table(nx, twx));
        EHD_CK(table(ny, twy));
        if (zdst) {
            // twiddles, then the z eigenvalues 4 sin^2(pi k / L), k = 0..L/2
            std::vector<double> t(2 * (size_t)lz2 + lz2 / 2 + 1);
            for (int k = 0; k < lz2; ++k) {
                const double a = -2.0 * M_PI * (double)k / (double)lz2;
                t[2 * k] = std::cos(a);
                t[2 * k + 1] = std::sin(a);
            }
            for (int k = 0; k <= lz2 / 2; ++k) {
                const double sn = std::sin(M_PI * (double)k / (double)lz2);
                t[2 * (size_t)lz2 + k] = 4.0 * sn * sn;
            }
            if (c->rsize == 8) {
                EHD_CK(cudaMemcpy(twz, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice));
            } else {
                std::vector<float> tf(t.begin(), t.end());
                EHD_CK(cudaMemcpy(twz, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice));
            }
        }
        // Thomas pivots per mode (kx, ky): beta = 2 + (kx^2 + ky^2) dz^2 with
        // the wavenumbers of main.cu:110-129, cp_0 = -1/beta,
        // cp_i = 1/(-beta - cp_{i-1})
        std::vector<double> hx(pa.nxh), hy(ny);
        for (int i = 0; i < pa.nxh; ++i) {
            const double k = (double)i * 2.0 * M_PI / params->lx;
            hx[i] = k * k;
        }
        for (int j = 0; j < ny; ++j) {
            const double k = (j <= ny / 2 ? (double)j : (double)j - ny) * 2.0 * M_PI / params->ly;
            hy[j] = k * k;
        }
        const int n = nz - 2;
        const double dz2 = params->dz * params->dz;
        if (split) {
            // the split-y slab kernel's two-sided table, layout [kx][j][r][k']
            // with ky = S k' + j, in the compute type: for n = NZ - 2 (odd)
            // interior planes, c_0..c_{m-1} (m = (n - 1)/2, the pivots of
            // either half) and mu = 1/(-beta - 2 c_{m-1}) (the middle plane)
            const int S = ny / 64, m = (n - 1) / 2;
            std::vector<double> cp(nmodes * (size_t)(m + 1));
            size_t o = 0;
            for (int i = 0; i < pa.nxh; ++i)
                for (int j = 0; j < S; ++j) {
                    double prev[64];
                    for (int kp = 0; kp < 64; ++kp) prev[kp] = 0.0;
                    for (int z = 0; z <= m; ++z)
                        for (int kp = 0; kp < 64; ++kp) {
                            const double beta = 2.0 + (hx[i] + hy[S * kp + j]) * dz2;
                            if (z < m) {
                                prev[kp] = 1.0 / (-beta - prev[kp]);
                                cp[o++] = prev[kp];
                            } else {
                                cp[o++] = 1.0 / (-beta - 2.0 * prev[kp]);
                            }
                        }
                }
            if (c->rsize == 8) {
                EHD_CK(cudaMemcpy(cps, cp.data(), sizeof(double) * cp.size(), cudaMemcpyHostToDevice));
            } else {
                std::vector<float> cf(cp.begin(), cp.end());
                EHD_CK(cudaMemcpy(cps, cf.data(), sizeof(float) * cf.size(), cudaMemcpyHostToDevice));
            }
        }
        if (thomas) {
            // layout [i][ky*nxh + kx]
            std::vector<double> cp(nmodes * (size_t)n);
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < pa.nxh; ++i) {
                    const size_t m = (size_t)j * pa.nxh + i;
                    const double beta = 2.0 + (hx[i] + hy[j]) * dz2;
                    double prev = 0.0;
                    for (int z = 0; z < n; ++z) {
                        prev = 1.0 / (-beta - prev);
                        cp[(size_t)z * nmodes + m] = prev;
                    }
                }
            EHD_CK(cudaMemcpy(cpt, cp.data(), sizeof(double) * cp.size(), cudaMemcpyHostToDevice));
        }
    }
    EHD_CK(cudaMemcpy(c->out_dev, c->out, sizeof(double *) * 9, cudaMemcpyHostToDevice));
    EHD_CK(cudaMemset(c->phip, 0, n * c->rsize));
    EHD_CK(cudaMemset(c->err, 0, sizeof(int)));
    EHD_CK(cudaMemset(c->phi00, 0, sizeof(double) * nz));
    EHD_CK(cudaMemset(c->ez00, 0, sizeof(double) * nz));
    // diagnostics scratch
    c->diag_blocks = (int)std::min<long long>(1024, (c->sc.n + 2047) / 2048);
    if (c->diag_blocks < 1) c->diag_blocks = 1;
    if ((r = dalloc(c, (void **)&c->diag_partial, sizeof(double) * 5 * c->diag_blocks))) return bail(r);
    if ((r = dalloc(c, (void **)&c->diag_result, sizeof(double) * 8))) return bail(r);
    {
        cudaError_t e = cudaMallocHost((void **)&c->host_diag, sizeof(double) * 8);
        if (e != cudaSuccess) return bail(fail(EHD_ERR_NOMEM, "cudaMallocHost failed"));
    }
    *out = c;
    return EHD_OK;
}

int ehd_destroy(ehd_ctx *c) {
    if (!c) return EHD_OK;
    DeviceGuard dg(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    for (void *p : c->allocs) cudaFree(p);
    if (c->host_diag) cudaFreeHost(c->host_diag);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return EHD_OK;
}

int ehd_device_bytes(const ehd_ctx *c, size_t *bytes) {
    if (!c || !bytes) return fail(EHD_ERR_INVALID, "NULL argument");
    *bytes = c->bytes;
    return EHD_OK;
}

int ehd_get_tuning(const ehd_ctx *c, ehd_tuning *t) {
    if (!c || !t) return fail(EHD_ERR_INVALID, "NULL argument");
    *t = c->tune;
    return EHD_OK;
}

int ehd_set_tuning(ehd_ctx *c, const ehd_tuning *t) {
    if (!c || !t) return fail(EHD_ERR_INVALID, "NULL argument");
    if (t->lbm_kernel != 0 && t->lbm_kernel != 1) return fail(EHD_ERR_INVALID, "lbm_kernel must be 0 or 1");
    if (t->poisson_path != 0 && t->poisson_path != 1)
        return fail(EHD_ERR_INVALID, "poisson_path must be 0 or 1");
    if (t->z_solve != 0 && t->z_solve != 1) return fail(EHD_ERR_INVALID, "z_solve must be 0 or 1");
    const int bx = t->node_block_x;
    if (bx != 16 && bx != 32 && bx != 64 && bx != 128)
        return fail(EHD_ERR_INVALID, "node_block_x must be 16, 32, 64 or 128 (got %d)", bx);
    const size_t c2 = 2 * c->rsize;
    if (t->fft_rows < 1 || t->fft_cols < 1 ||
        (size_t)2 * t->fft_rows * c->p.nx * c2 > 200 * 1024 ||
        (size_t)2 * t->fft_cols * c->p.ny * c2 > 200 * 1024)
        return fail(EHD_ERR_INVALID, "fft_rows/fft_cols out of range for the shared-memory FFT");
    for (int i : t->reserved)
        if (i != 0) return fail(EHD_ERR_INVALID, "reserved fields must be 0");
    DeviceGuard dg(c->device);
    EHD_CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->tune = *t;
    c->generation += 1;
    c->psum_blocks = lbm_blocks_per_plane(c->p.nx, c->p.ny, bx);
    c->pa.rows_per_block = t->fft_rows;
    c->pa.cols_per_block = t->fft_cols;
    c->pa.split = t->poisson_path == 0 ? 1 : 0;
    c->pa.thomas = t->z_solve == 1 && c->pa.cpt ? 1 : 0;
    return EHD_OK;
}

int ehd_set_fields(ehd_ctx *c, const double *rho, const double *u, const double *v,
                   const double *w, const double *q, const double *phi, const double *ex,
                   const double *ey, const double *ez) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    const double *in[9] = {rho, u, v, w, q, phi, ex, ey, ez};
    for (int i = 0; i < 9; ++i)
        if (!in[i]) return fail(EHD_ERR_INVALID, "field %d is NULL", i);
    DeviceGuard dg(c->device);
    const size_t b = sizeof(double) * (size_t)c->sc.n;
    for (int i = 0; i < 9; ++i)
        EHD_CK(cudaMemcpyAsync(c->out[i], in[i], b, cudaMemcpyHostToDevice, c->stream));
    return after_upload(c);
}

int ehd_initialize(ehd_ctx *c) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    DeviceGuard dg(c->device);
    cudaError_t e = launch_reference_init(c->out_dev, c->sc, c->p.voltage, c->p.lz, c->p.dz,
                                          c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "initialization: %s", cudaGetErrorString(e));
    return after_upload(c);
}

int ehd_get_fields(ehd_ctx *c, double *rho, double *u, double *v, double *w, double *q,
                   double *phi, double *ex, double *ey, double *ez) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    double *dst[9] = {rho, u, v, w, q, phi, ex, ey, ez};
    int r = materialize(c);
    if (r != EHD_OK) return r;
    const size_t b = sizeof(double) * (size_t)c->sc.n;
    for (int i = 0; i < 9; ++i)
        if (dst[i]) EHD_CK(cudaMemcpyAsync(dst[i], c->out[i], b, cudaMemcpyDeviceToHost, c->stream));
    EHD_CK(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int ehd_step(ehd_ctx *c, int nsteps) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    if (nsteps < 0) return fail(EHD_ERR_INVALID, "nsteps < 0");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    for (int i = 0; i < nsteps; ++i) {
        const bool macros = (i == nsteps - 1);
        int r;
        if (c->pops_local || c->e_arrays || !c->use_graphs) {
            if ((r = lbm(c, macros)) != EHD_OK) return r;
            if ((r = poisson(c)) != EHD_OK) return r;
        } else {
            r = step_graph(c, macros);
            if (r == 1) {  // capture unavailable: direct launches
                if ((r = lbm(c, macros)) != EHD_OK) return r;
                if ((r = poisson(c)) != EHD_OK) return r;
            } else if (r != EHD_OK) {
                return r;
            }
        }
        c->step += 1;
        c->t += c->p.dt;
    }
    if (nsteps > 0) c->out_valid = false;
    return EHD_OK;
}

int ehd_stream_collide_save(ehd_ctx *c) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    int r = lbm(c, true);
    if (r != EHD_OK) return r;
    c->out_valid = false;
    return EHD_OK;
}

int ehd_poisson(ehd_ctx *c) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    int r = poisson(c);
    if (r != EHD_OK) return r;
    c->out_valid = false;
    return EHD_OK;
}

int ehd_synchronize(ehd_ctx *c) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    DeviceGuard dg(c->device);
    EHD_CK(cudaStreamSynchronize(c->stream));
    return check_device_error(c);
}

int ehd_set_reference_current(ehd_ctx *c, double i0) {
    if (!c) return fail(EHD_ERR_INVALID, "ctx is NULL");
    if (!std::isfinite(i0)) return fail(EHD_ERR_INVALID, "i0 not finite");
    c->i0 = i0;
    return EHD_OK;
}

static DiagArgs diag_args(ehd_ctx *c) {
    DiagArgs a{};
    a.nx = c->p.nx;
    a.ny = c->p.ny;
    a.nz = c->p.nz;
    a.rho = c->rho;
    a.u = c->u;
    a.v = c->v;
    a.w = c->w;
    a.q = c->q;
    a.phip = c->phip;
    a.ez00 = c->ez00;
    a.ez = c->e_arrays ? c->out[8] : nullptr;
    a.inv2dz = c->sc.inv2dz;
    a.partial = c->diag_partial;
    a.result = c->diag_result;
    a.nblocks = c->diag_blocks;
    return a;
}

int ehd_diagnostics(ehd_ctx *c, ehd_diag *o) {
    if (!c || !o) return fail(EHD_ERR_INVALID, "NULL argument");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    const DiagArgs a = diag_args(c);
    cudaError_t e = c->rsize == 8 ? launch_diag<double>(a, c->stream) : launch_diag<float>(a, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "diagnostics: %s", cudaGetErrorString(e));
    EHD_CK(cudaMemcpyAsync(c->host_diag, c->diag_result, sizeof(double) * 5,
                           cudaMemcpyDeviceToHost, c->stream));
    EHD_CK(cudaStreamSynchronize(c->stream));
    if (int rc = check_device_error(c)) return rc;
    const double *r = c->host_diag;
    const double dv = c->p.dx * c->p.dy * c->p.dz;
    std::memset(o, 0, sizeof(*o));
    o->current = r[0] * c->p.K * c->p.dy * c->p.dy;  // LBM.cu:1669
    o->nu_e = c->i0 != 0.0 ? o->current / c->i0 : 0.0;
    o->kinetic_energy = 0.5 * r[1] * dv;
    o->total_charge = r[2] * dv;
    o->umax = r[3];
    o->time = c->t;
    o->step = c->step;
    o->nonfinite = r[4] > 0.0 ? 1 : 0;
    return EHD_OK;
}

int ehd_current(ehd_ctx *c, double *current) {
    if (!c || !current) return fail(EHD_ERR_INVALID, "NULL argument");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state: call ehd_set_fields first");
    DeviceGuard dg(c->device);
    const DiagArgs a = diag_args(c);
    cudaError_t e = c->rsize == 8 ? launch_current<double>(a, c->stream) : launch_current<float>(a, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "current: %s", cudaGetErrorString(e));
    EHD_CK(cudaMemcpyAsync(c->host_diag, c->diag_result, sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    EHD_CK(cudaStreamSynchronize(c->stream));
    if (int rc = check_device_error(c)) return rc;
    *current = c->host_diag[0] * c->p.K * c->p.dy * c->p.dy;  // LBM.cu:1669
    return EHD_OK;
}

int ehd_set_state_seeded(ehd_ctx *c, const double *profile, uint64_t seed, double amp) {
    if (!c || !profile) return fail(EHD_ERR_INVALID, "NULL argument");
    if (!std::isfinite(amp)) return fail(EHD_ERR_INVALID, "amp not finite");
    DeviceGuard dg(c->device);
    EHD_CK(cudaMemcpyAsync(c->prof_dev, profile, sizeof(double) * 9 * c->p.nz,
                           cudaMemcpyHostToDevice, c->stream));
    cudaError_t e = launch_seeded_state(c->out_dev, c->prof_dev, (unsigned long long)seed, amp,
                                        c->sc, c->stream);
    if (e != cudaSuccess) return fail(EHD_ERR_CUDA, "seeded state: %s", cudaGetErrorString(e));
    return after_upload(c);
}

int ehd_hydrostatic_column(const ehd_params *params, const ehd_config *config, int nsteps,
                           ehd_ctx **column, double *i0) {
    if (!params || !column) return fail(EHD_ERR_INVALID, "NULL argument");
    if (nsteps < 0) return fail(EHD_ERR_INVALID, "nsteps < 0");
    *column = nullptr;
    ehd_params q = *params;
    q.nx = 1;
    q.ny = 1;
    q.lx = params->dx;
    q.ly = params->dy;
    ehd_ctx *col = nullptr;
    int r = ehd_create(&q, config, &col);
    if (r != EHD_OK) return r;
    // I0: the mean of the currents after nsteps and nsteps + 1 steps; the
    // column is left after nsteps + 1
    ehd_diag d{}, d1{};
    if ((r = ehd_initialize(col)) == EHD_OK && (r = ehd_step(col, nsteps)) == EHD_OK &&
        (r = ehd_diagnostics(col, &d)) == EHD_OK && (r = ehd_step(col, 1)) == EHD_OK)
        r = ehd_diagnostics(col, &d1);
    if (r != EHD_OK) {
        ehd_destroy(col);
        return r;
    }
    if (i0) *i0 = 0.5 * (d.current + d1.current) * (double)params->nx * (double)params->ny;
    *column = col;
    return EHD_OK;
}

namespace {
// every parameter of a column context equal to the context's, but for the
// plane's extent (nx, ny, lx, ly)
bool column_matches(const ehd_params &a, const ehd_params &b) {
    const double x[] = {a.lz, a.dx, a.dy, a.dz, a.dt, a.cfl, a.rho0, a.charge0, a.voltage,
                        a.eps, a.diffu, a.nu, a.K, a.uw, a.exf, a.lambda_f, a.lambda_g};
    const double y[] = {b.lz, b.dx, b.dy, b.dz, b.dt, b.cfl, b.rho0, b.charge0, b.voltage,
                        b.eps, b.diffu, b.nu, b.K, b.uw, b.exf, b.lambda_f, b.lambda_g};
    if (a.nz != b.nz) return false;
    for (size_t i = 0; i < sizeof(x) / sizeof(x[0]); ++i)
        if (x[i] != y[i]) return false;
    return true;
}

double read_real(const std::vector<unsigned char> &b, size_t i, size_t size) {
    if (size == 8) {
        double v;
        std::memcpy(&v, b.data() + 8 * i, 8);
        return v;
    }
    float v;
    std::memcpy(&v, b.data() + 4 * i, 4);
    return v;
}

void write_real(std::vector<unsigned char> &b, size_t i, size_t size, double v) {
    if (size == 8) {
        std::memcpy(b.data() + 8 * i, &v, 8);
    } else {
        const float f = (float)v;
        std::memcpy(b.data() + 4 * i, &f, 4);
    }
}
}  // namespace

int ehd_set_state_from_column(ehd_ctx *c, ehd_ctx *col, uint64_t seed, double amp) {
    if (!c || !col) return fail(EHD_ERR_INVALID, "NULL argument");
    if (!std::isfinite(amp)) return fail(EHD_ERR_INVALID, "amp not finite");
    if (col->p.nx != 1 || col->p.ny != 1)
        return fail(EHD_ERR_INVALID, "column: nx and ny must be 1");
    if (!column_matches(c->p, col->p))
        return fail(EHD_ERR_INVALID, "column: parameters differ from the context's");
    if (!col->have_state || col->pops_local || col->e_arrays)
        return fail(EHD_ERR_STATE, "column: needs a state stepped at least once since its upload");
    if (col->fsize < 4 || col->gsize < 4)
        return fail(EHD_ERR_INVALID, "column: FP64 or FP32 populations needed");
    const int nz = c->p.nz;
    const size_t nzs = (size_t)nz;
    // the column's fields, population values and tables, on the host
    std::vector<double> prof(9 * nzs);
    int r = ehd_get_fields(col, prof.data(), prof.data() + nzs, prof.data() + 2 * nzs,
                           prof.data() + 3 * nzs, prof.data() + 4 * nzs, prof.data() + 5 * nzs,
                           prof.data() + 6 * nzs, prof.data() + 7 * nzs, prof.data() + 8 * nzs);
    if (r != EHD_OK) return r;
    std::vector<unsigned char> fb(Q * nzs * col->fsize), hb(Q * nzs * col->gsize);
    std::vector<unsigned char> kt[2] = {std::vector<unsigned char>(10 * nzs * col->rsize),
                                        std::vector<unsigned char>(10 * nzs * col->rsize)};
    std::vector<double> wref[2] = {std::vector<double>(2 * nzs), std::vector<double>(2 * nzs)};
    std::vector<double> mean[2] = {std::vector<double>(2 * nzs), std::vector<double>(2 * nzs)};
    std::vector<double> phi00(nzs), ez00(nzs);
    {
        DeviceGuard dg(col->device);
        EHD_CK(cudaMemcpy(fb.data(), col->f[col->cur], fb.size(), cudaMemcpyDeviceToHost));
        EHD_CK(cudaMemcpy(hb.data(), col->h[col->cur], hb.size(), cudaMemcpyDeviceToHost));
        for (int k = 0; k < 2; ++k) {
            EHD_CK(cudaMemcpy(kt[k].data(), col->ktab[k], kt[k].size(), cudaMemcpyDeviceToHost));
            EHD_CK(cudaMemcpy(wref[k].data(), col->wref[k], 16 * nzs, cudaMemcpyDeviceToHost));
            EHD_CK(cudaMemcpy(mean[k].data(), col->mean[k], 16 * nzs, cudaMemcpyDeviceToHost));
        }
        EHD_CK(cudaMemcpy(phi00.data(), col->phi00, 8 * nzs, cudaMemcpyDeviceToHost));
        EHD_CK(cudaMemcpy(ez00.data(), col->ez00, 8 * nzs, cudaMemcpyDeviceToHost));
    }
    // population values: stored deviation + w_d times the plane's reference
    const std::vector<double> &wc = wref[col->cur];
    std::vector<double> colv(2 * Q * nzs);
    for (int d = 0; d < Q; ++d)
        for (size_t z = 0; z < nzs; ++z) {
            colv[d * nzs + z] = read_real(fb, d * nzs + z, col->fsize) + w_of(d) * wc[2 * z];
            colv[(Q + d) * nzs + z] = read_real(hb, d * nzs + z, col->gsize) + w_of(d) * wc[2 * z + 1];
        }
    // the step kernel's tables in this context's compute type
    for (int k = 0; k < 2; ++k) {
        std::vector<unsigned char> conv(10 * nzs * c->rsize);
        for (size_t j = 0; j < 10 * nzs; ++j) write_real(conv, j, c->rsize, read_real(kt[k], j, col->rsize));
        kt[k].swap(conv);
    }
    DeviceGuard dg(c->device);
    EHD_CK(cudaStreamSynchronize(c->stream));
    double *colv_dev = nullptr;
    EHD_CK(cudaMalloc((void **)&colv_dev, sizeof(double) * colv.size()));
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        if ((e = cudaMemcpy(c->wref[k], wref[k].data(), 16 * nzs, cudaMemcpyHostToDevice)) == cudaSuccess &&
            (e = cudaMemcpy(c->mean[k], mean[k].data(), 16 * nzs, cudaMemcpyHostToDevice)) == cudaSuccess)
            e = cudaMemcpy(c->ktab[k], kt[k].data(), kt[k].size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(colv_dev, colv.data(), sizeof(double) * colv.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->phi00, phi00.data(), 8 * nzs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->ez00, ez00.data(), 8 * nzs, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(c->prof_dev, prof.data(), sizeof(double) * prof.size(), cudaMemcpyHostToDevice);
    c->cur = col->cur;
    if (e == cudaSuccess) e = launch_seeded_state(c->out_dev, c->prof_dev, (unsigned long long)seed, amp, c->sc, c->stream);
    if (e == cudaSuccess) {
        void *f = c->f[c->cur], *h = c->h[c->cur];
        const double *ref = c->wref[c->cur];
        switch (c->prec) {
            case EHD_PREC_FP64: e = launch_column_state<double, double>(f, h, c->out_dev, c->prof_dev, colv_dev, ref, c->phip, c->phi00, c->sc, c->stream); break;
            case EHD_PREC_FP32: e = launch_column_state<float, float>(f, h, c->out_dev, c->prof_dev, colv_dev, ref, c->phip, c->phi00, c->sc, c->stream); break;
            case EHD_PREC_FP16: e = launch_column_state<__half, float>(f, h, c->out_dev, c->prof_dev, colv_dev, ref, c->phip, c->phi00, c->sc, c->stream); break;
            case EHD_PREC_MIXED: e = launch_column_state<Mix16, float>(f, h, c->out_dev, c->prof_dev, colv_dev, ref, c->phip, c->phi00, c->sc, c->stream); break;
            default: e = launch_column_state<__nv_bfloat16, float>(f, h, c->out_dev, c->prof_dev, colv_dev, ref, c->phip, c->phi00, c->sc, c->stream); break;
        }
    }
    if (e == cudaSuccess)
        e = c->prec == EHD_PREC_FP64
                ? launch_fields_to_compute<double>(c->out_dev, c->rho, c->u, c->v, c->w, c->q, c->sc.n, c->stream)
                : launch_fields_to_compute<float>(c->out_dev, c->rho, c->u, c->v, c->w, c->q, c->sc.n, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(colv_dev);
    if (e != cudaSuccess) {
        c->have_state = false;
        return fail(EHD_ERR_CUDA, "state from column: %s", cudaGetErrorString(e));
    }
    c->have_state = true;
    c->pops_local = false;
    c->e_arrays = false;
    c->out_valid = false;
    c->step = 0;
    c->t = 0.0;
    return EHD_OK;
}

int ehd_hydrostatic_profile(const ehd_params *params, const ehd_config *config, int nsteps,
                            double *profile, double *i0) {
    if (!params || !profile) return fail(EHD_ERR_INVALID, "NULL argument");
    if (nsteps < 0) return fail(EHD_ERR_INVALID, "nsteps < 0");
    ehd_params q = *params;
    q.nx = 1;
    q.ny = 1;
    q.lx = params->dx;
    q.ly = params->dy;
    ehd_ctx *col = nullptr;
    int r = ehd_create(&q, config, &col);
    if (r != EHD_OK) return r;
    const int nz = q.nz;
    std::vector<double> f(9 * (size_t)nz);
    double *fp[9];
    for (int k = 0; k < 9; ++k) fp[k] = f.data() + (size_t)k * nz;
    // I0: the mean of the column's currents after nsteps and nsteps + 1 steps
    // (the injection boundary makes the current alternate with a period of
    // two steps; the profile is the state after nsteps)
    ehd_diag d{}, d1{};
    if ((r = ehd_initialize(col)) == EHD_OK && (r = ehd_step(col, nsteps)) == EHD_OK &&
        (r = ehd_get_fields(col, fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7],
                            fp[8])) == EHD_OK &&
        (r = ehd_diagnostics(col, &d)) == EHD_OK && (r = ehd_step(col, 1)) == EHD_OK)
        r = ehd_diagnostics(col, &d1);
    ehd_destroy(col);
    if (r != EHD_OK) return r;
    std::memcpy(profile, f.data(), sizeof(double) * 9 * nz);
    if (i0) *i0 = 0.5 * (d.current + d1.current) * (double)params->nx * (double)params->ny;
    return EHD_OK;
}

int ehd_run_to_saturation(ehd_ctx *c, int sample_every, double tol, int hold, int64_t max_steps,
                          double *nu_e, int64_t *steps, int *saturated) {
    if (!c || sample_every < 1 || hold < 1 || !(tol > 0) || max_steps < 0)
        return fail(EHD_ERR_INVALID, "bad arguments");
    if (c->i0 == 0.0) return fail(EHD_ERR_STATE, "reference current I0 not set");
    double prev = 0.0, nu = 0.0;
    int held = 0, ok = 0;
    int64_t done = 0;
    bool first = true;
    while (done < max_steps) {
        // a sample is the mean of the currents after the last two steps of
        // its interval: the injection boundary makes the current alternate
        // with a period of two steps
        const int n = (int)std::min<int64_t>(sample_every, max_steps - done);
        ehd_diag da{}, db{};
        int r = n >= 2 ? ehd_step(c, n - 1) : EHD_OK;
        if (r == EHD_OK && n >= 2) r = ehd_diagnostics(c, &da);
        if (r == EHD_OK) r = ehd_step(c, 1);
        if (r == EHD_OK) r = ehd_diagnostics(c, &db);
        if (r != EHD_OK) return r;
        done += n;
        if (da.nonfinite || db.nonfinite)
            return fail(EHD_ERR_NUMERIC, "non-finite field after %lld steps", (long long)done);
        nu = n >= 2 ? 0.5 * (da.current + db.current) / c->i0 : db.nu_e;
        if (!first && std::fabs(nu - prev) <= tol * std::fabs(nu)) {
            if (++held >= hold) {
                ok = 1;
                break;
            }
        } else {
            held = 0;
        }
        prev = nu;
        first = false;
    }
    if (nu_e) *nu_e = nu;
    if (steps) *steps = done;
    if (saturated) *saturated = ok;
    return EHD_OK;
}

namespace {
const char kCkptMagic[8] = {'E', 'H', 'D', 'C', 'K', 'P', 'T', '1'};

struct CkptHeader {
    char magic[8];
    uint32_t version, precision;
    ehd_params params;
    int64_t step;
    double t, i0;
    int32_t cur, pops_local, e_arrays, pad_;
};

// device buffers of the state, in file order
struct Blob {
    void *ptr;
    size_t bytes;
};
std::vector<Blob> state_blobs(ehd_ctx *c) {
    const size_t n = (size_t)c->sc.n, nz = (size_t)c->p.nz;
    std::vector<Blob> b = {
        {c->f[c->cur], (size_t)Q * n * c->fsize}, {c->h[c->cur], (size_t)Q * n * c->gsize},
        {c->phip, n * c->rsize}, {c->q, n * c->rsize}, {c->rho, n * c->rsize},
        {c->u, n * c->rsize}, {c->v, n * c->rsize}, {c->w, n * c->rsize},
        {c->phi00, nz * 8}, {c->ez00, nz * 8},
        {c->wref[0], 2 * nz * 8}, {c->wref[1], 2 * nz * 8},
        {c->mean[0], 2 * nz * 8}, {c->mean[1], 2 * nz * 8},
        {c->ktab[0], 10 * nz * c->rsize}, {c->ktab[1], 10 * nz * c->rsize}};
    if (c->e_arrays)  // the uploaded phi and E are still in use
        for (int k = 5; k < 9; ++k) b.push_back({c->out[k], n * 8});
    return b;
}
}  // namespace

int ehd_checkpoint(ehd_ctx *c, const char *path) {
    if (!c || !path) return fail(EHD_ERR_INVALID, "NULL argument");
    if (!c->have_state) return fail(EHD_ERR_STATE, "no state to checkpoint");
    DeviceGuard dg(c->device);
    EHD_CK(cudaStreamSynchronize(c->stream));
    FILE *fp = std::fopen(path, "wb");
    if (!fp) return fail(EHD_ERR_IO, "cannot open %s for writing", path);
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, 8);
    h.version = 1;
    h.precision = (uint32_t)c->prec;
    h.params = c->p;
    h.step = c->step;
    h.t = c->t;
    h.i0 = c->i0;
    h.cur = c->cur;
    h.pops_local = c->pops_local;
    h.e_arrays = c->e_arrays;
    bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1;
    std::vector<unsigned char> buf;
    for (const Blob &b : state_blobs(c)) {
        if (!ok) break;
        buf.resize(b.bytes);
        if (cudaMemcpy(buf.data(), b.ptr, b.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
            std::fclose(fp);
            return fail(EHD_ERR_CUDA, "checkpoint: device read failed");
        }
        const uint64_t sz = b.bytes;
        ok = std::fwrite(&sz, sizeof(sz), 1, fp) == 1 && std::fwrite(buf.data(), 1, b.bytes, fp) == b.bytes;
    }
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(EHD_ERR_IO, "checkpoint: write to %s failed", path);
    return EHD_OK;
}

int ehd_restore(ehd_ctx *c, const char *path) {
    if (!c || !path) return fail(EHD_ERR_INVALID, "NULL argument");
    DeviceGuard dg(c->device);
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return fail(EHD_ERR_IO, "cannot open %s", path);
    CkptHeader h{};
    if (std::fread(&h, sizeof(h), 1, fp) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 ||
        h.version != 1) {
        std::fclose(fp);
        return fail(EHD_ERR_IO, "%s is not an ehd checkpoint", path);
    }
    if ((int)h.precision != c->prec || std::memcmp(&h.params, &c->p, sizeof(ehd_params)) != 0) {
        std::fclose(fp);
        return fail(EHD_ERR_INVALID, "checkpoint parameters or precision differ from the context's");
    }
    EHD_CK(cudaStreamSynchronize(c->stream));
    c->cur = h.cur & 1;
    c->e_arrays = h.e_arrays != 0;
    std::vector<unsigned char> buf;
    for (const Blob &b : state_blobs(c)) {
        uint64_t sz = 0;
        buf.resize(b.bytes);
        if (std::fread(&sz, sizeof(sz), 1, fp) != 1 || sz != b.bytes ||
            std::fread(buf.data(), 1, b.bytes, fp) != b.bytes) {
            std::fclose(fp);
            c->have_state = false;
            return fail(EHD_ERR_IO, "checkpoint %s is truncated or corrupt", path);
        }
        if (cudaMemcpy(b.ptr, buf.data(), b.bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            std::fclose(fp);
            c->have_state = false;
            return fail(EHD_ERR_CUDA, "restore: device write failed");
        }
    }
    std::fclose(fp);
    c->pops_local = h.pops_local != 0;
    c->step = h.step;
    c->t = h.t;
    c->i0 = h.i0;
    c->have_state = true;
    c->out_valid = false;
    return EHD_OK;
}

}  // extern "C"
