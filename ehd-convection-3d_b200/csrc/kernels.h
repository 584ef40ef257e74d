// kernels.h -- launchers of the step kernels, called by the C ABI layer.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace ehd {

struct LbmArgs {
    const void *fa, *ha;  // populations read this step (pulled)
    void *fb, *hb;        // populations written this step
    const void *phip;     // phi' (compute type), zero on both electrodes
    const double *ez00;   // per-plane Ez of the mean potential phi00
    const double *exa, *eya, *eza;  // explicit E (first step after set_fields)
    void *q, *rho, *u, *v, *w;      // macroscopic outputs (compute type)
    const void *zref;               // step kernel's reference table (compute type, 10 per plane)
    float2 *psum;                   // per-warp sums of rho and q
    int *err;                       // device flag: a bounded wait gave up
    int rows_grid;                  // > 0: steady-state steps run the bulk-copy
                                    // row kernel on this many CTAs
    int node_bx;                    // per-node kernel block: node_bx x (128 / node_bx)
};

template <typename T, typename R>
cudaError_t launch_lbm_step(const LbmArgs &a, const StepConst &c, int local_pops, int e_arrays,
                            bool macros, cudaStream_t s);

// ref: per-plane {rho_w, q_w} in FP64 (what the stored deviations are relative to)
template <typename T>
cudaError_t launch_init_equilibrium(void *f, void *h, const double *const fields[9],
                                    const double *ref, const StepConst &c, cudaStream_t s);

template <typename R>
cudaError_t launch_materialize(const void *rho, const void *u, const void *v, const void *w,
                               const void *q, const void *phip, const double *phi00,
                               double *const out[9], int macros, const StepConst &c,
                               cudaStream_t s);

// out_dev: device array of the 9 FP64 field pointers
cudaError_t launch_reference_init(double *const *out_dev, const StepConst &c, double voltage,
                                  double lz, double dz, cudaStream_t s);
template <typename R>
cudaError_t launch_fields_to_compute(double *const *out_dev, void *rho, void *u, void *v,
                                     void *w, void *q, long long n, cudaStream_t s);

// Reference tables (see lbm.cu): plane means m (FP64, {rho, q} per plane)
// from the FP64 fields or from the step kernel's per-block sums, and the
// step kernel's table (compute type, 10 per plane).
cudaError_t launch_fields_plane_mean(const double *rho, const double *q, double *m,
                                     const StepConst &c, cudaStream_t s);
template <typename R>
cudaError_t launch_build_tables(const double *msrc, double *wdst, const double *wread,
                                void *ktab, const StepConst &c, cudaStream_t s);
// psum_reduce and build_tables in one launch (the tables read msrc, the
// previous means, so the two parts are independent)
template <typename R>
cudaError_t launch_reduce_tables(const float2 *psum, double *m, int nblk, const double *msrc,
                                 double *wdst, const double *wread, void *ktab,
                                 const StepConst &c, cudaStream_t s);
// ---- launches over a group of instances with the same grid ----------------
// (batch steps, csrc/batch.cu): one launch per kernel covers every instance.
template <typename T, typename R>
size_t lbm_group_desc_bytes(int n);
// the n instances' arguments of one per-node step (default block shape) into
// host memory of lbm_group_desc_bytes(n) bytes, to be copied to the device
template <typename T, typename R>
void build_lbm_group_desc(const LbmArgs *la, const StepConst *c, int n, void *host);
// bx: the per-node block width (16, 32, 64 or 128) of every instance of the group
template <typename T, typename R>
cudaError_t launch_lbm_group(const void *desc_dev, int n, int nx, int ny, int nz, int bx,
                             bool macros, cudaStream_t s);
// the same step on the bulk-copy row kernel (lbm_rows_usable grids), per_inst
// CTAs per instance
template <typename T, typename R>
cudaError_t launch_lbm_rows_group(const void *desc_dev, int n, int nx, int ny, int per_inst,
                                  bool macros, cudaStream_t s);
// one instance's arguments of launch_reduce_tables
struct ReduceDesc {
    const float2 *psum;
    double *m;
    const double *msrc;
    double *wdst;
    const double *wread;
    void *ktab;
    long long nxy;
    int nblk, nz;
};
template <typename R>
cudaError_t launch_reduce_tables_group(const ReduceDesc *desc_dev, int n, int nz, cudaStream_t s);

// psum slots per plane of the per-node kernel with blocks of bx x (128 / bx)
int lbm_blocks_per_plane(int nx, int ny, int bx);
// the per-node kernel's default block width for a grid nx wide
int lbm_default_block_x(int nx);
// whether the bulk-copy row kernel serves this grid and storage type
bool lbm_rows_usable(int nx, size_t fsize, size_t gsize);
// sets the row kernel's shared-memory attribute (before any stream capture)
// and returns its persistent grid size in *grid, 0 when it does not apply
template <typename T, typename R>
cudaError_t prepare_lbm_rows(int nx, int ny, int nz, int *grid);
// psum slots per plane: per-node kernel / row kernel
int lbm_rows_slots_per_plane(int nx, int ny);

// The nine FP64 fields from a per-plane profile [k][z] plus a seeded velocity
// perturbation (ehd_set_state_seeded).
cudaError_t launch_seeded_state(double *const *out_dev, const double *prof_dev,
                                unsigned long long seed, double amp, const StepConst &c,
                                cudaStream_t s);
// Populations of a state broadcast from a 1 x 1 x NZ column's: colv holds the
// column's population values [(s Q + d) NZ + z] (s = 0: f, 1: g), prof its
// nine fields [k][z]; out_dev the seeded fields (velocity = the perturbation,
// replaced by column velocity + perturbation); ref the per-plane references
// the populations are stored against; phip (compute type) receives the
// column's phi - phi00 (ehd_set_state_from_column).
template <typename T, typename R>
cudaError_t launch_column_state(void *f, void *h, double *const *out_dev, const double *prof_dev,
                                const double *colv_dev, const double *ref, void *phip,
                                const double *phi00, const StepConst &c, cudaStream_t s);

// ---- Poisson solve ---------------------------------------------------------

constexpr int kMaxRadix = 24;
struct FftPlan {
    int n;
    int nrad;
    int rad[kMaxRadix];
};

// Per-instance buffers of one Poisson solve in a launch over a group of
// instances with the same grid (blockIdx.z selects the instance); the tables
// (twiddles, eigenvalues, pivots) are the same for the whole group.
struct PoissonPtrs {
    void *spec;
    double *rowsum, *planesum, *phi00, *ez00;
    const void *q;
    const double *qmean;
    void *phip;
    double2 *dpw;
};

// Buffers and sizes of the FFT / tridiagonal Poisson solve.  spec holds the
// x,y spectrum of the planes z = 1..NZ-2 in the compute type, layout
// [z-1][ky][kx] with kx pitch `pitch`; the z solve works on it in place.
struct PoissonArgs {
    int nx, ny, nz, nxh, pitch;
    int split;           // 1: the split-y three-kernel path where it applies
    int thomas;          // 1: the Thomas z solve where the sine transform is run-time
    int rows_per_block;  // x-row FFT batch per block (run-time radix path)
    int cols_per_block;  // y-column FFT batch per block (run-time radix path)
    FftPlan px, py;
    const void *twx, *twy;   // exp(-2 pi i k/N) tables in the compute type
    FftPlan pz;              // run-time plan of length L = 2 (nz - 1) (sine-transform
                             // z solve when L is not a compile-time FFT size)
    int ztb;                 // modes per block of that solve
    const void *twz;         // sine-transform z solve, L = 2 (nz - 1), compute type:
                             // exp(-2 pi i k/L) (L complex), then 4 sin^2(pi k/L)
                             // (L/2 + 1 real); nullptr: Thomas solve
    double lx, ly;           // domain lengths (wavenumbers 2 pi k / l)
    const double *cpt;       // Thomas pivots [z-1][ky*nxh + kx], FP64
    const void *cps;         // split-y path: two-sided Thomas pivots [kx][j][r][k'] (ky = S k' + j,
                             // NY = 64 S; r < (NZ - 1)/2: c_r, then the middle plane's mu)
                             // in the compute type; nullptr: no split path
    double2 *dpw;            // FP64 scratch of the forward sweep, same layout
    void *spec;              // complex compute type
    double *rowsum;          // [z-1][y] FP64 sums of the source
    double *planesum;        // [z] FP64 sums of the source
    double *phi00, *ez00;    // [z] mean potential and its Ez
    const void *q;           // charge (compute type)
    const double *qmean;     // plane means {rho, q} of the current state, FP64: q_m = [2z+1]
    void *phip;              // output phi' (compute type)
    double eps, voltage, dz;
    const PoissonPtrs *grp = nullptr;  // device array: a launch over ngrp instances
    int ngrp = 1;
};

template <typename R>
cudaError_t launch_poisson(const PoissonArgs &a, cudaStream_t s);
// sets the shared-memory attributes of the kernels a's grid will use (call
// before any stream capture)
template <typename R>
cudaError_t prepare_poisson(const PoissonArgs &a);

bool poisson_fast_size(int n);
// whether the split-y path serves a grid in the compute type of rsize bytes
// (the context then builds its pivot table, PoissonArgs::cps)
bool poisson_split_grid(int nx, int ny, int nz, size_t rsize);
// shared memory of the run-time-radix sine-transform z solve with tb modes
// per block (compute type of rsize bytes)
size_t zdst_rt_smem(int L, int tb, size_t rsize);

// ---- diagnostics ---------------------------------------------------------

struct DiagArgs {
    int nx, ny, nz;
    const void *rho, *u, *v, *w, *q;  // type R (R = double for the FP64 field arrays)
    const void *phip;                 // phi' (type R) when ez == nullptr
    const double *ez00;               // mean-field Ez per plane when ez == nullptr
    const double *ez;                 // explicit FP64 Ez field, or nullptr
    double inv2dz;
    double *partial;                  // scratch: nblocks x 5 doubles
    double *result;                   // 5 doubles
    int nblocks;
};
template <typename R>
cudaError_t launch_diag(const DiagArgs &a, cudaStream_t s);
// the current alone into result[0] (partial: at least a.nblocks doubles)
template <typename R>
cudaError_t launch_current(const DiagArgs &a, cudaStream_t s);

// sets the calling thread's ehd_last_error message; returns code
int set_error(int code, const char *msg);
}  // namespace ehd

struct ehd_ctx;
struct ehd_params;
struct ehd_tuning;
namespace ehd {
// a context's parameters and its physical time (for the text writers)
const ::ehd_params *ctx_params(const ::ehd_ctx *c);
double *ctx_time(::ehd_ctx *c);

// For the batch (csrc/batch.cu): a context's stream, device and precision;
// whether its next step can be captured (not the first after an upload);
// its buffer parity; the launches of one steady step on its stream with the
// buffer parity left unchanged (as a graph capture needs); and the
// bookkeeping once that step has run.
cudaStream_t ctx_stream(const ::ehd_ctx *c);
int ctx_device(const ::ehd_ctx *c);
int ctx_precision(const ::ehd_ctx *c);
bool ctx_steady(const ::ehd_ctx *c);
int ctx_parity(const ::ehd_ctx *c);
int ctx_launch_step(::ehd_ctx *c, bool macros);
void ctx_commit_step(::ehd_ctx *c);
// changes whenever the context's launches change (ehd_set_tuning), so that
// captured graphs holding them are rebuilt
unsigned ctx_generation(const ::ehd_ctx *c);
// the context's launch shapes
void ctx_tuning(const ::ehd_ctx *c, ::ehd_tuning *t);
// the arguments of one steady step at the context's present buffer parity,
// with the LBM half on the per-node kernel (what a launch over a group of
// instances runs); nothing is launched
int ctx_step_args(::ehd_ctx *c, bool macros, LbmArgs *la, StepConst *sc, ReduceDesc *rd,
                  PoissonArgs *pa);
double ctx_reference_current(const ::ehd_ctx *c);

}  // namespace ehd
