/*
 * ehd.h -- C ABI of the B200 (sm_100a) EHD convection time step.
 *
 * Drop-in for the reference solver's step (gyf135/EHD-convection-3D).  The
 * reference has no plugin or FFI layer: its step is a sequence of free host
 * functions called from main() (main.cu:184-206) over global device pointers
 * and compile-time constants (LBM.h:30-113).  Each entry point below names the
 * reference interface it replaces.  Conventions:
 *
 *   - every function returns 0 (EHD_OK) or a negative ehd_status; nothing
 *     calls exit() (the reference exits on any error, LBM.cu:39-57,
 *     LBM.h:140-161).  ehd_last_error() gives the message of the last failure
 *     on the calling thread;
 *   - all field arguments are HOST pointers to NX*NY*NZ doubles in the
 *     reference layout, index x + NX*(y + NY*z) (LBM.cu:21-24), unless the
 *     name ends in _device;
 *   - one context per simulation instance; a context is not thread-safe.
 *     All device work of a context runs on its stream (ehd_config.stream, or
 *     a stream the context creates).
 */
#ifndef EHD_H
#define EHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EHD_ABI_VERSION 1

typedef enum ehd_status {
    EHD_OK = 0,
    EHD_ERR_INVALID = -1,   /* bad argument or parameter                  */
    EHD_ERR_CUDA = -2,      /* a CUDA runtime call failed                 */
    EHD_ERR_NOMEM = -3,     /* device or host allocation failed           */
    EHD_ERR_STATE = -4,     /* call out of order (e.g. step before set)   */
    EHD_ERR_NUMERIC = -5,   /* non-finite value detected                  */
    EHD_ERR_IO = -6         /* file read/write failed                     */
} ehd_status;

/* Physical, geometric and scheme parameters: the reference's compile-time
 * constants and __device__ scalars (LBM.h:30-80, main.cu:27-36) as a runtime
 * struct.  nz counts nodes; the electrodes are the planes z=0 and z=nz-1. */
typedef struct ehd_params {
    int32_t nx, ny, nz;      /* NX, NY, NZ (LBM.h:34-36)                       */
    int32_t pad_;            /* must be 0                                      */
    double lx, ly, lz;       /* Lx, Ly, Lz (LBM.h:40-42)                       */
    double dx, dy, dz;       /* dx, dy, dz (LBM.h:43-45)                       */
    double dt, cfl;          /* dt, CFL (LBM.h:50-52); cs^2 = 1/(3 CFL^2)      */
    double rho0, charge0;    /* rho0, charge0 (LBM.h:54-55)                    */
    double voltage, eps;     /* voltage, eps (LBM.h:56-57)                     */
    double diffu, nu, K;     /* diffu, nu, K (LBM.h:58-62)                     */
    double uw, exf;          /* uw, exf (LBM.h:47-50)                          */
    double lambda_f;         /* TRT magic parameter of f, V (LBM.h:79)        */
    double lambda_g;         /* TRT magic parameter of g, VC (LBM.h:80)       */
} ehd_params;

/* Arithmetic of the step.  The reference computes and stores in FP64. */
typedef enum ehd_precision {
    EHD_PREC_FP64 = 0,       /* FP64 compute, FP64 populations                 */
    EHD_PREC_FP32 = 1,       /* FP32 compute, FP32 populations                 */
    EHD_PREC_FP16 = 2,       /* FP32 compute, FP16 population deviations       */
    EHD_PREC_BF16 = 3,       /* FP32 compute, BF16 population deviations       */
    EHD_PREC_MIXED = 4       /* FP32 compute, FP16 deviations of the flow
                                populations f, FP32 deviations of the charge
                                populations g (no reference counterpart)     */
} ehd_precision;

typedef struct ehd_config {
    int32_t precision;       /* ehd_precision                                  */
    int32_t device;          /* CUDA device ordinal                            */
    void *stream;            /* cudaStream_t to run on, or NULL: own stream    */
    uint32_t flags;          /* EHD_FLAG_*                                     */
    uint32_t reserved[7];    /* must be 0                                      */
} ehd_config;

#define EHD_FLAG_NO_GRAPH 0x1u /* launch kernels one by one, no CUDA graphs   */
#define EHD_FLAG_NODE_KERNEL 0x2u /* every step on the one-thread-per-node
                                     kernel (no bulk-copy row kernel)       */

typedef struct ehd_ctx ehd_ctx;

/* Launch shapes of a context's kernels.  No reference counterpart: the
 * reference fixes its launch shape at compile time (nThreads, LBM.h).  A
 * shape changes only the order of the FP32 partial plane sums behind the
 * per-plane reference states, i.e. results at round-off level. */
typedef struct ehd_tuning {
    int32_t lbm_kernel;      /* 0: steady steps on the row kernel where it
                                applies, else the per-node kernel; 1: per-node */
    int32_t node_block_x;    /* per-node kernel block: x extent 16, 32, 64 or
                                128, y extent 128 / node_block_x              */
    int32_t fft_rows;        /* run-time-radix x FFT: rows per block          */
    int32_t fft_cols;        /* run-time-radix y FFT: columns per block       */
    int32_t poisson_path;    /* 0: the split-y three-kernel Poisson solve
                                where it applies (NX a power of two 64..512,
                                NY = 64, 128, 256 or 512, 2 (NZ-1) likewise),
                                else the five-kernel one; 1: five-kernel     */
    int32_t z_solve;         /* where 2 (NZ-1) is not a compile-time FFT
                                size (48, 64, 80, 96, 128, 256, 512): 0 the
                                sine transform with run-time FFT passes, 1 the
                                FP64 Thomas sweep                             */
    int32_t reserved[2];     /* must be 0                                     */
} ehd_tuning;

/* Scalar diagnostics, reduced on the device in FP64. */
typedef struct ehd_diag {
    double current;          /* I = K dy^2 sum_xy q(NZ-1) Ez(NZ-1), LBM.cu:1647 */
    double nu_e;             /* I / I0 (I0 from ehd_set_reference_current)     */
    double kinetic_energy;   /* 0.5 sum rho |u|^2 dx dy dz                      */
    double total_charge;     /* sum q dx dy dz                                  */
    double umax;             /* max uz over the domain, LBM.cu:1673-1713        */
    double time;             /* physical time t (main.cu:208)                   */
    int64_t step;            /* steps taken since ehd_set_fields               */
    int32_t nonfinite;       /* 1 if any field holds a NaN or Inf              */
    int32_t pad_;
} ehd_diag;

/* --- lifetime ------------------------------------------------------------ */

/* Allocates every device buffer of one instance and prepares the Poisson
 * solver.  Replaces main.cu:79-143 (cudaMalloc of the fields and populations,
 * cufftPlan3d, the kx/ky/kz tables). */
int ehd_create(const ehd_params *params, const ehd_config *config, ehd_ctx **out);

/* Frees everything.  Replaces main.cu:283-304. */
int ehd_destroy(ehd_ctx *ctx);

/* --- state ----------------------------------------------------------------- */

/* Uploads the nine macroscopic fields and builds the equilibrium populations
 * from them.  Replaces read_data (LBM.cu:1597-1643) + init_equilibrium
 * (LBM.cu:98-276).  The first step after this call uses the given E; later
 * steps use E = -grad(phi) from the Poisson solve, as the reference does. */
int ehd_set_fields(ehd_ctx *ctx, const double *rho, const double *u, const double *v,
                   const double *w, const double *q, const double *phi, const double *ex,
                   const double *ey, const double *ez);

/* The reference's own start (initialization, LBM.cu:69-96, then
 * init_equilibrium): rho = rho0, q = 0, phi linear, u = E = 0. */
int ehd_initialize(ehd_ctx *ctx);

/* Downloads the nine fields, raw (no wall extrapolation), in the reference
 * layout.  Any pointer may be NULL to skip that field.  Replaces the D2H
 * copies of save_data_* (LBM.cu:1427-1566). */
int ehd_get_fields(ehd_ctx *ctx, double *rho, double *u, double *v, double *w, double *q,
                   double *phi, double *ex, double *ey, double *ez);

/* --- the time step ------------------------------------------------------ */

/* Advances nsteps time steps: per step the fused LBM stream-collide with its
 * wall and injection rules, then the Poisson solve and E = -grad(phi).
 * Replaces the loop body main.cu:184-208: stream_collide_save (LBM.cu:278),
 * extension (poisson.cu:78), cufftExecZ2Z x2 (main.cu:194,200), derivative
 * (poisson.cu:123), extract (poisson.cu:145), efield (poisson.cu:33).
 * Asynchronous on the context's stream. */
int ehd_step(ehd_ctx *ctx, int nsteps);

/* The LBM half of one step only (stream_collide_save, LBM.cu:278-293). */
int ehd_stream_collide_save(ehd_ctx *ctx);

/* The Poisson half of one step only, from the current q: extension,
 * forward FFT, derivative, inverse FFT, extract and efield
 * (poisson.cu:33-167, main.cu:190-206). */
int ehd_poisson(ehd_ctx *ctx);

/* Blocks until the context's queued work is done. */
int ehd_synchronize(ehd_ctx *ctx);

/* --- diagnostics ---------------------------------------------------------- */

/* Collector current of the present fields.  Replaces current()
 * (LBM.cu:1647-1671) with its host loop over a full-field D2H copy. */
int ehd_current(ehd_ctx *ctx, double *current);

/* Sets I0, the hydrostatic current that normalises nu_e. */
int ehd_set_reference_current(ehd_ctx *ctx, double i0);

/* All scalar diagnostics, reduced on the device (blocks until done). */
int ehd_diagnostics(ehd_ctx *ctx, ehd_diag *out);

/* --- initial state, saturation, restart ----------------------------------- */

/* The hydrostatic state: the u = 0 steady state of the same discrete step,
 * found by running it on a 1 x 1 x NZ column of the grid's geometry from the
 * reference's initialization (LBM.cu:69-96) for nsteps steps (even; the
 * injector alternates with period 2).  profile receives 9*NZ doubles, field
 * k at profile[k*NZ + z] in the order rho, u, v, w, q, phi, ex, ey, ez;
 * *i0 the mean of the column's currents after nsteps and nsteps + 1 steps
 * on the full NX x NY plane (the Nu_e normaliser; the current alternates
 * between two values, 1.5 % apart at 64 x 64 x 33).  Not in the reference,
 * which starts from q = 0. */
int ehd_hydrostatic_profile(const ehd_params *params, const ehd_config *config, int nsteps,
                            double *profile, double *i0);

/* Sets the state to a per-plane profile (layout of ehd_hydrostatic_profile)
 * broadcast over x, y, at rest, plus a seeded velocity perturbation of
 * amplitude amp on the interior planes: component c of node i is
 * amp (2 r - 1) with r from splitmix64 of the counter seed * 2^32 + 3 i + c.
 * Builds the equilibrium populations like ehd_set_fields.  Not in the
 * reference (its perturbation, LBM.cu:389-415, is a disabled sinusoid). */
int ehd_set_state_seeded(ehd_ctx *ctx, const double *profile, uint64_t seed, double amp);

/* The hydrostatic state as a live 1 x 1 x NZ context: the column of
 * ehd_hydrostatic_profile, left after nsteps + 1 steps (*column, freed with
 * ehd_destroy), with *i0 as there.  Not in the reference. */
int ehd_hydrostatic_column(const ehd_params *params, const ehd_config *config, int nsteps,
                           ehd_ctx **column, double *i0);

/* Sets the state to a 1 x 1 x NZ column's state broadcast over x, y: its
 * populations (not equilibria rebuilt from its fields), reference tables,
 * potential and fields, plus the seeded velocity perturbation of
 * ehd_set_state_seeded, added to the populations as the change of their
 * equilibrium.  With amp = 0 every plane then evolves as the column does; a
 * start from the column's fields through ehd_set_state_seeded perturbs the
 * planes next to the injector instead.  The column (FP64 or FP32, the
 * context's parameters but for nx, ny, lx, ly) must have stepped at least
 * once since its upload.  Not in the reference. */
int ehd_set_state_from_column(ehd_ctx *ctx, ehd_ctx *column, uint64_t seed, double amp);

/* Steps until the electric Nusselt number Nu_e = I / I0 (I0 from
 * ehd_set_reference_current) changes by less than tol relative between
 * consecutive samples every sample_every steps, hold times in a row, or until
 * max_steps.  A sample is the mean of the currents after the last two steps
 * of its interval (the injector makes the current alternate with a period of
 * two steps), over I0.  *saturated tells which; *nu_e is the last sample.
 * ehd_diagnostics' nu_e is the single-step ratio. */
int ehd_run_to_saturation(ehd_ctx *ctx, int sample_every, double tol, int hold,
                          int64_t max_steps, double *nu_e, int64_t *steps, int *saturated);

/* Binary checkpoint of the complete state (populations of both sets,
 * reference tables, potential, fields, step and time) for a bit-exact
 * resume in a context with the same parameters and precision.  Replaces the
 * lossy save_data_end / read_data restart (LBM.cu:1506-1643), which restarts
 * from equilibrium populations. */
int ehd_checkpoint(ehd_ctx *ctx, const char *path);
int ehd_restore(ehd_ctx *ctx, const char *path);

/* The reference's text formats, on the host: data_end.dat (save_data_end,
 * LBM.cu:1506-1566: ten %10.6f columns t u v w rho q phi Ex Ey Ez, rho q u v w
 * extrapolated onto the walls), and its reader (read_data, LBM.cu:1597-1643)
 * followed by the equilibrium rebuild; the Tecplot writer (save_data_tecplot,
 * LBM.cu:1427-1503; first != 0 writes the VARIABLES header); the uz file for
 * DMD post-processing (save_data_dmd, LBM.cu:1569-1594: "%10.6f %10.6f" t, uz
 * per node, uz extrapolated onto the walls). */
int ehd_write_data_end(ehd_ctx *ctx, const char *path);
int ehd_read_data_end(ehd_ctx *ctx, const char *path);
int ehd_write_tecplot(ehd_ctx *ctx, const char *path, int first);
int ehd_write_dmd(ehd_ctx *ctx, const char *path);

/* --- information -------------------------------------------------------- */

/* Message of the last failed call on this thread ("" if none). */
const char *ehd_last_error(void);

/* ---- Batches of instances (parameter sweeps) ------------------------------
 * No reference counterpart: the reference runs one instance per process.  A
 * batch holds n independent instances (each an ehd_ctx, any grid, one GPU),
 * steps all active ones together -- one CUDA graph launch per step, holding
 * every instance's kernels as parallel branches -- and runs them to
 * saturation of Nu_e, each stopping on its own. */
typedef struct ehd_batch ehd_batch;

/* n instances from params[0..n-1]; config applies to each (its stream is
 * ignored: every instance gets a stream of its own). */
int ehd_batch_create(const ehd_params *params, int n, const ehd_config *config,
                     ehd_batch **out);
int ehd_batch_destroy(ehd_batch *batch);
int ehd_batch_size(const ehd_batch *batch);
/* Instance i as a context (set its state, diagnostics, checkpoints ...); the
 * batch owns it. */
int ehd_batch_instance(ehd_batch *batch, int i, ehd_ctx **ctx);
int ehd_batch_set_active(ehd_batch *batch, int i, int active);
/* How a batch step launches its instances (no reference counterpart).
 * mode 1 (the default): one CUDA graph per step with a branch per instance
 * holding that instance's own launches (the row kernel where it applies);
 * each instance's result is bitwise that of a lone context.  mode 0: instances
 * with the same grid, domain, spacing, permittivity, voltage and launch shapes
 * form a group, and each kernel of the step is one launch over every instance
 * of a group (the LBM half on the persistent row kernel or the per-node
 * kernel, as the instances' tuning says), one graph per step holding the
 * groups' launches; an instance's
 * result agrees with a lone context to FP32 round-off (the grouped kernels
 * are separate compilations, whose multiply-add contractions may differ). */
int ehd_batch_set_mode(ehd_batch *batch, int mode);
/* nsteps steps of every active instance.  Instances whose next step is the
 * first after an upload take that step on their own streams; after it, one
 * graph launch per step covers all active instances. */
int ehd_batch_step(ehd_batch *batch, int nsteps);
/* ehd_run_to_saturation for every active instance at once: each instance
 * stops when it saturates, reaches max_steps or has a non-finite field;
 * saturated[i] is 1, 0 or -1 for these, steps[i] and nu_e[i] as in
 * ehd_run_to_saturation (entries of inactive instances untouched).  Needs I0
 * set on every active instance. */
int ehd_batch_run_to_saturation(ehd_batch *batch, int sample_every, double tol, int hold,
                                int64_t max_steps, int32_t *saturated, int64_t *steps,
                                double *nu_e);
/* Autotuner: times batch steps (the best of three runs of trial_steps each)
 * of a scratch batch with the same parameters and mode while it varies, one
 * distinct grid at a time, the launch shapes of that grid's instances (row or
 * per-node kernel, per-node block, Poisson path, z solve, run-time-radix FFT
 * batches), keeps a change that saves more than 1 %, keeps the starting
 * shapes if the final choice is not faster than them, and applies the result
 * to every instance of that grid (ehd_get_tuning reads the choice).  The
 * instances' states are not touched. */
int ehd_batch_autotune(ehd_batch *batch, int trial_steps);

/* The context's launch shapes (defaults chosen at ehd_create) and a change
 * of them; no reference counterpart (see ehd_tuning). */
int ehd_get_tuning(const ehd_ctx *ctx, ehd_tuning *out);
int ehd_set_tuning(ehd_ctx *ctx, const ehd_tuning *tuning);

/* Bytes of device memory the context holds. */
int ehd_device_bytes(const ehd_ctx *ctx, size_t *bytes);

/* Inverse of compute_parameters (LBM.cu:1356-1379): fills K, nu, charge0 and
 * diffu of *p from the dimensionless groups T, M, C, Fe, keeping eps,
 * voltage, rho0 and lz as they are in *p. */
int ehd_params_from_groups(ehd_params *p, double T, double M, double C, double Fe);

/* compute_parameters itself (LBM.cu:1356-1379). */
int ehd_groups_from_params(const ehd_params *p, double *T, double *M, double *C, double *Fe);

int ehd_abi_version(void);

/* --- no device allocation -------------------------------------------------- */

/* Bytes of device memory held by the file-scope working array of
 * ehd_poisson_noalloc on each GPU it is used on, until the process exits.
 * Under CUDA's lazy module loading (the default) the driver commits the array
 * at the first call on a device; with CUDA_MODULE_LOADING=EAGER, on every GPU
 * when the library loads. */
#define EHD_NOALLOC_SCRATCH_BYTES (64u << 20)

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (their GPU memory is owned by another framework's pool, or an
 * allocation would synchronise a pipeline they run inside): the Poisson solve
 * and E = -grad(phi) of one time step, FP64, on device arrays the caller owns
 * -- q in; phi, ex, ey, ez out; NX*NY*NZ doubles each in the reference layout
 * -- with the same discrete solution as ehd_poisson.  It calls no cudaMalloc,
 * cudaFree or other allocating routine; its working storage is one
 * file-scope device array of EHD_NOALLOC_SCRATCH_BYTES, so grids whose
 * working set exceeds it are rejected with EHD_ERR_INVALID (about
 * 128 x 128 x 129 nodes fit).  The first call on each device (and again
 * after a cudaDeviceReset) looks up the array's device address, which under
 * lazy module loading is when the driver commits the array: make that first
 * call at start-up, before any stream capture.  A CUDA error already pending
 * from the caller's earlier work is returned as EHD_ERR_CUDA before anything
 * is launched, and left pending.  All calls on a device share the array and
 * each call leaves its contents behind: calls whose GPU work overlaps
 * (different streams, host threads) race on it.  Runs on `stream` (NULL: the
 * legacy default stream) on the current device; asynchronous. */
int ehd_poisson_noalloc(const ehd_params *params, const double *q, double *phi, double *ex,
                        double *ey, double *ez, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* EHD_H */
