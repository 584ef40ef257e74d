/* ehd_fno.h -- a 3D Fourier neural operator that predicts a later state of the
 * EHD step from its initial fields and dimensionless groups, as a warm start
 * that skips the linear-growth transient.  No counterpart in the reference
 * (gyf135/EHD-convection-3D has no learned component); the plain step stays
 * the arbiter of every warm start: each one is run on by the step itself.
 *
 * Architecture (the published Fourier neural operator, Li et al. 2021):
 *   v0 = a P + p                                  (lift, pointwise)
 *   v_{l+1} = gelu(K_l(v_l) + v_l W_l + b_l)      (no gelu after the last layer)
 *   u = gelu(v_L Q1 + q1) Q2 + q2                 (projection, pointwise)
 * with the spectral convolution K_l(v) = IDFT(R_l . DFT(v)) keeping the modes
 * kx = 0..mx-1 of a real transform along x and the mx_y, mx_z lowest
 * positive and negative modes along y and z; R_l is a complex
 * width x width matrix per kept mode.  Transforms are truncated DFTs carried
 * out as matrix products, so the lift, pointwise layers, transforms,
 * projection and all of their adjoints run on the BF16 tensor cores with
 * FP32 accumulation, the weights read as BF16 copies of the FP32 ones (the
 * optimizer's).  The mode mixing -- per kept mode a matrix-vector product
 * for each sample, weight-bound -- runs in FP32 on the FP32 weights.
 *
 * Fields are channels-last FP32 device arrays [batch][z][y][x][channel]. */
#ifndef EHD_FNO_H
#define EHD_FNO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ehd_fno ehd_fno;

typedef struct ehd_fno_config {
    int32_t nx, ny, nz;           /* grid                                       */
    int32_t in_channels;          /* channels of the input a                    */
    int32_t out_channels;         /* channels of the output u                   */
    int32_t width;                /* channels of the hidden layers              */
    int32_t layers;               /* Fourier layers                             */
    int32_t modes_x;              /* kx = 0 .. modes_x - 1 (real transform)     */
    int32_t modes_y, modes_z;     /* 0 .. m-1 and n-m .. n-1 along y, z         */
    int32_t hidden;               /* width of the projection's inner layer     */
    int32_t max_batch;            /* largest batch passed to the calls below   */
    uint64_t seed;                /* weight initialisation                      */
    int32_t device;               /* CUDA device                                */
    int32_t reserved[5];          /* must be 0                                  */
} ehd_fno_config;

int ehd_fno_create(const ehd_fno_config *config, ehd_fno **out);
int ehd_fno_destroy(ehd_fno *fno);
/* Number of FP32 parameters; their order is: P, p, then per layer W_l, b_l,
 * Re R_l, Im R_l (R_l as [mode][out][in], modes ordered (kz, ky, kx) with
 * kz, ky counted 0..m-1 then the negative ones), then Q1, q1, Q2, q2;
 * matrices as [in][out]. */
int ehd_fno_param_count(const ehd_fno *fno, int64_t *count);
int ehd_fno_get_params(ehd_fno *fno, float *host);
int ehd_fno_set_params(ehd_fno *fno, const float *host);
/* u = FNO(a) for `batch` samples (device pointers). */
int ehd_fno_forward(ehd_fno *fno, int batch, const float *a, float *u);
/* Forward, the mean-square loss against `target`, and the gradient of the
 * loss with respect to every parameter (kept in the object, replacing the
 * previous one).  *loss gets the loss; NULL skips it. */
int ehd_fno_backward(ehd_fno *fno, int batch, const float *a, const float *target,
                     double *loss);
int ehd_fno_get_grads(ehd_fno *fno, float *host);
/* One Adam step (bias-corrected) on the parameters with the kept gradient. */
int ehd_fno_adam_step(ehd_fno *fno, float lr, float beta1, float beta2, float eps);
/* The calls run on the object's own stream; this waits for them. */
int ehd_fno_synchronize(ehd_fno *fno);

/* The tensor-core product the FNO is built on, exposed for testing:
 * C[b][m][n] = alpha sum_k A[b][m][k] B[b][k][n] + beta C[b][m][n], FP32
 * operands on the device rounded to BF16, FP32 accumulation; element (i, j)
 * of X is at X + b * xb + i * x_row + j * x_col. */
int ehd_bf16_gemm(int M, int N, int K, int batch, const float *A, int64_t a_row,
                  int64_t a_col, int64_t ab, const float *B, int64_t b_row, int64_t b_col,
                  int64_t bb, float *C, int64_t c_row, int64_t c_col, int64_t cb, float alpha,
                  float beta, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* EHD_FNO_H */
