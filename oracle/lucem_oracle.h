/*
 * lucem_oracle.h -- CPU restatement of lucem-ops' separable Gaussian family and
 * Richardson-Lucy deconvolution.  TEST INFRASTRUCTURE ONLY: the parity tests,
 * the smoke check and the benchmark's CPU-baseline leg call it to check results.
 * The product (lucem_b200) never links or calls anything in this directory.
 *
 * Parity status: the reference (Rust + CubeCL 0.11.4, not vendored) cannot be
 * built in this environment (no Rust toolchain, no network), and its tests
 * hold no golden vectors.  This restatement is pinned instead to
 *   - the reference's own known-answer tests for the path, restated in
 *     tests/test_oracle.py (crates/lucem-ops/src/filter/gaussian.rs:442-459,
 *     crates/lucem-ops/src/filter/convolve.rs:185-228,
 *     crates/lucem-ops/src/restore/deconvolve.rs:517-578), and
 *   - scipy.ndimage (an independent implementation of the same published
 *     filters, same radius rule and half-sample reflect) through fixtures in
 *     tests/golden/ made by tests/golden/make_golden.py.
 * Bit-level CubeCL CPU-runtime output is therefore not pinned.
 *
 * Every f32 routine accumulates exactly as the reference kernel does: an f32
 * accumulator starting at 0, taps in index order, acc += w[t] * x (the
 * compiler may contract to FMA, as CubeCL's CPU runtime may).
 */
#ifndef LUCEM_ORACLE_H
#define LUCEM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pad modes, ids as crates/lucem-ops/src/core/pad.rs:84-88. */
enum { ORC_REFLECT = 0, ORC_CONSTANT = 1, ORC_NEAREST = 2, ORC_MIRROR = 3, ORC_WRAP = 4 };

/* crates/lucem-ops/src/filter/gaussian.rs:22-63: 2*radius+1 f64 taps. */
void orc_gaussian_kernel_1d(double sigma, uint32_t order, int64_t radius, double *out);

/* crates/lucem-ops/src/filter/gaussian.rs:83-85. */
int64_t orc_resolved_radius(double truncate, double sigma);

/* crates/lucem-ops/src/core/kernels/pad.rs:11-34 (-1 = constant fill). */
int64_t orc_pad_index(int64_t p, int64_t len, int mode);

/* crates/lucem-ops/src/filter/kernels/convolve.rs:14-59 over a C-contiguous
 * array of ndim dims, along `axis` (already normalised), f32 arithmetic. */
void orc_correlate_1d_f32(const float *in, float *out, const int64_t *dims, int ndim, int axis,
                          const float *w, int64_t size, int32_t origin, int mode, float cval);
/* Same in f64 (the reference's host test model, convolve.rs:185-209). */
void orc_correlate_1d_f64(const double *in, double *out, const int64_t *dims, int ndim, int axis,
                          const double *w, int64_t size, int32_t origin, int mode, double cval);

/* crates/lucem-ops/src/filter/gaussian.rs:176-237 with core/separable.rs:20-61:
 * per-axis sigmas/orders/radii already broadcast over `naxes` axes (ascending
 * order of the reference's pass list); sigma==0 axes are skipped; radius<0
 * means "resolved from truncate".  Returns 0.  f32 / f64 variants. */
int orc_gaussian_blur_f32(const float *in, float *out, const int64_t *dims, int ndim,
                          const int *axes, int naxes, const double *sigmas, const uint32_t *orders,
                          const int64_t *radii, int mode, double cval, double truncate);
int orc_gaussian_blur_f64(const double *in, double *out, const int64_t *dims, int ndim,
                          const int *axes, int naxes, const double *sigmas, const uint32_t *orders,
                          const int64_t *radii, int mode, double cval, double truncate);

/* crates/lucem-ops/src/core/kernels/elementwise.rs:136-149:
 * out = alpha*a + beta*b + bias in f32. */
void orc_linear_comb_f32(const float *a, const float *b, float *out, int64_t n, float alpha,
                         float beta, float bias);

/* crates/lucem-ops/src/filter/gaussian.rs:255-288 (LoG), :307-356 (gradient
 * magnitude), :374-390 (DoG), :407-421 (unsharp), all axes, f32. */
int orc_gaussian_laplace_f32(const float *in, float *out, const int64_t *dims, int ndim,
                             const double *sigmas, int mode, double cval, double truncate);
int orc_gaussian_grad_mag_f32(const float *in, float *out, const int64_t *dims, int ndim,
                              const double *sigmas, int mode, double cval, double truncate);
int orc_difference_of_gaussians_f32(const float *in, float *out, const int64_t *dims, int ndim,
                                    const double *low, const double *high, int mode, double cval,
                                    double truncate);
int orc_unsharp_mask_f32(const float *in, float *out, const int64_t *dims, int ndim,
                         const double *sigmas, double amount, int mode, double cval,
                         double truncate);

/* crates/lucem-ops/src/filter/kernels/convolve.rs:62-118 generalised to N-D
 * (ndim 1..3): dense correlation, window centred at k/2 per axis, pad maps per
 * axis, cval where any axis is out (Constant), taps in C order. */
void orc_correlate_nd_f32(const float *in, float *out, const int64_t *dims, int ndim,
                          const float *w, const int64_t *kdims, int mode, float cval);
void orc_correlate_nd_f64(const double *in, double *out, const int64_t *dims, int ndim,
                          const double *w, const int64_t *kdims, int mode, double cval);

/* crates/lucem-ops/src/restore/deconvolve.rs:45-149 generalised to N-D
 * (the reference is 2-D only): host PSF normalisation, flipped copy, est0=0.5,
 * guard |c|<eps -> eps, update est*corr, clip on the last iteration.
 * `eps` is the already-floored epsilon (max(eps, 1e-15)).  f32 / f64. */
int orc_richardson_lucy_f32(const float *obs, const float *psf, float *out, const int64_t *dims,
                            const int64_t *kdims, int ndim, int num_iter, int clip, double eps,
                            int mode);
int orc_richardson_lucy_f64(const double *obs, const double *psf, double *out,
                            const int64_t *dims, const int64_t *kdims, int ndim, int num_iter,
                            int clip, double eps, int mode);

/* Threads the OpenMP loops above use (0 = OpenMP default). */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
