/*
 * lucem_oracle.c -- CPU restatement of the reference path (see the header for
 * its role and parity status).  Test infrastructure only.
 */
#include "lucem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

static inline float fabs_f32(float x) { return fabsf(x); }
static inline double fabs_f64(double x) { return fabs(x); }

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

/* crates/lucem-ops/src/filter/gaussian.rs:22-63.  phi(x) = exp(-x^2 / 2s^2)
 * over x in [-r, r], normalised by its f64 sum; orders 1..3 multiply by the
 * Hermite factor q_k(x), higher orders by the recurrence at :46-56, and odd
 * orders are negated for the correlation convention (:58-60). */
void orc_gaussian_kernel_1d(double sigma, uint32_t order, int64_t radius, double *out) {
    if (radius == 0) {
        out[0] = order == 0 ? 1.0 : 0.0;
        return;
    }
    double sigma2 = sigma * sigma;
    int64_t n = 2 * radius + 1;
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double x = (double)(i - radius);
        out[i] = exp(-0.5 * (x * x) / sigma2);
    }
    for (int64_t i = 0; i < n; ++i) sum += out[i];
    for (int64_t i = 0; i < n; ++i) out[i] /= sum;
    if (order == 0) return;
    for (int64_t i = 0; i < n; ++i) {
        double x = (double)(i - radius);
        double q;
        if (order == 1) q = -x / sigma2;
        else if (order == 2) q = (x * x - sigma2) / (sigma2 * sigma2);
        else if (order == 3) q = -(x * x * x - 3.0 * x * sigma2) / (sigma2 * sigma2 * sigma2);
        else {
            double h_prev = 1.0, h_cur = -x / sigma2;
            for (uint32_t k = 1; k < order; ++k) {
                double h_next = (-x / sigma2) * h_cur - ((double)k / sigma2) * h_prev;
                h_prev = h_cur;
                h_cur = h_next;
            }
            q = h_cur;
        }
        double sign = (order % 2 == 1) ? -1.0 : 1.0;
        out[i] = sign * q * out[i];
    }
}

/* crates/lucem-ops/src/filter/gaussian.rs:83-85: floor(truncate*sigma + 0.5), >= 0. */
int64_t orc_resolved_radius(double truncate, double sigma) {
    double r = floor(truncate * sigma + 0.5);
    return r > 0.0 ? (int64_t)r : 0;
}

/* crates/lucem-ops/src/core/kernels/pad.rs:11-34. */
int64_t orc_pad_index(int64_t p, int64_t len, int mode) {
    if (p >= 0 && p < len) return p;
    switch (mode) {
    case ORC_CONSTANT: return -1;
    case ORC_NEAREST: return p < 0 ? 0 : len - 1;
    case ORC_WRAP: return ((p % len) + len) % len;
    case ORC_REFLECT: {
        int64_t period = 2 * len;
        int64_t r = ((p % period) + period) % period;
        return r < len ? r : period - 1 - r;
    }
    default: { /* Mirror; a length-1 axis has period clamped to 1 (:26-30). */
        int64_t period = 2 * len - 2;
        if (period < 1) period = 1;
        int64_t r = ((p % period) + period) % period;
        return r < len ? r : period - r;
    }
    }
}

#define REAL float
#define SFX f32
#include "lucem_oracle_body.inc"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "lucem_oracle_body.inc"
#undef REAL
#undef SFX

/* crates/lucem-ops/src/core/kernels/elementwise.rs:136-149. */
void orc_linear_comb_f32(const float *a, const float *b, float *out, int64_t n, float alpha,
                         float beta, float bias) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) out[i] = alpha * a[i] + beta * b[i] + bias;
}

static int all_axes(int ndim, int *axes) {
    for (int d = 0; d < ndim; ++d) axes[d] = d;
    return ndim;
}

/* crates/lucem-ops/src/filter/gaussian.rs:255-288: output = G_{ax0 order 2};
 * then per further axis term = G_{order 2 on that axis}, accum = out + term,
 * out = accum. */
int orc_gaussian_laplace_f32(const float *in, float *out, const int64_t *dims, int ndim,
                             const double *sigmas, int mode, double cval, double truncate) {
    int64_t total = 1;
    for (int d = 0; d < ndim; ++d) total *= dims[d];
    if (total == 0) return 0;
    int axes[8];
    all_axes(ndim, axes);
    float *term = (float *)malloc(sizeof(float) * (size_t)total);
    for (int ax = 0; ax < ndim; ++ax) {
        uint32_t orders[8] = {0};
        orders[ax] = 2;
        if (ax == 0) {
            orc_gaussian_blur_f32(in, out, dims, ndim, axes, ndim, sigmas, orders, NULL, mode,
                                  cval, truncate);
        } else {
            orc_gaussian_blur_f32(in, term, dims, ndim, axes, ndim, sigmas, orders, NULL, mode,
                                  cval, truncate);
            orc_linear_comb_f32(out, term, out, total, 1.0f, 1.0f, 0.0f);
        }
    }
    free(term);
    return 0;
}

/* crates/lucem-ops/src/filter/gaussian.rs:307-356 with the kernels
 * filter/kernels/gradient.rs:36-52: accum += d*d per axis, then
 * sqrt(max(accum, 0)) * 1. */
int orc_gaussian_grad_mag_f32(const float *in, float *out, const int64_t *dims, int ndim,
                              const double *sigmas, int mode, double cval, double truncate) {
    int64_t total = 1;
    for (int d = 0; d < ndim; ++d) total *= dims[d];
    if (total == 0) return 0;
    int axes[8];
    all_axes(ndim, axes);
    float *acc = (float *)calloc((size_t)total, sizeof(float));
    float *deriv = (float *)malloc(sizeof(float) * (size_t)total);
    for (int ax = 0; ax < ndim; ++ax) {
        uint32_t orders[8] = {0};
        orders[ax] = 1;
        orc_gaussian_blur_f32(in, deriv, dims, ndim, axes, ndim, sigmas, orders, NULL, mode, cval,
                              truncate);
        for (int64_t i = 0; i < total; ++i) acc[i] += deriv[i] * deriv[i];
    }
    for (int64_t i = 0; i < total; ++i) out[i] = sqrtf(acc[i] > 0.0f ? acc[i] : 0.0f) * 1.0f;
    free(acc);
    free(deriv);
    return 0;
}

/* crates/lucem-ops/src/filter/gaussian.rs:374-390. */
int orc_difference_of_gaussians_f32(const float *in, float *out, const int64_t *dims, int ndim,
                                    const double *low, const double *high, int mode, double cval,
                                    double truncate) {
    int64_t total = 1;
    for (int d = 0; d < ndim; ++d) total *= dims[d];
    if (total == 0) return 0;
    int axes[8];
    all_axes(ndim, axes);
    uint32_t orders[8] = {0};
    float *lo = (float *)malloc(sizeof(float) * (size_t)total);
    float *hi = (float *)malloc(sizeof(float) * (size_t)total);
    orc_gaussian_blur_f32(in, lo, dims, ndim, axes, ndim, low, orders, NULL, mode, cval, truncate);
    orc_gaussian_blur_f32(in, hi, dims, ndim, axes, ndim, high, orders, NULL, mode, cval, truncate);
    orc_linear_comb_f32(lo, hi, out, total, 1.0f, -1.0f, 0.0f);
    free(lo);
    free(hi);
    return 0;
}

/* crates/lucem-ops/src/filter/gaussian.rs:407-421. */
int orc_unsharp_mask_f32(const float *in, float *out, const int64_t *dims, int ndim,
                         const double *sigmas, double amount, int mode, double cval,
                         double truncate) {
    int64_t total = 1;
    for (int d = 0; d < ndim; ++d) total *= dims[d];
    if (total == 0) return 0;
    int axes[8];
    all_axes(ndim, axes);
    uint32_t orders[8] = {0};
    float *bl = (float *)malloc(sizeof(float) * (size_t)total);
    orc_gaussian_blur_f32(in, bl, dims, ndim, axes, ndim, sigmas, orders, NULL, mode, cval, truncate);
    orc_linear_comb_f32(in, bl, out, total, (float)(1.0 + amount), (float)(-amount), 0.0f);
    free(bl);
    return 0;
}
