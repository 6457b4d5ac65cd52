// tensor_ops.cuh -- per-pixel functions of a 2-D symmetric tensor field
// (a, b, c) = (A_rr, A_rc, A_cc): the epilogues the fused Gaussian-family
// kernel applies to its first three filter responses, and the elementwise
// kernel that applies them to stored components.  Each restates the
// reference kernel it replaces, in f32 with every product rounded (no
// contraction), as the reference's CubeCL kernels:
//   - det:        hessian_det_2d_kernel, crates/lucem-ops/src/feature/kernels/structure.rs:6-20
//   - eigvals:    sym_eigvals_2x2_kernel, crates/lucem-ops/src/core/kernels/eigen.rs:13-33
//   - shape index: shape_index_2d_kernel, feature/kernels/structure.rs:40-80 (the
//                 reference's own odd polynomial for atan on [0, 1])
//   - Frangi, Sato, Meijering: filter/kernels/ridge.rs:11-98 (one scale,
//                 folded into the running maximum)
//   - outer products: outer_product_2d_kernel, feature/kernels/structure.rs:22-38
//   - blob responses: the scaled LoG / DoG (scale_offset_into after the sum
//                 or difference, core/elementwise.rs:50-75) and doh_scale_kernel
//                 (feature/kernels/blobs.rs:8-21)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace lucem {

namespace tens {

__device__ __forceinline__ void eigvals(float a, float b, float c, float *l1, float *l2) {
    const float mean = __fmul_rn(__fadd_rn(a, c), 0.5f);
    const float diff = __fmul_rn(__fsub_rn(a, c), 0.5f);
    const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(diff, diff), __fmul_rn(b, b)));
    *l1 = __fadd_rn(mean, r);
    *l2 = __fsub_rn(mean, r);
}

__device__ __forceinline__ float shape_index(float l1, float l2) {
    const float diff = __fsub_rn(l1, l2), sum = __fadd_rn(l1, l2);
    const float scale = __fadd_rn(fabsf(l1), fabsf(l2));
    if (fabsf(diff) <= __fmul_rn(1e-6f, scale) || scale <= 1e-20f) {
        // Equal curvatures: the formula's limit (+1 dome, -1 cup, 0 flat).
        if (sum < 0.0f && scale > 1e-20f) return 1.0f;
        if (sum > 0.0f && scale > 1e-20f) return -1.0f;
        return 0.0f;
    }
    const float ratio = __fdiv_rn(-sum, diff);
    const float ax = fabsf(ratio);
    const bool inv = ax > 1.0f;
    const float z = inv ? __fdiv_rn(1.0f, ax) : ax;
    const float z2 = __fmul_rn(z, z);
    float poly = __fadd_rn(-0.085133f, __fmul_rn(z2, 0.0208351f));
    poly = __fadd_rn(0.180141f, __fmul_rn(z2, poly));
    poly = __fadd_rn(-0.3302995f, __fmul_rn(z2, poly));
    poly = __fadd_rn(0.999866f, __fmul_rn(z2, poly));
    const float atan_z = __fmul_rn(z, poly);
    const float angle = inv ? __fsub_rn(1.5707964f, atan_z) : atan_z;
    return __fmul_rn(ratio < 0.0f ? -angle : angle, 0.63661975f);
}

// One scale of a ridge filter from the Hessian eigenvalues; `valid` false:
// the running maximum is left as it is.
__device__ __forceinline__ float ridge(int mode, float e1, float e2, float p0, float p1, bool black, bool *valid) {
    *valid = true;
    if (mode == kTensorFrangi) {
        const bool le = fabsf(e1) <= fabsf(e2);
        const float l1 = le ? e1 : e2, l2 = le ? e2 : e1;
        *valid = black ? l2 > 0.0f : l2 < 0.0f;
        if (!*valid) return 0.0f;
        const float al2 = fmaxf(fabsf(l2), 1e-10f);
        const float rb = __fdiv_rn(l1, al2);
        const float s2 = __fadd_rn(__fmul_rn(l1, l1), __fmul_rn(l2, l2));
        const float e_rb = expf(__fsub_rn(0.0f, __fmul_rn(__fmul_rn(rb, rb), p0)));
        const float e_s = expf(__fsub_rn(0.0f, __fmul_rn(s2, p1)));
        return __fmul_rn(e_rb, __fsub_rn(1.0f, e_s));
    }
    if (mode == kTensorSato) {
        const float s1 = __fmul_rn(e1, p0), s2 = __fmul_rn(e2, p0);
        const float l2 = fabsf(s1) <= fabsf(s2) ? s2 : s1;
        return black ? fmaxf(l2, 0.0f) : fmaxf(__fsub_rn(0.0f, l2), 0.0f);
    }
    // Meijering: modified eigenvalues l1 - l2/3, l2 - l1/3.
    const float third = -1.0f / 3.0f;
    const float m1 = __fadd_rn(e1, __fmul_rn(third, e2)), m2 = __fadd_rn(e2, __fmul_rn(third, e1));
    const float dom = fabsf(m1) >= fabsf(m2) ? m1 : m2;
    return black ? fmaxf(dom, 0.0f) : fmaxf(__fsub_rn(0.0f, dom), 0.0f);
}

// The epilogue of one pixel: (a, b, c) in, up to three outputs; prev: the
// running maximum of the ridge modes.
__device__ __forceinline__ int apply(int mode, float a, float b, float c, float prev, float p0, float p1, bool black,
                                     float *o0, float *o1, float *o2) {
    switch (mode) {
    case kTensorDet:
        *o0 = __fsub_rn(__fmul_rn(a, c), __fmul_rn(b, b));
        return 1;
    case kTensorEigvals:
        eigvals(a, b, c, o0, o1);
        return 2;
    case kTensorShapeIndex: {
        float l1, l2;
        eigvals(a, b, c, &l1, &l2);
        *o0 = shape_index(l1, l2);
        return 1;
    }
    case kTensorScaledSum:
        // scale_offset_into of the reference applied to the sum
        // (gaussian_laplace_into) or difference (difference_of_gaussians_into).
        *o0 = __fmul_rn(p0, __fadd_rn(a, __fmul_rn(p1, b)));
        return 1;
    case kTensorScaledDet:
        // doh_scale_kernel, crates/lucem-ops/src/feature/kernels/blobs.rs:8-21.
        *o0 = __fmul_rn(p0, __fsub_rn(__fmul_rn(a, c), __fmul_rn(b, b)));
        return 1;
    case kTensorCannyGrad: {
        // canny_grad_dir_kernel, crates/lucem-ops/src/feature/kernels/canny.rs:13-41.
        *o0 = __fsqrt_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)));
        const float ay = fabsf(a), ax = fabsf(b), t = 0.41421357f;
        *o1 = ay <= __fmul_rn(ax, t) ? 0.0f : (ax <= __fmul_rn(ay, t) ? 2.0f : (__fmul_rn(a, b) >= 0.0f ? 1.0f : 3.0f));
        return 2;
    }
    case kTensorOuter:
        *o0 = __fmul_rn(a, a);
        *o1 = __fmul_rn(a, b);
        *o2 = __fmul_rn(b, b);
        return 3;
    default: {
        float l1, l2;
        eigvals(a, b, c, &l1, &l2);
        bool valid;
        const float r = ridge(mode, l1, l2, p0, p1, black, &valid);
        *o0 = valid ? fmaxf(prev, r) : prev;
        return 1;
    }
    }
}

}  // namespace tens
}  // namespace lucem
