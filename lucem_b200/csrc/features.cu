// features.cu -- the resampling of the pyramids, and the scale-space maxima
// of the blob detectors.
//
// Resampling (resize, crates/lucem-ops/src/transform/warp.rs:207-251, through
// affine_coords_2d_kernel, transform/kernels/warp.rs:10-33, and the order 0
// and 1 arms of sample_2d_kernel, core/kernels/spline.rs:90-139): output
// pixel (oy, ox) samples the input at (m0 oy + m2, m4 ox + m5), the
// reference's f32 coordinate arithmetic, nearest or bilinear with the pad
// map outside the image; one thread per output pixel.
//
// Blob maxima: the scale-space maxima of the blob detectors
// (extract_scale_space_blobs, crates/lucem-ops/src/feature/blobs.rs:139-201):
// one thread per (scale, y, x) sample of the response stack, kept on the
// device, tested against its 3 x 3 x 3 neighbourhood (scales clamped to the
// stack) with the reference's threshold, border and tie rule (a neighbour
// wins on a larger value, or on an equal value at a lexicographically
// smaller (scale, y, x)).  Survivors are appended to a list through an
// atomic counter; the host sorts and prunes them.  The reference scans the
// whole stack on the host.
//
// No two survivors are neighbours (each would have to beat the other), so at
// most one survives per 2 x 2 x 2 block: ceil(ns/2) ceil(H/2) ceil(W/2)
// bounds the list (blob_candidate_bound).
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace lucem {

namespace {

__global__ void blob_candidates_kernel(const float *__restrict__ cube, int ns, int H, int W, int border,
                                       double threshold, BlobCandidate *__restrict__ out, int64_t cap,
                                       unsigned long long *__restrict__ count) {
    const int64_t plane = (int64_t)H * W, total = plane * ns;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(e / plane);
        const int64_t r = e - (int64_t)s * plane;
        const int y = (int)(r / W), x = (int)(r - (int64_t)y * W);
        if (y < border || y >= H - border || x < border || x >= W - border) continue;
        const float val = cube[e];
        if ((double)val <= threshold) continue;
        const int s_lo = s > 0 ? s - 1 : 0, s_hi = s + 1 < ns ? s + 1 : ns - 1;
        bool is_max = true;
        for (int ts = s_lo; ts <= s_hi && is_max; ++ts) {
            for (int ty = y - 1; ty <= y + 1 && is_max; ++ty) {
                for (int tx = x - 1; tx <= x + 1; ++tx) {
                    if (ts == s && ty == y && tx == x) continue;
                    const float nv = cube[(int64_t)ts * plane + (int64_t)ty * W + tx];
                    const bool before = ts < s || (ts == s && (ty < y || (ty == y && tx < x)));
                    if (nv > val || (nv == val && before)) {
                        is_max = false;
                        break;
                    }
                }
            }
        }
        if (!is_max) continue;
        const unsigned long long i = atomicAdd(count, 1ull);
        if ((int64_t)i < cap) out[i] = BlobCandidate{val, s, y, x};
    }
}

// The reference's pad map (core/kernels/pad.rs:11-34); -1: the constant.
__device__ __forceinline__ int pad_at(int p, int len, int mode) {
    if (p >= 0 && p < len) return p;
    if (mode == LUCEM_PAD_CONSTANT) return -1;
    if (mode == LUCEM_PAD_NEAREST) return p < 0 ? 0 : len - 1;
    if (mode == LUCEM_PAD_WRAP) return ((p % len) + len) % len;
    if (mode == LUCEM_PAD_REFLECT) {
        const int period = 2 * len;
        const int r = ((p % period) + period) % period;
        return r < len ? r : period - 1 - r;
    }
    const int period = max(2 * len - 2, 1);
    const int r = ((p % period) + period) % period;
    return r < len ? r : period - r;
}

__global__ void resample_kernel(const float *__restrict__ in, int H, int W, float *__restrict__ out, int OH, int OW,
                                float m0, float m2, float m4, float m5, int order, int mode, float cval) {
    const int64_t total = (int64_t)OH * OW;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float oy = (float)(int)(i / OW), ox = (float)(int)(i - (i / OW) * OW);
        // affine_coords_2d_kernel with the resize matrix (the off-diagonal
        // terms and the homogeneous row are 0 0 1: exact).
        const float y = __fadd_rn(__fmul_rn(m0, oy), m2), x = __fadd_rn(__fmul_rn(m4, ox), m5);
        float v;
        if (order == 0) {
            const int py = pad_at((int)floorf(__fadd_rn(y, 0.5f)), H, mode);
            const int px = pad_at((int)floorf(__fadd_rn(x, 0.5f)), W, mode);
            v = (py < 0 || px < 0) ? cval : in[(int64_t)py * W + px];
        } else {
            const float fyl = floorf(y), fxl = floorf(x);
            const int y0 = (int)fyl, x0 = (int)fxl;
            const float fy = __fsub_rn(y, fyl), fx = __fsub_rn(x, fxl);
            float acc = 0.0f;
#pragma unroll
            for (int dy = 0; dy < 2; ++dy) {
                const float wy = dy == 0 ? __fsub_rn(1.0f, fy) : fy;
                const int py = pad_at(y0 + dy, H, mode);
#pragma unroll
                for (int dx = 0; dx < 2; ++dx) {
                    const float wx = dx == 0 ? __fsub_rn(1.0f, fx) : fx;
                    const int px = pad_at(x0 + dx, W, mode);
                    const float sample = (py < 0 || px < 0) ? cval : in[(int64_t)py * W + px];
                    acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(wy, wx), sample));
                }
            }
            v = acc;
        }
        out[i] = v;
    }
}

}  // namespace

int launch_resample(const float *in, int H, int W, float *out, int OH, int OW, float m0, float m2, float m4,
                    float m5, int order, int mode, float cval, void *stream) {
    const int64_t total = (int64_t)OH * OW;
    if (total <= 0) return 0;
    int64_t blocks = (total + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    resample_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(in, H, W, out, OH, OW, m0, m2,
                                                                                     m4, m5, order, mode, cval);
    return (int)cudaGetLastError();
}

int64_t blob_candidate_bound(int ns, int64_t H, int64_t W) {
    return (int64_t)((ns + 1) / 2) * ((H + 1) / 2) * ((W + 1) / 2);
}

int launch_blob_candidates(const float *cube, int ns, int H, int W, int border, double threshold,
                           BlobCandidate *out, int64_t cap, unsigned long long *count, void *stream) {
    const int64_t total = (int64_t)ns * H * W;
    if (total <= 0) return 0;
    const int threads = 256;
    int64_t blocks = (total + threads - 1) / threads;
    if (blocks > 148 * 32) blocks = 148 * 32;
    blob_candidates_kernel<<<(unsigned)blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(
        cube, ns, H, W, border, threshold, out, cap, count);
    return (int)cudaGetLastError();
}

}  // namespace lucem
