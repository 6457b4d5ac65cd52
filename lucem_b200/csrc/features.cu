// features.cu -- the resampling of the pyramids, the scale-space maxima of
// the blob detectors, and Canny's suppression and hysteresis.
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
//
// Canny (crates/lucem-ops/src/feature/canny.rs:47-165): the non-maximum
// suppression of canny_nms_kernel (feature/kernels/canny.rs:44-86), with the
// maximum gradient magnitude reduced in the same pass, and the hysteresis.
// The reference's hysteresis is a host BFS from the strong pixels (nms >=
// high) through the weak ones (nms >= low), 8-connected.  The pixels it
// reaches are exactly the 8-connected components of the weak mask that hold
// a strong pixel, so here it is connected-component labelling on the device:
// union-find over the mask where a label only ever moves to a smaller pixel
// index (atomicMin; per 32 x 32 tile in shared memory first, then across the
// tile borders in global memory), roots flagged by their strong pixels, then
// every masked pixel takes its root's flag.  Four launches, no host round
// trip.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
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

__global__ void __launch_bounds__(256) canny_nms_kernel(const float *__restrict__ mag,
                                                        const float *__restrict__ sector, float *__restrict__ nms,
                                                        int H, int W, unsigned int *__restrict__ max_bits) {
    const int64_t total = (int64_t)H * W;
    float local = 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (int64_t)y * W);
        const float m = mag[i];
        if (m > local) local = m;  // NaN and -0 never raise it
        float v = 0.0f;
        if (y > 0 && x > 0 && y + 1 < H && x + 1 < W) {
            const int s = (int)sector[i];
            // Sector 0 compares along the row, 2 along the column, 1 on the
            // main diagonal, 3 on the anti-diagonal.
            const int64_t d = s == 0 ? 1 : (s == 2 ? W : (s == 1 ? (int64_t)W + 1 : (int64_t)W - 1));
            const float n1 = mag[i - d], n2 = mag[i + d];
            v = (m >= n1 && m >= n2) ? m : 0.0f;
        }
        nms[i] = v;
    }
    // Block maximum, then one atomic per block: non-negative floats order as
    // their bit patterns do.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local = fmaxf(local, __shfl_xor_sync(0xffffffffu, local, o));
    __shared__ float warp_max[8];
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = warp_max[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = fmaxf(b, warp_max[w]);
        atomicMax(max_bits, __float_as_uint(b));
    }
}

constexpr uint32_t kNoLabel = 0xffffffffu;

// Root of x: labels point to smaller indices until a root points to itself,
// so the walk ends within x steps.  Loads bypass L1 (other SMs relink).
__device__ __forceinline__ uint32_t find_root(const uint32_t *labels, uint32_t x) {
    uint32_t p = __ldcg(labels + x);
    while (p != x) {
        x = p;
        p = __ldcg(labels + x);
    }
    return x;
}

// Joins the trees of a and b by hanging the larger root under the smaller.
// When the atomic finds the larger root already relinked, the retry starts
// from the value it found, which is smaller: every retry lowers a + b, so
// the loop ends within 2 n rounds (the bound below is never reached).
__device__ __forceinline__ void unite(uint32_t *labels, uint32_t a, uint32_t b, int64_t bound) {
    for (int64_t it = 0; it < bound; ++it) {
        a = find_root(labels, a);
        b = find_root(labels, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicMin(labels + a, b);
        if (old == a) return;
        a = old;
    }
}

// canny.rs:108-116 with both thresholds left to their defaults: 0.1 and 0.2
// of max(max |g|, 0), times that maximum again with use_quantiles; written
// to thr[0..1] on the device, so the call needs no host round trip.
__global__ void canny_thresholds_kernel(const unsigned int *__restrict__ max_bits, int quantiles,
                                        double *__restrict__ thr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double m = fmax((double)__uint_as_float(*max_bits), 0.0);
    double lo = 0.1 * m, hi = 0.2 * m;
    if (quantiles) {
        lo *= m;
        hi *= m;
    }
    thr[0] = lo;
    thr[1] = hi;
}

// The thresholds: from thr (device) when given, else the arguments.  The
// mask is nms >= low when low > 0, else the strong pixels themselves (no
// growth without a positive low threshold); nothing when high <= 0.
__device__ __forceinline__ void canny_thr(const double *thr, double low, double high, double *mask_low,
                                          double *strong) {
    if (thr) {
        low = thr[0];
        high = thr[1];
    }
    *strong = high;
    *mask_low = high > 0.0 ? (low > 0.0 ? low : high) : CUDART_INF;
}

// The labelling runs per 32 x 32 tile in shared memory first: the unions
// inside a tile use shared-memory atomics, and every masked pixel leaves
// with the global index of its tile-local root (the smallest index of its
// tile-local component: row-major order inside a tile is raster order).
// Only the pairs that cross a tile border are then joined in global memory.
constexpr int kLabelTile = 32;

__device__ __forceinline__ uint32_t find_root_s(const volatile uint32_t *L, uint32_t x) {
    uint32_t p = L[x];
    while (p != x) {
        x = p;
        p = L[x];
    }
    return x;
}

// As unite(), on a tile's shared labels (every retry lowers a + b, so the
// loop ends within 2 * 1024 rounds).
__device__ __forceinline__ void unite_s(uint32_t *L, uint32_t a, uint32_t b) {
    for (int it = 0; it < 2 * kLabelTile * kLabelTile + 2; ++it) {
        a = find_root_s(L, a);
        b = find_root_s(L, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicMin(L + a, b);
        if (old == a) return;
        a = old;
    }
}

__global__ void __launch_bounds__(256) canny_label_local_kernel(const float *__restrict__ nms, int H, int W,
                                                                const double *thr, double low, double high,
                                                                uint32_t *__restrict__ labels,
                                                                uint32_t *__restrict__ edges) {
    constexpr int T = kLabelTile, TT = T * T;
    __shared__ uint32_t L[TT];
    double mask_low, strong;
    canny_thr(thr, low, high, &mask_low, &strong);
    const int tiles_x = (W + T - 1) / T, tiles = tiles_x * ((H + T - 1) / T);
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int y0 = (tile / tiles_x) * T, x0 = (tile % tiles_x) * T;
        for (int k = threadIdx.x; k < TT; k += blockDim.x) {
            const int y = y0 + k / T, x = x0 + k % T;
            bool m = false;
            if (y < H && x < W) {
                const int64_t i = (int64_t)y * W + x;
                m = (double)nms[i] >= mask_low;
                edges[i] = 0u;
            }
            L[k] = m ? (uint32_t)k : kNoLabel;
        }
        __syncthreads();
        // Unions with the raster-earlier neighbours inside the tile.
        for (int k = threadIdx.x; k < TT; k += blockDim.x) {
            if (L[k] == kNoLabel) continue;
            const int ly = k / T, lx = k % T;
            if (lx > 0 && L[k - 1] != kNoLabel) unite_s(L, (uint32_t)k, (uint32_t)(k - 1));
            if (ly > 0) {
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = lx + dx;
                    if (nx < 0 || nx >= T) continue;
                    const int j = k - T + dx;
                    if (L[j] != kNoLabel) unite_s(L, (uint32_t)k, (uint32_t)j);
                }
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < TT; k += blockDim.x) {
            const int y = y0 + k / T, x = x0 + k % T;
            if (y >= H || x >= W) continue;
            uint32_t g = kNoLabel;
            if (L[k] != kNoLabel) {
                const uint32_t r = find_root_s(L, (uint32_t)k);
                g = (uint32_t)((int64_t)(y0 + (int)r / T) * W + x0 + (int)r % T);
            }
            labels[(int64_t)y * W + x] = g;
        }
        __syncthreads();
    }
}

// The pairs across tile borders: a pixel on a tile's top row joins its
// three neighbours above, one on its left column its left and upper-left
// neighbours, one on its right column its upper-right neighbour (all in
// other tiles, all raster-earlier).  One thread per (tile, border slot).
__global__ void canny_label_border_kernel(int H, int W, uint32_t *__restrict__ labels) {
    constexpr int T = kLabelTile;
    const int tiles_x = (W + T - 1) / T, tiles = tiles_x * ((H + T - 1) / T);
    const int64_t total = (int64_t)tiles * 3 * T, bound = 2 * (int64_t)H * W + 2;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < total; s += (int64_t)gridDim.x * blockDim.x) {
        const int tile = (int)(s / (3 * T)), slot = (int)(s % (3 * T));
        const int y0 = (tile / tiles_x) * T, x0 = (tile % tiles_x) * T;
        int y, x;
        if (slot < T) { y = y0; x = x0 + slot; }                    // top row
        else if (slot < 2 * T) { y = y0 + slot - T; x = x0; }       // left column
        else { y = y0 + slot - 2 * T; x = x0 + T - 1; }             // right column
        if (y >= H || x >= W) continue;
        const int64_t i = (int64_t)y * W + x;
        if (__ldcg(labels + i) == kNoLabel) continue;
        const bool top = y == y0 && y > 0, left = x == x0 && x > 0, right = x == x0 + T - 1 && y > y0;
        if (top) {
            for (int dx = -1; dx <= 1; ++dx) {
                const int nx = x + dx;
                if (nx < 0 || nx >= W) continue;
                const int64_t j = i - W + dx;
                if (__ldcg(labels + j) != kNoLabel) unite(labels, (uint32_t)i, (uint32_t)j, bound);
            }
        }
        if (left) {
            if (__ldcg(labels + i - 1) != kNoLabel) unite(labels, (uint32_t)i, (uint32_t)(i - 1), bound);
            if (y > y0 && __ldcg(labels + i - W - 1) != kNoLabel)
                unite(labels, (uint32_t)i, (uint32_t)(i - W - 1), bound);
        }
        if (right && x + 1 < W && __ldcg(labels + i - W + 1) != kNoLabel)
            unite(labels, (uint32_t)i, (uint32_t)(i - W + 1), bound);
    }
}

// Every masked pixel's label becomes its root; a strong pixel flags its root.
__global__ void canny_label_root_kernel(const float *__restrict__ nms, int64_t total, const double *thr, double low,
                                        double high, uint32_t *__restrict__ labels, uint32_t *__restrict__ edges) {
    double mask_low, strong;
    canny_thr(thr, low, high, &mask_low, &strong);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        if (__ldcg(labels + i) == kNoLabel) continue;
        const uint32_t r = find_root(labels, (uint32_t)i);
        labels[i] = r;
        if ((double)nms[i] >= strong) edges[r] = 2u;
    }
}

// Edges: the masked pixels whose root was flagged.  A root rewrites its own
// flag 2 -> 1 while others read it; both are non-zero.
__global__ void canny_label_final_kernel(int64_t total, const uint32_t *__restrict__ labels,
                                         uint32_t *__restrict__ edges) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = labels[i];
        edges[i] = (r != kNoLabel && __ldcg(edges + r) != 0u) ? 1u : 0u;
    }
}

unsigned grid_for(int64_t total, int threads) {
    int64_t blocks = (total + threads - 1) / threads;
    if (blocks > 148 * 16) blocks = 148 * 16;
    return (unsigned)(blocks < 1 ? 1 : blocks);
}

}  // namespace

int launch_canny_nms(const float *mag, const float *sector, float *nms, int H, int W, unsigned int *max_bits,
                     void *stream) {
    const int64_t total = (int64_t)H * W;
    if (total <= 0) return 0;
    canny_nms_kernel<<<grid_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(mag, sector, nms, H, W,
                                                                                          max_bits);
    return (int)cudaGetLastError();
}

int launch_canny_thresholds(const unsigned int *max_bits, int quantiles, double *thr, void *stream) {
    canny_thresholds_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(max_bits, quantiles, thr);
    return (int)cudaGetLastError();
}

int launch_canny_hysteresis(const float *nms, int H, int W, const double *thr, double low, double high,
                            uint32_t *labels, uint32_t *edges, void *stream) {
    const int64_t total = (int64_t)H * W;
    if (total <= 0) return 0;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const unsigned g = grid_for(total, 256);
    const int64_t tiles = (int64_t)((W + kLabelTile - 1) / kLabelTile) * ((H + kLabelTile - 1) / kLabelTile);
    canny_label_local_kernel<<<(unsigned)std::min<int64_t>(tiles, 148 * 8), 256, 0, cs>>>(nms, H, W, thr, low, high,
                                                                                         labels, edges);
    canny_label_border_kernel<<<grid_for(tiles * 3 * kLabelTile, 256), 256, 0, cs>>>(H, W, labels);
    canny_label_root_kernel<<<g, 256, 0, cs>>>(nms, total, thr, low, high, labels, edges);
    canny_label_final_kernel<<<g, 256, 0, cs>>>(total, labels, edges);
    return (int)cudaGetLastError();
}

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
