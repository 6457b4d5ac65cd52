// filter.cu -- sm_100a kernels for lucem-ops' separable Gaussian family.
//
// family_kernel: every Gaussian-family response of one 2-D input in one pass.
//   Reference path replaced: gaussian_blur_into -> separable::run ->
//   correlate_1d_kernel, one launch per axis, plus linear_comb_kernel /
//   add_sq_kernel / sqrt_scale_kernel for DoG, LoG, gradient magnitude and
//   unsharp (crates/lucem-ops/src/filter/gaussian.rs:176-435,
//   crates/lucem-ops/src/filter/kernels/convolve.rs:14-59,
//   crates/lucem-ops/src/filter/kernels/gradient.rs:36-52,
//   crates/lucem-ops/src/core/kernels/elementwise.rs:136-149).
//   A 64x64 output tile plus its halo is staged once in shared memory with
//   the u8/u16 -> f32 cast (and scale) fused into the load.  For each
//   separable filter the axis-0 pass (rows, first, as the reference orders
//   its passes) runs over the tile and the columns of the axis-1 halo and is
//   stored transposed; the axis-1 pass then reads it conflict-free.  Each
//   thread keeps 8 outputs in registers along the filtered direction and
//   slides over the taps 8 at a time, so shared-memory loads are 1/8 of the
//   FMAs.  Responses that combine two filters (DoG, LoG, |grad|, unsharp) are
//   accumulated in registers across filters and written once.
//
// correlate_1d kernels: the reference's 1-D correlation along any axis of an
//   N-D array ([outer, len, inner] view, crates/lucem-core/src/shape.rs:9-20),
//   any weights, origin and pad mode, staged through shared memory; same
//   accumulation order as the reference (f32, taps ascending).

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"


#include "filter_family.cuh"

namespace lucem {

using namespace famk;


int family_tile_dims(int *th, int *tw) {
    *th = kTH;
    *tw = kTW;
    return 0;
}

size_t family_smem_bytes(int rmax0, int rmax1) {
    size_t a = (size_t)(kTH + 2 * rmax0) * (kTW + 2 * rmax1);
    size_t it = (size_t)(kTW + 2 * rmax1) * kITP;
    return (a + it) * sizeof(float) + 64;
}

int launch_family_planes(const FamParams &p, int in_dtype, void *stream) {
    switch (in_dtype) {
    case LUCEM_U8: return planes_u8(p, stream);
    case LUCEM_U16: return planes_u16(p, stream);
    case LUCEM_F32: return planes_f32(p, stream);
    default: return (int)cudaErrorInvalidValue;
    }
}

int launch_family_batch(const FamParams &p, int in_dtype, const FamImage *items_dev, int32_t n_items,
                        int32_t n_tiles, void *stream) {
    switch (in_dtype) {
    case LUCEM_U8: return batch_u8(p, items_dev, n_items, n_tiles, stream);
    case LUCEM_U16: return batch_u16(p, items_dev, n_items, n_tiles, stream);
    case LUCEM_F32: return batch_f32(p, items_dev, n_items, n_tiles, stream);
    default: return (int)cudaErrorInvalidValue;
    }
}

int launch_family_work(const FamParams &p, int in_dtype, const FamWork *work_dev, int32_t n_work,
                       int32_t n_tiles_total, int32_t tile_base, int32_t *counter_dev,
                       int32_t persistent_ctas, void *stream) {
    switch (in_dtype) {
    case LUCEM_U8: return work_u8(p, work_dev, n_work, n_tiles_total, tile_base, counter_dev, persistent_ctas, stream);
    case LUCEM_U16: return work_u16(p, work_dev, n_work, n_tiles_total, tile_base, counter_dev, persistent_ctas, stream);
    case LUCEM_F32: return work_f32(p, work_dev, n_work, n_tiles_total, tile_base, counter_dev, persistent_ctas, stream);
    default: return (int)cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Generic 1-D correlation (crates/lucem-ops/src/filter/kernels/convolve.rs:14-59).

namespace {

constexpr int kRowSeg = 1024;      // outputs per CTA along a contiguous axis
constexpr int kRowMaxHalo = 15360; // beyond this: direct kernel
constexpr int kColI = 128, kColK = 32;
constexpr int kColPer = kColI / 8;  // consecutive outputs per thread along a strided axis (8 row groups)
constexpr int kColMaxHalo = 960;

// Register blocking of both kernels: a thread computes several consecutive
// outputs, taps in blocks of 8 held in registers, each staged sample loaded
// once per block and used by every output it reaches.  Every output still
// accumulates its taps in index order from 0 (the reference's order), so
// the results are those of one fmaf chain per output.
constexpr int kRowPer = 4;  // consecutive outputs per thread along a contiguous axis

// Staged samples along a contiguous axis at index i + i / 32: four
// consecutive outputs per lane read 32 distinct banks.
__device__ __forceinline__ int row_slot(int i) { return i + (i >> 5); }

template <typename T, int MODE>
__global__ void __launch_bounds__(256)
corr_row_kernel(const T *__restrict__ in, float scale, float *__restrict__ out, int64_t outer,
                int len, const float *__restrict__ w, int size, int left, float cval) {
    extern __shared__ float4 smem4[];
    float *S = reinterpret_cast<float *>(smem4);
    const int n_in = kRowSeg + size - 1;
    float *Wsm = S + row_slot(n_in + 16);
    const int segs = (len + kRowSeg - 1) / kRowSeg;
    for (int t = threadIdx.x; t < size; t += blockDim.x) Wsm[t] = w[t];
    for (int64_t b = blockIdx.x; b < outer * segs; b += gridDim.x) {
        int64_t o = b / segs;
        int i0 = (int)(b - o * segs) * kRowSeg;
        const T *row = in + o * len;
        __syncthreads();
        for (int j = threadIdx.x; j < n_in; j += blockDim.x) {
            int q = pad_index<MODE>(i0 - left + j, len);
            S[row_slot(j)] = q < 0 ? cval : static_cast<float>(row[q]) * scale;
        }
        __syncthreads();
        for (int jb = threadIdx.x; jb < kRowSeg / kRowPer; jb += blockDim.x) {
            const int j0 = jb * kRowPer;
            if (i0 + j0 >= len) break;
            float acc[kRowPer];
#pragma unroll
            for (int j = 0; j < kRowPer; ++j) acc[j] = 0.0f;
            for (int s0 = 0; s0 < size; s0 += 8) {
                float wv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) wv[u] = s0 + u < size ? Wsm[s0 + u] : 0.0f;
                // Samples past the staged ones (at most 7, in the slack
                // after S) meet only taps past the end: never accumulated.
#pragma unroll
                for (int m = 0; m < 8 + kRowPer - 1; ++m) {
                    const float x = S[row_slot(j0 + s0 + m)];
#pragma unroll
                    for (int j = 0; j < kRowPer; ++j) {
                        const int u = m - j;
                        if (u >= 0 && u < 8 && s0 + u < size) acc[j] = fmaf(wv[u], x, acc[j]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kRowPer; ++j)
                if (i0 + j0 + j < len) out[o * len + i0 + j0 + j] = acc[j];
        }
    }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256)
corr_col_kernel(const T *__restrict__ in, float scale, float *__restrict__ out, int64_t outer,
                int len, int64_t inner, const float *__restrict__ w, int size, int left, float cval) {
    extern __shared__ float4 smem4[];
    float *S = reinterpret_cast<float *>(smem4);  // [kColI + size - 1 + 8 slack rows][kColK]
    float *Wsm = S + (kColI + size - 1 + 8) * kColK;
    const int64_t ks = (inner + kColK - 1) / kColK;
    const int is = (len + kColI - 1) / kColI;
    const int64_t nblk = outer * is * ks;
    for (int t = threadIdx.x; t < size; t += blockDim.x) Wsm[t] = w[t];
    const int kk = threadIdx.x & (kColK - 1);
    const int ig = threadIdx.x / kColK;  // 0..7, kColPer outputs each
    for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
        int64_t o = b / (is * ks);
        int64_t r = b - o * is * ks;
        int i0 = (int)(r / ks) * kColI;
        int64_t k0 = (r % ks) * kColK;
        const T *base = in + o * len * inner;
        int n_in = kColI + size - 1;
        __syncthreads();
        for (int j = threadIdx.x; j < n_in * kColK; j += blockDim.x) {
            int ii = j / kColK, kc = j - ii * kColK;
            int64_t k = k0 + kc;
            float v = 0.0f;
            if (k < inner) {
                int q = pad_index<MODE>(i0 - left + ii, len);
                v = q < 0 ? cval : static_cast<float>(base[(int64_t)q * inner + k]) * scale;
            }
            S[j] = v;
        }
        __syncthreads();
        int64_t k = k0 + kk;
        if (k < inner) {
            const int ii0 = ig * kColPer;
            float acc[kColPer];
#pragma unroll
            for (int j = 0; j < kColPer; ++j) acc[j] = 0.0f;
            for (int s0 = 0; s0 < size; s0 += 8) {
                float wv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) wv[u] = s0 + u < size ? Wsm[s0 + u] : 0.0f;
                // Rows past the staged ones (at most 7, in the slack rows
                // after S) meet only taps past the end: never accumulated.
#pragma unroll
                for (int m = 0; m < 8 + kColPer - 1; ++m) {
                    const float x = S[(ii0 + s0 + m) * kColK + kk];
#pragma unroll
                    for (int j = 0; j < kColPer; ++j) {
                        const int u = m - j;
                        if (u >= 0 && u < 8 && s0 + u < size) acc[j] = fmaf(wv[u], x, acc[j]);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < kColPer; ++j)
                if (i0 + ii0 + j < len) out[(o * len + i0 + ii0 + j) * inner + k] = acc[j];
        }
    }
}

template <typename T, int MODE>
__global__ void corr_direct_kernel(const T *__restrict__ in, float scale, float *__restrict__ out,
                                   int64_t total, int len, int64_t inner,
                                   const float *__restrict__ w, int size, int left, float cval) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = (e / inner) % len;
        int64_t base = e - i * inner;
        int start = (int)i - left;
        float acc = 0.0f;
        for (int t = 0; t < size; ++t) {
            int q = pad_index<MODE>(start + t, len);
            float v = q < 0 ? cval : static_cast<float>(in[base + (int64_t)q * inner]) * scale;
            acc = fmaf(w[t], v, acc);
        }
        out[e] = acc;
    }
}

template <typename T, int MODE>
int corr_launch(const T *in, float scale, float *out, int64_t outer, int64_t len, int64_t inner,
                const float *w, int size, int left, float cval, cudaStream_t s) {
    const int sms = sm_count();
    if (inner == 1 && size - 1 <= kRowMaxHalo) {
        size_t smem = (size_t)((kRowSeg + size - 1 + 16) + (kRowSeg + size + 15) / 32 + 1 + size) * sizeof(float) + 16;
        int64_t nb = outer * ((len + kRowSeg - 1) / kRowSeg);
        int grid = (int)(nb < (int64_t)sms * 16 ? nb : (int64_t)sms * 16);
        cudaFuncSetAttribute(corr_row_kernel<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        corr_row_kernel<T, MODE><<<grid, 256, smem, s>>>(in, scale, out, outer, (int)len, w, size, left, cval);
    } else if (inner > 1 && size - 1 <= kColMaxHalo) {
        size_t smem = (size_t)((kColI + size - 1 + 8) * kColK + size) * sizeof(float) + 16;
        int64_t nb = outer * ((len + kColI - 1) / kColI) * ((inner + kColK - 1) / kColK);
        int grid = (int)(nb < (int64_t)sms * 16 ? nb : (int64_t)sms * 16);
        cudaFuncSetAttribute(corr_col_kernel<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        corr_col_kernel<T, MODE><<<grid, 256, smem, s>>>(in, scale, out, outer, (int)len, inner, w, size, left, cval);
    } else {
        int64_t total = outer * len * inner;
        int64_t nb = (total + 255) / 256;
        int grid = (int)(nb < (int64_t)sms * 32 ? nb : (int64_t)sms * 32);
        corr_direct_kernel<T, MODE><<<grid, 256, 0, s>>>(in, scale, out, total, (int)len, inner, w, size, left, cval);
    }
    return (int)cudaGetLastError();
}

template <typename T>
int corr_mode(const T *in, float scale, float *out, int64_t outer, int64_t len, int64_t inner,
              const float *w, int size, int left, int mode, float cval, cudaStream_t s) {
    switch (mode) {
    case 0: return corr_launch<T, 0>(in, scale, out, outer, len, inner, w, size, left, cval, s);
    case 1: return corr_launch<T, 1>(in, scale, out, outer, len, inner, w, size, left, cval, s);
    case 2: return corr_launch<T, 2>(in, scale, out, outer, len, inner, w, size, left, cval, s);
    case 3: return corr_launch<T, 3>(in, scale, out, outer, len, inner, w, size, left, cval, s);
    case 4: return corr_launch<T, 4>(in, scale, out, outer, len, inner, w, size, left, cval, s);
    default: return (int)cudaErrorInvalidValue;
    }
}

// ---- elementwise -----------------------------------------------------------

__global__ void linear_comb_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                   float *__restrict__ out, int64_t n, float alpha, float beta,
                                   float bias) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float v = alpha * a[i];
        if (b) v = v + beta * b[i];
        out[i] = v + bias;
    }
}

__global__ void add_sq_kernel(const float *__restrict__ d, float *__restrict__ acc, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float g = d[i];
        acc[i] = fmaf(g, g, acc[i]);
    }
}

__global__ void sqrt_scale_kernel(const float *__restrict__ acc, float *__restrict__ out, int64_t n,
                                  float scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = sqrtf(fmaxf(acc[i], 0.0f)) * scale;
}

template <typename T>
__global__ void cast_kernel(const T *__restrict__ in, float scale, float *__restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = static_cast<float>(in[i]) * scale;
}

__global__ void fill_kernel(float *__restrict__ out, int64_t n, float v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = v;
}

int ew_grid(int64_t n) {
    int64_t nb = (n + 255) / 256;
    int64_t cap = (int64_t)sm_count() * 16;
    return (int)(nb < cap ? (nb > 0 ? nb : 1) : cap);
}

}  // namespace

int launch_correlate_1d(const void *in, int in_dtype, float in_scale, float *out, int64_t outer,
                        int64_t len, int64_t inner, const float *w_dev, int32_t size, int32_t left,
                        int32_t mode, float cval, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (in_dtype) {
    case LUCEM_U8: return corr_mode(static_cast<const uint8_t *>(in), in_scale, out, outer, len, inner, w_dev, size, left, mode, cval, s);
    case LUCEM_U16: return corr_mode(static_cast<const uint16_t *>(in), in_scale, out, outer, len, inner, w_dev, size, left, mode, cval, s);
    case LUCEM_F32: return corr_mode(static_cast<const float *>(in), in_scale, out, outer, len, inner, w_dev, size, left, mode, cval, s);
    default: return (int)cudaErrorInvalidValue;
    }
}

// Halo part of the adjoint of one correlate_1d pass.  The forward pass reads
// in[pad(i + t - left)] for output i and tap t; its adjoint scatters
// w[t] * g[i] back to pad(i + t - left).  The interior part (positions that
// are already inside the line) is a zero-padded correlation with the reversed
// taps (launch_correlate_1d); this kernel adds, per line, what the forward
// read from the extended positions p < 0 and p >= len, at pad(p) (nothing for
// the constant mode).  One thread owns one line, so the sums into a line are
// race-free and in a fixed order.
__global__ void adjoint_fold_kernel(const float *__restrict__ g, float scale, float *__restrict__ out,
                                    int64_t outer, int64_t len, int64_t inner, const float *__restrict__ w,
                                    int size, int left, int mode) {
    const int64_t lines = outer * inner;
    const int n = (int)len;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < lines;
         l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = l / inner, c = l - o * inner;
        const float *gl = g + o * len * inner + c;
        float *ol = out + o * len * inner + c;
        // Extended positions: [-left, 0) then [n, n + size - 1 - left).
        const int n_lo = left, n_hi = size - 1 - left;
        for (int k = 0; k < n_lo + n_hi; ++k) {
            const int p = k < n_lo ? k - left : n + (k - n_lo);
            const int q = pad_index_rt(p, n, mode);
            if (q < 0) continue;
            // taps t with i = p + left - t inside [0, n)
            const int t0 = max(0, p + left - n + 1), t1 = min(size - 1, p + left);
            float acc = 0.0f;
            for (int t = t0; t <= t1; ++t) acc = fmaf(w[t], gl[(int64_t)(p + left - t) * inner], acc);
            ol[(int64_t)q * inner] += scale * acc;
        }
    }
}

int launch_adjoint_fold(const float *g, float scale, float *out, int64_t outer, int64_t len, int64_t inner,
                        const float *w_dev, int32_t size, int32_t left, int32_t mode, void *stream) {
    const int64_t lines = outer * inner;
    if (lines == 0 || mode == LUCEM_PAD_CONSTANT) return 0;
    adjoint_fold_kernel<<<ew_grid(lines), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        g, scale, out, outer, len, inner, w_dev, size, left, mode);
    return (int)cudaGetLastError();
}

namespace {
// The tensor epilogue (tensor_ops.cuh) over stored components: the path of
// filters too wide for the fused kernel, and structure_tensor_eigvals.
__global__ void tensor_elementwise_kernel(const float *__restrict__ a, const float *__restrict__ b,
                                          const float *__restrict__ c, float *o0, float *o1, float *o2, int64_t n,
                                          int mode, float p0, float p1, int black, int first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float prev = first ? 0.0f : o0[i];
        float v0, v1 = 0.0f, v2 = 0.0f;
        const int k = tens::apply(mode, a[i], b[i], c ? c[i] : 0.0f, prev, p0, p1, black != 0, &v0, &v1, &v2);
        o0[i] = v0;
        if (k > 1) o1[i] = v1;
        if (k > 2) o2[i] = v2;
    }
}
}  // namespace

int launch_tensor_elementwise(const float *a, const float *b, const float *c, float *o0, float *o1, float *o2,
                              int64_t n, int mode, float p0, float p1, int black, int first, void *stream) {
    if (n == 0) return 0;
    tensor_elementwise_kernel<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(a, b, c, o0, o1, o2, n,
                                                                                          mode, p0, p1, black, first);
    return (int)cudaGetLastError();
}

int launch_linear_comb(const float *a, const float *b, float *out, int64_t n, float alpha,
                       float beta, float bias, void *stream) {
    if (n == 0) return 0;
    linear_comb_kernel<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(a, b, out, n, alpha, beta, bias);
    return (int)cudaGetLastError();
}

int launch_add_sq(const float *d, float *acc, int64_t n, void *stream) {
    if (n == 0) return 0;
    add_sq_kernel<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(d, acc, n);
    return (int)cudaGetLastError();
}

int launch_sqrt_scale(const float *acc, float *out, int64_t n, float scale, void *stream) {
    if (n == 0) return 0;
    sqrt_scale_kernel<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(acc, out, n, scale);
    return (int)cudaGetLastError();
}

int launch_cast(const void *in, int in_dtype, float scale, float *out, int64_t n, void *stream) {
    if (n == 0) return 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (in_dtype) {
    case LUCEM_U8: cast_kernel<<<ew_grid(n), 256, 0, s>>>(static_cast<const uint8_t *>(in), scale, out, n); break;
    case LUCEM_U16: cast_kernel<<<ew_grid(n), 256, 0, s>>>(static_cast<const uint16_t *>(in), scale, out, n); break;
    case LUCEM_F32: cast_kernel<<<ew_grid(n), 256, 0, s>>>(static_cast<const float *>(in), scale, out, n); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

int launch_fill(float *out, int64_t n, float v, void *stream) {
    if (n == 0) return 0;
    fill_kernel<<<ew_grid(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, n, v);
    return (int)cudaGetLastError();
}

}  // namespace lucem
