// spectral.cu -- complex FFTs along one axis of an [outer, len, inner] array:
// the O(N log N) replacement of the reference's direct DFT
// (dft_axis_kernel, crates/lucem-ops/src/core/kernels/fft.rs:9-47, driven by
// fft_1d_into / fft_nd_into, crates/lucem-ops/src/core/fft.rs:14-100), and the
// frequency-domain filter of Wiener deconvolution
// (wiener_freq_filter_kernel, restore/kernels/deconvolve.rs:49-73).
//
// One kernel (fft_lines_kernel) transforms C lines per CTA in shared memory
// with the self-sorting Stockham stages of fft.cuh (any 2,3,5,7-smooth
// length up to kFftLinesMax).  Options on the way in and out make the other
// lengths out of the same kernel:
//   - four-step (smooth lengths above kFftLinesMax, n = n1 n2): lines of n1
//     with a twiddle W_n^(m2 k1) on the way out, then lines of n2 whose
//     output rows are scattered to k1 + n1 k2;
//   - Bluestein (other lengths, 2 len - 1 <= kFftLinesMax): chirp on the way
//     in, the chirp filter's spectrum between a forward and an inverse
//     transform of a smooth length M >= 2 len - 1, chirp on the way out;
//   - anything else: a direct DFT kernel (the reference's algorithm, with
//     exact integer phase reduction and host-computed twiddles).
// Inputs and outputs are split complex (separate real and imaginary arrays,
// as the reference's DeviceArray pairs) or interleaved (the scratch between
// axes).
#include <cuda_runtime.h>

#include <cstdint>

#include "fft.cuh"
#include "internal.h"

namespace lucem {

namespace {

using fft::cmul;

__device__ __forceinline__ int64_t line_base(int64_t O, int32_t odiv, int64_t os_hi, int64_t os_lo) {
    if (odiv > 1) {
        const int64_t hi = O / odiv;
        return hi * os_hi + (O - hi * odiv) * os_lo;
    }
    return O * os_hi;
}

__global__ void __launch_bounds__(512) fft_lines_kernel(const __grid_constant__ FftLines p) {
    extern __shared__ float4 smem4[];
    const float2 *sc = reinterpret_cast<const float2 *>(p.sc), *pre = reinterpret_cast<const float2 *>(p.pre);
    const float2 *mid = reinterpret_cast<const float2 *>(p.mid), *post = reinterpret_cast<const float2 *>(p.post);
    const float2 *twg = reinterpret_cast<const float2 *>(p.tw), *tw_big = reinterpret_cast<const float2 *>(p.tw_big);
    float2 *dc = reinterpret_cast<float2 *>(p.dc);
    const int n = p.n, C = p.C, CP = p.CP, T = blockDim.x, tid = threadIdx.x;
    float2 *tws = reinterpret_cast<float2 *>(smem4);
    float2 *bufA = tws + n;
    float2 *bufB = bufA + n * CP;
    for (int i = tid; i < n; i += T) tws[i] = twg[i];
    const fft::Tw tw{tws, 1};
    const int64_t nlines = p.n_outer * p.inner;
    const int64_t ntiles = (nlines + C - 1) / C;
    // Lines along a contiguous axis (inner == 1): lanes run along the rows of
    // a line; otherwise along neighbouring lines (coalesced either way).
    const bool rows_fast = p.inner == 1;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t L0 = t * C;
        __syncthreads();
        for (int it = tid; it < n * C; it += T) {
            int row, c;
            if (rows_fast) {
                c = it / n;
                row = it - c * n;
            } else {
                row = it / C;
                c = it - row * C;
            }
            const int64_t L = L0 + c;
            float2 v = make_float2(0.f, 0.f);
            if (L < nlines && row < p.src_rows) {
                const int64_t O = L / p.inner, k = L - O * p.inner;
                const int64_t at = line_base(O, p.s_odiv, p.s_os_hi, p.s_os_lo) + k + row * p.s_rs;
                v = sc ? sc[at] : make_float2(p.sre[at], p.sim ? p.sim[at] : 0.f);
                if (p.conj_in) v.y = -v.y;
                if (pre) v = cmul(v, pre[row]);
            }
            bufA[row * CP + c] = v;
        }
        __syncthreads();
        float2 *buf = fft::stockham(bufA, bufB, n, C, CP, p.plan.radix, p.plan.nstages, tw, p.inverse != 0);
        if (mid) {
            for (int it = tid; it < n * C; it += T) {
                const int row = it / C, c = it - row * C;
                buf[row * CP + c] = cmul(buf[row * CP + c], mid[row]);
            }
            __syncthreads();
            buf = fft::stockham(buf, buf == bufA ? bufB : bufA, n, C, CP, p.plan.radix, p.plan.nstages, tw,
                                p.inverse == 0);
        }
        for (int it = tid; it < p.dst_rows * C; it += T) {
            int row, c;
            if (rows_fast) {
                c = it / p.dst_rows;
                row = it - c * p.dst_rows;
            } else {
                row = it / C;
                c = it - row * C;
            }
            const int64_t L = L0 + c;
            if (L >= nlines) continue;
            const int64_t O = L / p.inner, k = L - O * p.inner;
            float2 v = buf[row * CP + c];
            if (post) v = cmul(v, post[row]);
            if (p.twiddle_n) {
                // Four-step: W_N^(m2 k1), m2 = the line's index along the
                // second factor (k / inner2), k1 = this output row.
                const int64_t m2 = k / p.tw_div;
                float2 w = tw_big[(m2 * row) % p.twiddle_n];
                if (p.inverse) w.y = -w.y;
                v = cmul(v, w);
            }
            if (p.conj_out) v.y = -v.y;
            v.x *= p.scale;
            v.y *= p.scale;
            const int64_t at = line_base(O, p.d_odiv, p.d_os_hi, p.d_os_lo) + k + row * p.d_rs;
            if (dc) {
                dc[at] = v;
            } else {
                if (p.clip) v.x = fminf(fmaxf(v.x, -1.0f), 1.0f);
                p.dre[at] = v.x;
                if (p.dim) p.dim[at] = v.y;
            }
        }
    }
}

// The reference's direct DFT along the axis (one thread per output), for
// lengths with no smooth Bluestein length within kFftLinesMax: twiddles from
// the host table W_len^m with the exact phase (j m) mod len.
__global__ void dft_direct_kernel(const __grid_constant__ FftLines p) {
    const float2 *sc = reinterpret_cast<const float2 *>(p.sc), *twg = reinterpret_cast<const float2 *>(p.tw);
    float2 *dc = reinterpret_cast<float2 *>(p.dc);
    const int64_t total = p.n_outer * p.inner * p.n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t L = e / p.n;
        const int j = (int)(e - L * p.n);
        const int64_t O = L / p.inner, k = L - O * p.inner;
        const int64_t sb = line_base(O, p.s_odiv, p.s_os_hi, p.s_os_lo) + k;
        float sr = 0.f, si = 0.f;
        for (int m = 0; m < p.n; ++m) {
            const int64_t at = sb + m * p.s_rs;
            float2 x = sc ? sc[at] : make_float2(p.sre[at], p.sim ? p.sim[at] : 0.f);
            float2 w = twg[(int)(((int64_t)j * m) % p.n)];
            if (p.inverse) w.y = -w.y;
            sr = fmaf(x.x, w.x, fmaf(-x.y, w.y, sr));
            si = fmaf(x.x, w.y, fmaf(x.y, w.x, si));
        }
        float2 v = make_float2(sr * p.scale, si * p.scale);
        const int64_t at = line_base(O, p.d_odiv, p.d_os_hi, p.d_os_lo) + k + j * p.d_rs;
        if (dc) {
            dc[at] = v;
        } else {
            if (p.clip) v.x = fminf(fmaxf(v.x, -1.0f), 1.0f);
            p.dre[at] = v.x;
            if (p.dim) p.dim[at] = v.y;
        }
    }
}

// Wiener filter in the frequency domain (restore/kernels/deconvolve.rs:61-72):
// X = conj(H) Y / max(|H|^2 + balance |L|^2, eps), |L|^2 = L conj(L).
__global__ void wiener_filter_kernel(const float2 *__restrict__ y, const float2 *__restrict__ h,
                                     const float2 *__restrict__ l, float2 *__restrict__ x, int64_t n,
                                     float balance, float eps) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 yv = y[i], hv = h[i], lv = l[i];
        const float l2 = lv.x * lv.x - lv.y * -lv.y;  // re of L conj(L) (complex_mul_kernel with conj_b)
        const float h2 = hv.x * hv.x + hv.y * hv.y;
        const float den = fmaxf(h2 + balance * l2, eps);
        x[i] = make_float2((hv.x * yv.x + hv.y * yv.y) / den, (hv.x * yv.y - hv.y * yv.x) / den);
    }
}

// out = a * b or a * conj(b), split complex (complex_mul_kernel,
// crates/lucem-ops/src/core/kernels/fft.rs:53-75).
__global__ void complex_mul_kernel(const float *__restrict__ ar, const float *__restrict__ ai,
                                   const float *__restrict__ br, const float *__restrict__ bi, float *__restrict__ outr,
                                   float *__restrict__ outi, int64_t n, int conj_b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float a = ar[i], b = ai[i], c = br[i], d = conj_b ? 0.0f - bi[i] : bi[i];
        outr[i] = a * c - b * d;
        outi[i] = a * d + b * c;
    }
}

// Zero-filled [H][W] complex buffer with the small kernel's tap (ky, kx) at
// ((ky - kh/2) mod H, (kx - kw/2) mod W) (fft_shift_2d_kernel,
// restore/kernels/deconvolve.rs:79-99).
__global__ void centre_kernel_kernel(const float *__restrict__ k, int kh, int kw, float2 *__restrict__ out, int H,
                                     int W) {
    const int n = kh * kw;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int ky = i / kw, kx = i - ky * kw;
        const int y = ((ky - kh / 2) % H + H) % H, x = ((kx - kw / 2) % W + W) % W;
        out[(int64_t)y * W + x] = make_float2(k[i], 0.0f);
    }
}

int grid_for(int64_t n, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t nb = (n + threads - 1) / threads, cap = (int64_t)sms * 16;
    return (int)(nb < cap ? (nb > 0 ? nb : 1) : cap);
}

}  // namespace

int fft_lines_max() { return kFftLinesMax; }

int launch_fft_lines(FftLines p, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = p.n;
    // Lines per CTA: two n x CP buffers plus the twiddles within ~200 KB;
    // one line needs no padding column.
    int C = 64;
    while (C > 1 && ((size_t)n * (1 + 2 * (size_t)(C + 1))) * sizeof(float2) > 200 * 1024) C >>= 1;
    p.C = C;
    p.CP = C > 1 ? C + 1 : 1;
    const size_t smem = ((size_t)n + 2 * (size_t)n * p.CP) * sizeof(float2);
    int T = (int)((((int64_t)n * C / 8) + 31) / 32 * 32);
    T = T < 128 ? 128 : (T > 512 ? 512 : T);
    const int64_t nlines = p.n_outer * p.inner, ntiles = (nlines + C - 1) / C;
    if (ntiles == 0) return 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = (int)((227 * 1024) / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    const int64_t slots = (int64_t)sms * per_sm;
    const int grid = (int)(ntiles < slots ? ntiles : slots);
    cudaFuncSetAttribute(fft_lines_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fft_lines_kernel<<<grid, T, smem, s>>>(p);
    return (int)cudaGetLastError();
}

int launch_dft_direct(const FftLines &p, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t total = p.n_outer * p.inner * p.n;
    if (total == 0) return 0;
    dft_direct_kernel<<<grid_for(total, 256), 256, 0, s>>>(p);
    return (int)cudaGetLastError();
}

int launch_wiener_filter(const float2_ *y, const float2_ *h, const float2_ *l, float2_ *x, int64_t n, float balance,
                         float eps, void *stream) {
    wiener_filter_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2 *>(y), reinterpret_cast<const float2 *>(h), reinterpret_cast<const float2 *>(l),
        reinterpret_cast<float2 *>(x), n, balance, eps);
    return (int)cudaGetLastError();
}

int launch_complex_mul(const float *ar, const float *ai, const float *br, const float *bi, float *outr, float *outi,
                       int64_t n, int conj_b, void *stream) {
    complex_mul_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(ar, ai, br, bi, outr, outi, n,
                                                                                      conj_b);
    return (int)cudaGetLastError();
}

int launch_centre_kernel(const float *k, int kh, int kw, float2_ *out, int H, int W, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int e = (int)cudaMemsetAsync(out, 0, (size_t)H * W * sizeof(float2_), s);
    if (e) return e;
    centre_kernel_kernel<<<grid_for((int64_t)kh * kw, 256), 256, 0, s>>>(k, kh, kw, reinterpret_cast<float2 *>(out),
                                                                          H, W);
    return (int)cudaGetLastError();
}

}  // namespace lucem
