// spectral_ops.cu -- the frequency-domain operators built on lucem_fft_nd
// (host side in api.cpp):
//   - per-axis spectral filters of crates/lucem-ops/src/filter/spectral.rs:21-164
//     (fourier_gaussian_into, fourier_box_into, fourier_shift_into): every
//     axis's factor in one pass over the spectrum, applied in axis order with
//     the reference's f32 products (spectral_scale_axis_kernel /
//     spectral_phase_axis_kernel, filter/kernels/spectral.rs:10-51);
//   - the Butterworth transfer function of filter/spectral.rs:168-213,
//     evaluated per bin in FP64 on the device instead of a host array;
//   - phase correlation (crates/lucem-ops/src/register/phase.rs:51-255): the
//     cross-power spectrum, the |cc|^2 argmax, and the subpixel refinement's
//     candidate sums as FP64 reductions on the device (the reference pulls
//     the spectrum to the host and loops there);
//   - unsupervised Wiener (crates/lucem-ops/src/restore/deconvolve.rs:357-509):
//     each iteration's residual / prior / trace sums as one FP64 reduction on
//     the device and the balance update (with the reference's PCG jitter) in
//     a one-thread kernel, so the whole chain runs without host round trips.
// Reductions are two-stage (per-block partials, then one block in fixed
// order): results do not depend on scheduling.
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.h"

namespace lucem {

namespace {

constexpr int kRedThreads = 256;
constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of v (all threads get nothing back; thread 0 returns the sum).
__device__ double block_sum(double v, double *sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Signed normalised frequency of bin k of an n-point axis (k <= n/2: k/n,
// else (k - n)/n), as the reference's host tables.
__device__ __forceinline__ double freq_of(int64_t k, int64_t n) {
    return k <= n / 2 ? (double)k / (double)n : (double)(k - n) / (double)n;
}

// ---- per-axis spectral filters --------------------------------------------

__global__ void spectral_axes_kernel(float *__restrict__ re, float *__restrict__ im, uint32_t n,
                                     const float *__restrict__ tab, const SpecAxes a) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        float r = re[e], m = im[e];
        for (int d = 0; d < a.ndim; ++d) {
            const uint32_t k = (e / a.inner[d]) % a.len[d];
            if (a.phase) {
                const float c = tab[a.off[d] + k], s = tab[a.off[d] + a.len[d] + k];
                // r * c - m * s, r * s + m * c, each product rounded (no contraction).
                const float nr = __fsub_rn(__fmul_rn(r, c), __fmul_rn(m, s));
                const float nm = __fadd_rn(__fmul_rn(r, s), __fmul_rn(m, c));
                r = nr;
                m = nm;
            } else {
                const float w = tab[a.off[d] + k];
                r = __fmul_rn(r, w);
                m = __fmul_rn(m, w);
            }
        }
        re[e] = r;
        im[e] = m;
    }
}

// ---- Butterworth ------------------------------------------------------------

// X[e] *= w(e), w = 1 / (1 + |f / cutoff|^(2 order)) (low pass) or 1 - that,
// in FP64 and rounded once to f32, as the reference's host array.
__global__ void butterworth_kernel(float2_ *__restrict__ X, uint32_t n, const SpecAxes a, double cutoff, double order,
                                   int high_pass) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        double r2 = 0.0;
        for (int d = 0; d < a.ndim; ++d) {
            const uint32_t k = (e / a.inner[d]) % a.len[d];
            const double q = freq_of(k, a.len[d]) / cutoff;
            r2 += q * q;
        }
        const double lp = 1.0 / (1.0 + pow(sqrt(r2), 2.0 * order));
        const float w = (float)(high_pass ? 1.0 - lp : lp);
        float2_ v = X[e];
        v.x = __fmul_rn(v.x, w);
        v.y = __fmul_rn(v.y, w);
        X[e] = v;
    }
}

// ---- phase correlation (register/phase.rs) ---------------------------------

// R = A * conj(B), optionally divided by |R| where |R| > eps (0 elsewhere):
// cross_power_spectrum_kernel, register/kernels/phase.rs:10-44, f32.
__global__ void cross_power_kernel(const float2_ *__restrict__ A, const float2_ *__restrict__ B, float2_ *__restrict__ R,
                                   uint32_t n, int normalize, float eps) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float2_ a = A[e], b = B[e];
        float re = __fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
        float im = __fsub_rn(__fmul_rn(a.y, b.x), __fmul_rn(a.x, b.y));
        if (normalize) {
            const float mag = __fsqrt_rn(__fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)));
            const float sc = mag > eps ? __fdiv_rn(1.0f, mag) : 0.0f;
            re = __fmul_rn(re, sc);
            im = __fmul_rn(im, sc);
        }
        R[e] = float2_{re, im};
    }
}

// Stage 1 of the argmax of |cc|^2 (f32 re*re + im*im, first index on ties).
__global__ void argmax_mag2_kernel(const float2_ *__restrict__ X, uint32_t n, float *__restrict__ pv,
                                   uint32_t *__restrict__ pi) {
    __shared__ float sv[kRedThreads];
    __shared__ uint32_t si[kRedThreads];
    float best = -1.0f;
    uint32_t bi = 0xffffffffu;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float2_ v = X[e];
        const float m = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
        if (m > best) {  // e grows along the loop: the first index wins ties
            best = m;
            bi = e;
        }
    }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const float v2 = sv[threadIdx.x + o];
            const uint32_t i2 = si[threadIdx.x + o];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 < si[threadIdx.x])) {
                sv[threadIdx.x] = v2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pv[blockIdx.x] = sv[0];
        pi[blockIdx.x] = si[0];
    }
}

// Stage 2: the winner over the blocks; the integer shift and the peak value.
__global__ void argmax_final_kernel(const float *__restrict__ pv, const uint32_t *__restrict__ pi, int nb,
                                    const float2_ *__restrict__ X, const SpecAxes a, PcState *st) {
    if (threadIdx.x != 0) return;
    float best = -1.0f;
    uint32_t bi = 0;
    for (int b = 0; b < nb; ++b) {
        if (pi[b] == 0xffffffffu) continue;
        if (pv[b] > best || (pv[b] == best && pi[b] < bi)) {
            best = pv[b];
            bi = pi[b];
        }
    }
    st->max_idx = bi;
    for (int d = 0; d < a.ndim; ++d) {
        const int64_t k = (bi / a.inner[d]) % a.len[d];
        st->shift[d] = k <= a.len[d] / 2 ? (double)k : (double)(k - a.len[d]);
    }
    st->peak_re = (double)X[bi].x;
    st->peak_im = (double)X[bi].y;
}

// The phase of every bin from the axes other than `ax` at the current
// shift: angle = 2 pi sum_{d != ax} f_d[k_d] shift_d (phase.rs:169-181).
__global__ void pc_other_phase_kernel(double2 *__restrict__ oth, uint32_t n, const SpecAxes a, int ax,
                                      const PcState *__restrict__ st) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        double ang = 0.0;
        for (int d = 0; d < a.ndim; ++d) {
            if (d == ax) continue;
            const uint32_t k = (e / a.inner[d]) % a.len[d];
            ang += kTwoPi * freq_of(k, a.len[d]) * st->shift[d];
        }
        double s, c;
        sincos(ang, &s, &c);
        oth[e] = make_double2(c, s);
    }
}

// The axis's phase per candidate: cos / sin of 2 pi f_ax[k] s_m with
// s_m = shift[ax] + (m - radius) step (phase.rs:183-191).
__global__ void pc_axis_phase_kernel(double2 *__restrict__ axt, int len, int ncand, int radius, double step, int ax,
                                     const PcState *__restrict__ st) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= len * ncand) return;
    const int m = i / len, k = i - m * len;
    const double cs = st->shift[ax] + (double)(m - radius) * step;
    double s, c;
    sincos(kTwoPi * freq_of(k, len) * cs, &s, &c);
    axt[i] = make_double2(c, s);
}

// Candidate sums sum_e R[e] e^{i (other[e] + axis_m[k_ax(e)])}, candidate m =
// blockIdx.y, partial per block (phase.rs:193-209).
__global__ void pc_candidate_kernel(const float2_ *__restrict__ R, const double2 *__restrict__ oth,
                                    const double2 *__restrict__ axt, uint32_t n, uint32_t inner, uint32_t len,
                                    double2 *__restrict__ part) {
    __shared__ double sh[32];
    const double2 *at = axt + (size_t)blockIdx.y * len;
    double sr = 0.0, si = 0.0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double2 o = oth[e], w = at[(e / inner) % len];
        const double c = o.x * w.x - o.y * w.y, s = o.y * w.x + o.x * w.y;
        const double r = (double)R[e].x, m = (double)R[e].y;
        sr += r * c - m * s;
        si += r * s + m * c;
    }
    sr = block_sum(sr, sh);
    si = block_sum(si, sh);
    if (threadIdx.x == 0) part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = make_double2(sr, si);
}

// The best candidate (first strict maximum of |sum / n|^2, candidates in
// order), written back to the shift and the peak (phase.rs:210-222).
__global__ void pc_select_kernel(const double2 *__restrict__ part, int nb, int ncand, int radius, double step, int ax,
                                 double n_total, PcState *st) {
    if (threadIdx.x != 0) return;
    const double center = st->shift[ax];
    double best = -1.0, bs = center, br = st->peak_re, bim = st->peak_im;
    for (int m = 0; m < ncand; ++m) {
        double sr = 0.0, si = 0.0;
        for (int b = 0; b < nb; ++b) {
            sr += part[(size_t)m * nb + b].x;
            si += part[(size_t)m * nb + b].y;
        }
        sr /= n_total;
        si /= n_total;
        const double mag2 = sr * sr + si * si;
        if (mag2 > best) {
            best = mag2;
            bs = center + (double)(m - radius) * step;
            br = sr;
            bim = si;
        }
    }
    st->shift[ax] = bs;
    st->peak_re = br;
    st->peak_im = bim;
}

// Partials of the registration error's terms: sum ref^2, sum mov^2 and the
// unnormalised cross-correlation (A conj(B), inverse DFT scaled by 1/n) at
// the peak bin, the phase reduced exactly per axis as (k_d m_d) mod N_d.
__global__ void pc_error_kernel(const float *__restrict__ ref, const float *__restrict__ mov,
                                const float2_ *__restrict__ A, const float2_ *__restrict__ B, uint32_t n, const SpecAxes a,
                                const PcState *__restrict__ st, int want_cc, double *__restrict__ part) {
    __shared__ double sh[32];
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const uint32_t mi = st->max_idx;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double x = ref[e], y = mov[e];
        s0 += x * x;
        s1 += y * y;
        if (want_cc) {
            // A * conj(B) in f32 as complex_mul_into(.., conj = true).
            const float2_ av = A[e], bv = B[e];
            const float bi = -bv.y;
            const float ur = __fsub_rn(__fmul_rn(av.x, bv.x), __fmul_rn(av.y, bi));
            const float ui = __fadd_rn(__fmul_rn(av.x, bi), __fmul_rn(av.y, bv.x));
            double ang = 0.0;
            for (int d = 0; d < a.ndim; ++d) {
                const uint64_t k = (e / a.inner[d]) % a.len[d], m = (mi / a.inner[d]) % a.len[d];
                ang += (double)((k * m) % (uint64_t)a.len[d]) / (double)a.len[d];
            }
            double sn, cs;
            sincospi(2.0 * ang, &sn, &cs);
            s2 += (double)ur * cs - (double)ui * sn;
            s3 += (double)ur * sn + (double)ui * cs;
        }
    }
    s0 = block_sum(s0, sh);
    s1 = block_sum(s1, sh);
    s2 = block_sum(s2, sh);
    s3 = block_sum(s3, sh);
    if (threadIdx.x == 0) {
        double *p = part + 4 * (size_t)blockIdx.x;
        p[0] = s0; p[1] = s1; p[2] = s2; p[3] = s3;
    }
}

__global__ void sum_partials_kernel(const double *__restrict__ part, int nb, int width, double *__restrict__ out) {
    const int j = threadIdx.x;
    if (j >= width) return;
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(size_t)b * width + j];
    out[j] = s;
}

// ---- unsupervised Wiener (restore/deconvolve.rs:357-509) --------------------

// Per bin, f32 as the reference's complex_mul_into(.., conj = true) calls:
// P = (Re conj(H) Y, Im conj(H) Y, |H|^2, |L|^2).
__global__ void uw_prep_kernel(const float2_ *__restrict__ Y, const float2_ *__restrict__ H,
                               const float2_ *__restrict__ L, float4 *__restrict__ P, uint32_t n) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float2_ y = Y[e], h = H[e], l = L[e];
        const float hi = -h.y, li = -l.y;
        const float hyr = __fsub_rn(__fmul_rn(y.x, h.x), __fmul_rn(y.y, hi));
        const float hyi = __fadd_rn(__fmul_rn(y.x, hi), __fmul_rn(y.y, h.x));
        const float hm2 = __fsub_rn(__fmul_rn(h.x, h.x), __fmul_rn(h.y, hi));
        const float lm2 = __fsub_rn(__fmul_rn(l.x, l.x), __fmul_rn(l.y, li));
        P[e] = make_float4(hyr, hyi, hm2, lm2);
    }
}

// One iteration's sums at the current balance (rss, reg, trace; FP64), and
// the posterior mean's running sums after the burn-in.
__global__ void uw_iter_kernel(const float2_ *__restrict__ Y, const float2_ *__restrict__ H,
                               const float4 *__restrict__ P, uint32_t n, const UwState *__restrict__ st, int accumulate,
                               double2 *__restrict__ mean, double *__restrict__ part) {
    __shared__ double sh[32];
    const double bal = st->balance, nn = (double)n;
    double rss = 0.0, reg = 0.0, tr = 0.0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float4 q = P[e];
        const float2_ y = Y[e], h = H[e];
        const double hm2 = q.z, lm2 = q.w;
        const double denom = fmax(hm2 + bal * lm2, 1.0e-12);
        const double xr = (double)q.x / denom, xi = (double)q.y / denom;
        const double hr = h.x, hi = h.y;
        const double hxr = hr * xr - hi * xi, hxi = hr * xi + hi * xr;
        const double dr = (double)y.x - hxr, di = (double)y.y - hxi;
        rss += (dr * dr + di * di) / nn;
        reg += lm2 * ((xr * xr + xi * xi) / nn);
        tr += hm2 / denom;
        if (accumulate) {
            double2 m = mean[e];
            m.x += xr;
            m.y += xi;
            mean[e] = m;
        }
    }
    rss = block_sum(rss, sh);
    reg = block_sum(reg, sh);
    tr = block_sum(tr, sh);
    if (threadIdx.x == 0) {
        double *p = part + 3 * (size_t)blockIdx.x;
        p[0] = rss; p[1] = reg; p[2] = tr;
    }
}

// Balance update of iteration `it` (deconvolve.rs:470-482): the sums over the
// blocks in fixed order, the empirical-Bayes variances, the PCG jitter.
__global__ void uw_update_kernel(const double *__restrict__ part, int nb, uint32_t n, UwState *st, double *chain,
                                 int it) {
    if (threadIdx.x != 0) return;
    double rss = 0.0, reg = 0.0, tr = 0.0;
    for (int b = 0; b < nb; ++b) {
        rss += part[3 * (size_t)b];
        reg += part[3 * (size_t)b + 1];
        tr += part[3 * (size_t)b + 2];
    }
    const double nn = (double)n;
    const double eff_dof = fmax(nn - tr, 1.0);
    const double sigma_n2 = fmax(rss / eff_dof, 1.0e-8 * fmax(st->img_var, 1.0e-6));
    const double sigma_x2 = fmax(reg / fmax(tr, 1.0), 1.0e-8);
    st->rng = st->rng * 6364136223846793005ull + 1ull;
    const double u = (double)(st->rng >> 33) / (double)(1ull << 31) - 0.5;
    const double jitter = exp(u * (2.0 / sqrt(nn)));
    const double b = fmin(fmax(sigma_n2 / sigma_x2 * jitter, 1.0e-6), 1.0e3);
    st->balance = b;
    chain[it] = b;
}

// Posterior mean -> f32 spectrum (the reference scales in f64, then casts).
__global__ void uw_mean_kernel(const double2 *__restrict__ mean, uint32_t n, double inv_count,
                               float2_ *__restrict__ X) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double2 m = mean[e];
        X[e] = float2_{(float)(m.x * inv_count), (float)(m.y * inv_count)};
    }
}

// Sum and sum of squares of a real array (FP64 partials).
__global__ void sum_sq_kernel(const float *__restrict__ x, uint32_t n, double *__restrict__ part) {
    __shared__ double sh[32];
    double s = 0.0, q = 0.0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const double v = x[e];
        s += v;
        q += v * v;
    }
    s = block_sum(s, sh);
    q = block_sum(q, sh);
    if (threadIdx.x == 0) {
        part[2 * (size_t)blockIdx.x] = s;
        part[2 * (size_t)blockIdx.x + 1] = q;
    }
}

__global__ void uw_init_kernel(const double *__restrict__ sums, uint32_t n, uint64_t seed, UwState *st) {
    if (threadIdx.x != 0) return;
    const double mean = sums[0] / (double)n;
    st->img_var = fmax(sums[1] / (double)n - mean * mean, 0.0);
    st->balance = 0.05;
    st->rng = seed + 0x9E3779B97F4A7C15ull;
}

}  // namespace

int launch_spectral_axes(float *re, float *im, int64_t n, const float *tab, const SpecAxes &a, void *stream) {
    if (n <= 0) return 0;
    const int threads = 256;
    const int64_t blocks = (n + threads - 1) / threads;
    spectral_axes_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), threads, 0, (cudaStream_t)stream>>>(
        re, im, (uint32_t)n, tab, a);
    return (int)cudaGetLastError();
}

int launch_butterworth(float2_ *X, int64_t n, const SpecAxes &a, double cutoff, double order, int high_pass,
                       void *stream) {
    if (n <= 0) return 0;
    const int threads = 256;
    const int64_t blocks = (n + threads - 1) / threads;
    butterworth_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), threads, 0, (cudaStream_t)stream>>>(
        X, (uint32_t)n, a, cutoff, order, high_pass);
    return (int)cudaGetLastError();
}

namespace {
inline unsigned red_blocks(int64_t n) {
    const int64_t b = (n + kRedThreads - 1) / kRedThreads;
    return (unsigned)(b < kRedBlocks ? (b < 1 ? 1 : b) : kRedBlocks);
}
}  // namespace

int launch_phase_cross_power(const float2_ *A, const float2_ *B, float2_ *R, int64_t n, int normalize, void *stream) {
    cross_power_kernel<<<red_blocks(n), kRedThreads, 0, (cudaStream_t)stream>>>(A, B, R, (uint32_t)n, normalize,
                                                                                1.0e-12f);
    return (int)cudaGetLastError();
}

int launch_phase_argmax(const float2_ *X, int64_t n, const SpecAxes &a, float *pv, uint32_t *pi, PcState *st,
                        void *stream) {
    const unsigned nb = red_blocks(n);
    argmax_mag2_kernel<<<nb, kRedThreads, 0, (cudaStream_t)stream>>>(X, (uint32_t)n, pv, pi);
    argmax_final_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(pv, pi, (int)nb, X, a, st);
    return (int)cudaGetLastError();
}

int launch_phase_refine_axis(const float2_ *R, int64_t n, const SpecAxes &a, int ax, int radius, double step,
                             double2 *oth, double2 *axt, double2 *part, PcState *st, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int ncand = 2 * radius + 1, len = (int)a.len[ax];
    pc_other_phase_kernel<<<red_blocks(n), kRedThreads, 0, s>>>(oth, (uint32_t)n, a, ax, st);
    pc_axis_phase_kernel<<<(len * ncand + 255) / 256, 256, 0, s>>>(axt, len, ncand, radius, step, ax, st);
    const unsigned nb = red_blocks(n) < kCandBlocks ? red_blocks(n) : kCandBlocks;
    pc_candidate_kernel<<<dim3(nb, ncand), kRedThreads, 0, s>>>(R, oth, axt, (uint32_t)n, (uint32_t)a.inner[ax],
                                                                (uint32_t)len, part);
    pc_select_kernel<<<1, 32, 0, s>>>(part, (int)nb, ncand, radius, step, ax, (double)n, st);
    return (int)cudaGetLastError();
}

int launch_phase_error_terms(const float *ref, const float *mov, const float2_ *A, const float2_ *B, int64_t n,
                             const SpecAxes &a, const PcState *st, int want_cc, double *part, double *out,
                             void *stream) {
    const unsigned nb = red_blocks(n);
    pc_error_kernel<<<nb, kRedThreads, 0, (cudaStream_t)stream>>>(ref, mov, A, B, (uint32_t)n, a, st, want_cc, part);
    sum_partials_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(part, (int)nb, 4, out);
    return (int)cudaGetLastError();
}

int launch_uw_setup(const float *in, const float2_ *Y, const float2_ *H, const float2_ *L, float4_ *P, int64_t n,
                    uint64_t seed, double *part, UwState *st, double2 *mean, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = red_blocks(n);
    uw_prep_kernel<<<nb, kRedThreads, 0, s>>>(Y, H, L, reinterpret_cast<float4 *>(P), (uint32_t)n);
    sum_sq_kernel<<<nb, kRedThreads, 0, s>>>(in, (uint32_t)n, part);
    sum_partials_kernel<<<1, 32, 0, s>>>(part, (int)nb, 2, part + 2 * kRedBlocks);
    uw_init_kernel<<<1, 32, 0, s>>>(part + 2 * kRedBlocks, (uint32_t)n, seed, st);
    cudaMemsetAsync(mean, 0, (size_t)n * sizeof(double2), s);
    return (int)cudaGetLastError();
}

int launch_uw_iteration(const float2_ *Y, const float2_ *H, const float4_ *P, int64_t n, int accumulate,
                        double2 *mean, double *part, UwState *st, double *chain, int it, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = red_blocks(n);
    uw_iter_kernel<<<nb, kRedThreads, 0, s>>>(Y, H, reinterpret_cast<const float4 *>(P), (uint32_t)n, st, accumulate,
                                              mean, part);
    uw_update_kernel<<<1, 32, 0, s>>>(part, (int)nb, (uint32_t)n, st, chain, it);
    return (int)cudaGetLastError();
}

int launch_uw_mean(const double2 *mean, int64_t n, double inv_count, float2_ *X, void *stream) {
    uw_mean_kernel<<<red_blocks(n), kRedThreads, 0, (cudaStream_t)stream>>>(mean, (uint32_t)n, inv_count, X);
    return (int)cudaGetLastError();
}

}  // namespace lucem
