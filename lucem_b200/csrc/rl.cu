// rl.cu -- Richardson-Lucy deconvolution on FFT convolution, sm_100a.
//
// Reference: richardson_lucy_into (crates/lucem-ops/src/restore/deconvolve.rs
// :45-149) runs per iteration
//   est_conv = correlate_2d(est, flipped psf)        (a convolution)
//   rel_blur = obs / (|est_conv| < eps ? eps : est_conv)   (rl_div_clamp_kernel,
//              restore/kernels/deconvolve.rs:8-22)
//   err_est  = correlate_2d(rel_blur, psf)           (the adjoint)
//   est      = est * err_est  (+ clip on the last iteration, rl_mul_clamp_kernel
//              restore/kernels/deconvolve.rs:27-43)
// with direct spatial correlations.  Here both correlations are products with
// the PSF's transfer function on an FFT grid (Pz, Py, Px).  The pad mode is
// honoured by extending each array by h = k/2 samples per axis with the
// reference's pad map (zero padding == PadMode::Constant needs no extension),
// which makes the linear correlation on the extended array equal to the
// reference's padded correlation on the image.
//
// Data flow per iteration (3-D; 2-D drops the z pass and fuses the
// transfer-function product into its y pass):
//   row pass   : C2R(x) -> ratio epilogue -> x extension -> R2C(x)    [s1]
//   y forward  : rows pad(j - hy) of s1 -> FFT(y) -> s2
//   z pass     : planes pad(j - hz) of s2 -> FFT(z) -> * H -> IFFT(z) -> s2
//   y inverse  : s2 -> IFFT(y) -> rows [hy, hy+Y) -> s1
//   row pass   : C2R(x) -> update epilogue (est *= corr) -> R2C(x)     [s1]
//   ... same three column passes with conj(H) ...
// The real-to-complex transforms pack the real row into Px/2 complex samples
// (x[2m] + i x[2m+1]) and split / merge the half spectrum around that
// transform.  The transfer functions carry the 1/(Pz*Py*Px) normalisation.

#include <cuda_runtime.h>

#include <cstdint>

#include "rl_pass.cuh"

namespace lucem {

using namespace rlp;

namespace {

// Generic column pass (any 2/3/5/7-smooth length): self-sorting transform in
// shared memory, two buffers, natural order in and out.
__global__ void __launch_bounds__(512, 1) col_pass_kernel(const __grid_constant__ ColPass p) {
    extern __shared__ float4 smem4[];
    const int n = p.plan.n;
    float2 *tws = reinterpret_cast<float2 *>(smem4);
    float2 *bufA = tws + n;
    float2 *bufB = bufA + n * p.CP;
    const int C = p.C, CP = p.CP, T = blockDim.x, tid = threadIdx.x;
    for (int i = tid; i < n; i += T) tws[i] = p.tw[i];
    const fft::Tw tw{tws, 1};
    const int ntiles = p.items ? p.total_tiles : (p.ncols + C - 1) / C;
    for (int gt = blockIdx.x; gt < ntiles; gt += gridDim.x) {
        int tile;
        const ColItem q = col_tile(p, gt, &tile);
        const int c0 = tile * C;
        for (int it = tid; it < n * C; it += T) {
            int row = it / C, c = it - row * C;
            int col = c0 + c;
            float2 val = make_float2(0.f, 0.f);
            if (col < q.ncols) {
                int outer = col / q.Hx, kx = col - outer * q.Hx;
                const ColOffsets off = col_offsets(p, q, outer);
                int srow;
                if (p.mode == kColInv) srow = row;
                else if (p.pad_mode == LUCEM_PAD_CONSTANT)  // zero padding: a range check, no pad map
                    srow = (unsigned)(row - q.halo) < (unsigned)q.n_img ? row - q.halo : -1;
                else srow = row < q.n_img + 2 * q.halo ? pad_index_rt(row - q.halo, q.n_img, p.pad_mode) : -1;
                if (srow >= 0) val = q.src[off.src + srow * q.src_row + kx];
            }
            bufA[row * CP + c] = val;
        }
        __syncthreads();
        float2 *buf = fft::stockham(bufA, bufB, n, C, CP, p.plan.radix, p.plan.nstages, tw, p.mode == kColInv);
        if (p.mode == kColFull) {
            for (int it = tid; it < n * C; it += T) {
                int row = it / C, c = it - row * C;
                int col = c0 + c;
                if (col < q.ncols) {
                    int outer = col / q.Hx, kx = col - outer * q.Hx;
                    const ColOffsets off = col_offsets(p, q, outer);
                    if (q.spec_out) q.spec_out[off.spec + row * p.spec_row + kx] = buf[row * CP + c];
                    float2 h = q.H ? q.H[off.h + row * q.h_row + kx] : make_float2(1.f, 0.f);
                    if (p.Hrow) h = cmul(h, p.Hrow[row]);
                    if (p.conj_h) h.y = -h.y;
                    buf[row * CP + c] = cmul(buf[row * CP + c], h);
                }
            }
            __syncthreads();
            buf = fft::stockham(buf, buf == bufA ? bufB : bufA, n, C, CP, p.plan.radix, p.plan.nstages, tw, true);
        }
        const int rows = p.mode == kColFwd ? n : q.store_count;
        const int r0 = p.mode == kColFwd ? 0 : q.store_begin;
        for (int it = tid; it < rows * C; it += T) {
            int row = it / C, c = it - row * C;
            int col = c0 + c;
            if (col < q.ncols) {
                int outer = col / q.Hx, kx = col - outer * q.Hx;
                q.dst[col_offsets(p, q, outer).dst + row * q.dst_row + kx] = buf[(r0 + row) * CP + c];
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(512, 1) row_pass_kernel(const __grid_constant__ RowPass p) {
    extern __shared__ float4 smem4[];
    const int Px = p.Px, M = p.M;
    const int C = p.C, CP = p.CP, T = blockDim.x, tid = threadIdx.x;
    float2 *tws = reinterpret_cast<float2 *>(smem4);
    float2 *bufA = tws + Px;
    float2 *bufB = bufA + (M + 1) * CP;
    for (int i = tid; i < Px; i += T) tws[i] = p.tw[i];
    const fft::Tw twM{tws, 2};   // W_M^m = W_Px^{2m}
    const int ntiles = p.items ? p.total_tiles : (p.nrows + C - 1) / C;
    for (int gt = blockIdx.x; gt < ntiles; gt += gridDim.x) {
        int tile;
        const RowItem pi = row_tile(p, gt, &tile);
        const int row0 = tile * C;
        float2 *buf = bufA;  // holds the natural-order real row after C2R
        __syncthreads();
        if (p.kind != kRowInit && p.kind != kRowRealIn) {
            // Half spectrum X[0..M] of each row (lanes along k: coalesced).
            for (int it = tid; it < (M + 1) * C; it += T) {
                int c = it / (M + 1), k = it - c * (M + 1);
                int row = row0 + c;
                float2 v = make_float2(0.f, 0.f);
                if (row < pi.nrows) v = pi.s1[(int64_t)row * p.Hp + k];
                bufA[k * CP + c] = v;
            }
            __syncthreads();
            // Merge the half spectrum into the packed M-point spectrum:
            // Z[k] = (X[k] + X*[M-k]) + i (X[k] - X*[M-k]) W_Px^{-k}.
            for (int it = tid; it < (M / 2 + 1) * C; it += T) {
                int k = it / C, c = it - k * C;
                float2 xk = bufA[k * CP + c], xm = bufA[(M - k) * CP + c];
                float2 xmc = make_float2(xm.x, -xm.y), xkc = make_float2(xk.x, -xk.y);
                float2 wk = tws[k];
                wk.y = -wk.y;  // W^{-k}
                float2 e = cadd(xk, xmc), d = cmul(csub(xk, xmc), wk);
                float2 zk = make_float2(e.x - d.y, e.y + d.x);
                if (k != 0 && 2 * k != M) {
                    float2 wm = tws[M - k];
                    wm.y = -wm.y;
                    float2 e2 = cadd(xm, xkc), d2 = cmul(csub(xm, xkc), wm);
                    bufA[(M - k) * CP + c] = make_float2(e2.x - d2.y, e2.y + d2.x);
                }
                bufA[k * CP + c] = zk;
            }
            __syncthreads();
            buf = fft::stockham(bufA, bufB, M, C, CP, p.plan.radix, p.plan.nstages, twM, true);
        }
        float *bufr = reinterpret_cast<float *>(buf);
        // Epilogue on the image columns; the real sample at position i of the
        // row is component (i & 1) of packed element i >> 1.
        const bool emit = !(p.kind == kRowUpdate && p.last) && p.kind != kRowRealOut && p.kind != kRowEbar;
        for (int it = tid; it < pi.X * C; it += T) {
            int c = it / pi.X, xi = it - c * pi.X;
            int row = row0 + c;
            if (row >= pi.nrows) continue;
            int i = xi + pi.hx;
            float *slot = bufr + ((i >> 1) * CP + c) * 2 + (i & 1);
            int64_t g = (int64_t)row * pi.X + xi;
            float v;
            if (p.kind == kRowInit) {
                v = 0.5f;
            } else if (p.kind == kRowRealIn) {
                v = pi.obs[g];
            } else if (p.kind == kRowRealOut) {
                v = *slot;
                pi.est[g] = v;
            } else if (p.kind == kRowRatio || p.kind == kRowRatioKeep) {
                float conv = *slot;
                float d = fabsf(conv) < p.eps ? p.eps : conv;
                v = pi.obs[g] / d;
                if (p.kind == kRowRatioKeep) pi.est[g] = conv;
            } else if (p.kind == kRowCbar) {
                const float rb = *slot, ci = p.aux[g];
                const bool gd = fabsf(ci) < p.eps;
                const float d = gd ? p.eps : ci;
                v = gd ? 0.0f : -rb * pi.obs[g] / (d * d);
                if (p.aux2) p.aux2[g] += rb / d;
            } else if (p.kind == kRowAbar) {
                pi.est[g] = *slot;
                v = p.aux[g] * pi.obs[g];
            } else if (p.kind == kRowEbar) {
                v = fmaf(p.aux2[g], p.aux[g], *slot);
                p.aux2[g] = v;
            } else {
                float corr = *slot;
                float old = p.est_first ? 0.5f : pi.est[g];
                v = old * corr;
                if (p.last && p.clip) v = fminf(fmaxf(v, -1.0f), 1.0f);
                pi.est[g] = v;
            }
            if (emit) *slot = v;
        }
        if (!emit) continue;
        __syncthreads();
        // Extension along x: positions [0, hx) and [hx+X, hx+X+hx) take the
        // pad-mapped image samples, everything past X + 2*hx is zero.
        for (int it = tid; it < Px * C; it += T) {
            int c = it / Px, j = it - c * Px;
            if (j >= pi.hx && j < pi.hx + pi.X) continue;
            float v = 0.0f;
            if (j < pi.X + 2 * pi.hx) {
                int q = pad_index_rt(j - pi.hx, pi.X, p.pad_mode);
                if (q >= 0) {
                    int s = q + pi.hx;
                    v = bufr[((s >> 1) * CP + c) * 2 + (s & 1)];
                }
            }
            bufr[((j >> 1) * CP + c) * 2 + (j & 1)] = v;
        }
        __syncthreads();
        float2 *other = buf == bufA ? bufB : bufA;
        float2 *z = fft::stockham(buf, other, M, C, CP, p.plan.radix, p.plan.nstages, twM, false);
        // Split the packed spectrum into the half spectrum:
        // X[k] = 1/2 (Z[k] + Z*[M-k]) - i/2 W_Px^k (Z[k] - Z*[M-k]).
        for (int it = tid; it < (M / 2 + 1) * C; it += T) {
            int k = it / C, c = it - k * C;
            float2 zk = z[k * CP + c];
            float2 zm = z[((M - k) % M) * CP + c];
            float2 zmc = make_float2(zm.x, -zm.y), zkc = make_float2(zk.x, -zk.y);
            float2 e = cadd(zk, zmc), d = cmul(csub(zk, zmc), tws[k]);
            float2 xk = make_float2(0.5f * (e.x + d.y), 0.5f * (e.y - d.x));
            float2 e2 = cadd(zm, zkc), d2 = cmul(csub(zm, zkc), tws[M - k]);
            float2 xm = make_float2(0.5f * (e2.x + d2.y), 0.5f * (e2.y - d2.x));
            z[k * CP + c] = xk;
            if (2 * k != M) z[(M - k) * CP + c] = xm;
        }
        __syncthreads();
        for (int it = tid; it < (M + 1) * C; it += T) {
            int c = it / (M + 1), k = it - c * (M + 1);
            int row = row0 + c;
            if (row < pi.nrows) pi.s1[(int64_t)row * p.Hp + k] = z[k * CP + c];
        }
    }
}

// ---- transfer function (FP64, direct small-support DFT per axis) ----------

// A[z][y][kx] = sum_x psf[z][y][x] e^{-2 pi i kx (x - cx) / Px}
__global__ void otf_x_kernel(const double *__restrict__ psf, int kz, int ky, int kx, int cx, int Px,
                             int Hx, int Hp, const double2 *__restrict__ twd, double2 *__restrict__ A) {
    int64_t total = (int64_t)kz * ky * Hx;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int f = (int)(e % Hx);
        int64_t zy = e / Hx;
        const double *row = psf + zy * kx;
        double re = 0.0, im = 0.0;
        for (int x = 0; x < kx; ++x) {
            int m = (int)(((int64_t)f * (x - cx)) % Px);
            if (m < 0) m += Px;
            double2 w = twd[m];
            double v = row[x];
            re = fma(v, w.x, re);
            im = fma(v, w.y, im);
        }
        A[zy * Hp + f] = make_double2(re, im);
    }
}

// B[z][ky][kx] = sum_y A[z][y][kx] e^{-2 pi i ky (y - cy) / Py}
__global__ void otf_y_kernel(const double2 *__restrict__ A, int kz, int ky, int cy, int Py, int Hx,
                             int Hp, const double2 *__restrict__ twd,
                             double2 *__restrict__ B) {
    int64_t total = (int64_t)kz * Py * Hx;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int f = (int)(e % Hx);
        int64_t r = e / Hx;
        int fy = (int)(r % Py);
        int z = (int)(r / Py);
        double re = 0.0, im = 0.0;
        for (int y = 0; y < ky; ++y) {
            int m = (int)(((int64_t)fy * (y - cy)) % Py);
            if (m < 0) m += Py;
            double2 w = twd[m];
            double2 a = A[((int64_t)z * ky + y) * Hp + f];
            re += a.x * w.x - a.y * w.y;
            im += a.x * w.y + a.y * w.x;
        }
        B[((int64_t)z * Py + fy) * Hp + f] = make_double2(re, im);
    }
}

// H[kz][ky][kx] = scale * sum_z B[z][ky][kx] e^{-2 pi i kz (z - cz) / Pz}, rounded to f32
__global__ void otf_z_kernel(const double2 *__restrict__ B, int kz, int cz, int Pz, int Py, int Hx,
                             int Hp, const double2 *__restrict__ twd,
                             double scale, float2 *__restrict__ H) {
    int64_t total = (int64_t)Pz * Py * Hx;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int f = (int)(e % Hx);
        int64_t r = e / Hx;
        int fy = (int)(r % Py);
        int fz = (int)(r / Py);
        double re = 0.0, im = 0.0;
        for (int z = 0; z < kz; ++z) {
            int m = (int)(((int64_t)fz * (z - cz)) % Pz);
            if (m < 0) m += Pz;
            double2 w = twd[m];
            double2 b = B[((int64_t)z * Py + fy) * Hp + f];
            re += b.x * w.x - b.y * w.y;
            im += b.x * w.y + b.y * w.x;
        }
        H[((int64_t)fz * Py + fy) * Hp + f] = make_float2((float)(re * scale), (float)(im * scale));
    }
}

}  // namespace

// Columns per tile of the column pass for transform length n (the launch
// shapes of launch_col below).
int col_tile_width(int n) {
    switch (n) {
    case 64: case 128: case 256: case 512: return 16;
    case 1024: case 2048: return 8;
    default: break;
    }
    // Generic: two (n x (C+1)) buffers plus twiddles within ~200 KB.
    int C = 64;
    while (C > 2 && ((size_t)n * (1 + 2 * (size_t)(C + 1))) * sizeof(float2) > 200 * 1024) C >>= 1;
    return C;
}

// Rows per tile of the row pass for packed length M = Px / 2.
int row_tile_rows(int M) {
    switch (M) {
    case 64: case 128: return 32;
    case 256: case 512: return 16;
    case 1024: return 8;
    default: break;
    }
    // Two (M+1) x (C+1) buffers plus the twiddles, about 100 KB at most.
    int C = 16;
    while (C > 2 && ((size_t)2 * M + 2 * (size_t)(M + 1) * (C + 1)) * sizeof(float2) > 110 * 1024) C >>= 1;
    return C;
}

namespace {

int launch_col(ColPass p, cudaStream_t s) {
    switch (p.plan.n) {
    case 64: case 128: case 256: return launch_col_64_256(p.plan.n, p, s);
    case 512: return launch_col_512(p, s);
    case 1024: return launch_col_1024(p, s);
    case 2048: return launch_col_2048(p, s);
    default: break;
    }
    const int C = col_tile_width(p.plan.n);
    int T = (int)(((int64_t)p.plan.n * C / 8 + 31) / 32) * 32;
    T = T < 128 ? 128 : (T > 512 ? 512 : T);
    p.C = C;
    p.CP = C + 1;
    size_t smem = ((size_t)p.plan.n + 2 * (size_t)p.plan.n * p.CP) * sizeof(float2);
    int ntiles = p.items ? p.total_tiles : (p.ncols + C - 1) / C;
    int per_sm = (int)((227 * 1024) / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    int grid = ntiles < sms() * per_sm ? ntiles : sms() * per_sm;
    cudaFuncSetAttribute(col_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    col_pass_kernel<<<grid, T, smem, s>>>(p);
    return (int)cudaGetLastError();
}

int launch_row(RowPass p, cudaStream_t s) {
    switch (p.M) {
    case 64: case 128: case 256: return launch_row_64_256(p.M, p, s);
    case 512: return launch_row_512(p, s);
    case 1024: return launch_row_1024(p, s);
    default: break;
    }
    const int M = p.M;
    const int C = row_tile_rows(M);
    int T = (int)(((int64_t)M * C / 8 + 31) / 32) * 32;
    if (T < 128) T = 128;
    if (T > 512) T = 512;
    p.C = C;
    p.CP = C + 1;
    size_t smem = ((size_t)p.Px + 2 * (size_t)(M + 1) * p.CP) * sizeof(float2);
    int ntiles = p.items ? p.total_tiles : (p.nrows + C - 1) / C;
    int per_sm = (int)((227 * 1024) / (smem + 1024));
    if (per_sm < 1) per_sm = 1;
    int grid = ntiles < sms() * per_sm ? ntiles : sms() * per_sm;
    cudaFuncSetAttribute(row_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    row_pass_kernel<<<grid, T, smem, s>>>(p);
    return (int)cudaGetLastError();
}

}  // namespace

// Radix plan: 8s first, then 4, 2, 3, 5, 7.
bool fft_make_plan(int64_t n, FftPlan *plan) {
    plan->n = (int32_t)n;
    plan->nstages = 0;
    int64_t m = n;
    const int order[] = {8, 4, 2, 3, 5, 7};
    for (int r : order) {
        while (m % r == 0 && plan->nstages < kFftMaxStages) {
            plan->radix[plan->nstages++] = r;
            m /= r;
        }
    }
    return m == 1 && n >= 1;
}

int64_t fft_good_length(int64_t n, bool even) {
    if (n < 1) n = 1;
    for (int64_t m = n;; ++m) {
        if (even && (m & 1)) continue;
        int64_t r = m;
        for (int f : {2, 3, 5, 7})
            while (r % f == 0) r /= f;
        if (r == 1) return m;
    }
}

namespace {

// Builds and launches the passes of one problem geometry.
struct RlRunner {
    const RlGeom &g;
    const RlBuffers &b;
    cudaStream_t s;
    void *stream;
    PassTimer *timer;
    RowPass rp{};
    FftPlan py_plan{}, pz_plan{};
    int nb = 1;  // volumes sharing the PSF (RlGeom::nb)
    bool ok = true;

    RlRunner(const RlGeom &g_, const RlBuffers &b_, void *stream_, PassTimer *timer_)
        : g(g_), b(b_), s(static_cast<cudaStream_t>(stream_)), stream(stream_), timer(timer_) {
        nb = g.nb > 1 ? g.nb : 1;
        rp.nrows = nb * g.Z * g.Y;
        rp.X = g.X;
        rp.Px = g.Px;
        rp.M = g.Px / 2;
        rp.Hx = g.Hx;
        rp.Hp = g.Hp;
        rp.hx = g.hx;
        rp.pad_mode = g.mode;
        rp.s1 = static_cast<float2 *>(b.s1);
        rp.tw = reinterpret_cast<const float2 *>(b.tw_x);
        ok = fft_make_plan(rp.M, &rp.plan) && fft_make_plan(g.Py, &py_plan) &&
             (g.ndim != 3 || fft_make_plan(g.Pz, &pz_plan));
    }

    int col(const ColPass &c, int kind = -1) {
        if (kind < 0) kind = c.mode == kColFwd ? kPassRlColFwd : (c.mode == kColFull ? kPassRlColFull : kPassRlColInv);
        if (timer) timer->begin(kind, stream);
        int e = launch_col(c, s);
        if (timer) timer->end(kind, stream);
        return e;
    }

    int row(int kind, const float *in_real, float *out_real, int est_first, int last, int clip, float eps,
            const float *aux = nullptr, float *aux2 = nullptr) {
        RowPass r = rp;
        r.kind = kind;
        r.obs = in_real;
        r.est = out_real;
        r.aux = aux;
        r.aux2 = aux2;
        r.est_first = est_first;
        r.last = last;
        r.clip = clip;
        r.eps = eps;
        if (timer) timer->begin(kPassRlRow, stream);
        int e = launch_row(r, s);
        if (timer) timer->end(kPassRlRow, stream);
        return e;
    }

    ColPass y_forward(float2 *dst, int64_t dst_outer) const {
        ColPass c{};
        c.ncols = nb * g.Z * g.Hx; c.Hx = g.Hx;
        c.src = static_cast<const float2 *>(b.s1); c.src_outer = (int64_t)g.Y * g.Hp; c.src_row = g.Hp;
        c.n_img = g.Y; c.halo = g.hy;
        c.dst = dst; c.dst_outer = dst_outer; c.dst_row = g.Hp;
        c.mode = kColFwd; c.pad_mode = g.mode;
        c.plan = py_plan; c.tw = reinterpret_cast<const float2 *>(b.tw_y);
        return c;
    }

    ColPass y_inverse(const float2 *src, int64_t src_outer) const {
        ColPass c{};
        c.ncols = nb * g.Z * g.Hx; c.Hx = g.Hx;
        c.src = src; c.src_outer = src_outer; c.src_row = g.Hp;
        c.n_img = g.Py; c.halo = 0;
        c.dst = static_cast<float2 *>(b.s1); c.dst_outer = (int64_t)g.Y * g.Hp; c.dst_row = g.Hp;
        c.store_begin = g.hy; c.store_count = g.Y;
        c.mode = kColInv; c.pad_mode = g.mode;
        c.plan = py_plan; c.tw = reinterpret_cast<const float2 *>(b.tw_y);
        return c;
    }

    // The column passes between the two row passes of one convolution with H
    // (or correlation with conj(H)): s1 in, s1 out.  spec_out (optional)
    // receives the full forward spectrum [Pz][Py][Hp] of the row-transformed
    // input.
    int pair(const void *H, int conj, float2 *spec_out) {
        float2 *s1 = static_cast<float2 *>(b.s1);
        float2 *s2 = static_cast<float2 *>(b.s2);
        // A separable transfer function comes with its factor along the last
        // transformed axis (z in 3-D, y in 2-D).
        const float2 *Hrow = static_cast<const float2 *>(
            H == b.h_conv ? b.hrow_conv : (H == b.h_corr ? b.hrow_corr : nullptr));
        if (g.ndim == 2) {
            ColPass c{};
            c.ncols = nb * g.Hx; c.Hx = g.Hx;
            c.src = s1; c.src_outer = 0; c.src_row = g.Hp;
            c.n_img = g.Y; c.halo = g.hy;
            c.dst = s1; c.dst_outer = 0; c.dst_row = g.Hp;
            // One column block per image: image v at v * Y * Hp, its spectrum
            // at v * Py * Hp.
            c.bdiv = 1; c.src_b = c.dst_b = (int64_t)g.Y * g.Hp; c.spec_b = (int64_t)g.Py * g.Hp;
            c.store_begin = g.hy; c.store_count = g.Y;
            c.mode = kColFull; c.pad_mode = g.mode;
            c.H = static_cast<const float2 *>(H); c.h_outer = 0; c.h_row = Hrow ? 0 : g.Hp; c.conj_h = conj;
            c.Hrow = Hrow;
            c.spec_out = spec_out;
            c.spec_row = g.Hp;
            c.plan = py_plan; c.tw = reinterpret_cast<const float2 *>(b.tw_y);
            return col(c);
        }
        int e;
        const bool hy = H == b.h_conv ? b.hy_conv != nullptr : (H == b.h_corr && b.hy_corr != nullptr);
        if (hy && spec_out == nullptr) {
            // Separable: the y and z factors commute with each other and with
            // the x transform, so the convolution is a y convolution then a z
            // convolution, each in place on s1 (the pad map of each axis
            // applied in its own loads).
            const void *fy = H == b.h_conv ? b.hy_conv : b.hy_corr;
            const void *fx = H == b.h_conv ? b.hx_conv : b.hx_corr;
            ColPass yc{};
            yc.ncols = nb * g.Z * g.Hx; yc.Hx = g.Hx;
            yc.src = s1; yc.src_outer = (int64_t)g.Y * g.Hp; yc.src_row = g.Hp;
            yc.n_img = g.Y; yc.halo = g.hy;
            yc.dst = s1; yc.dst_outer = (int64_t)g.Y * g.Hp; yc.dst_row = g.Hp;
            yc.store_begin = g.hy; yc.store_count = g.Y;
            yc.mode = kColFull; yc.pad_mode = g.mode;
            yc.H = static_cast<const float2 *>(fx); yc.h_outer = 0; yc.h_row = 0; yc.conj_h = conj;
            yc.Hrow = static_cast<const float2 *>(fy);
            yc.plan = py_plan; yc.tw = reinterpret_cast<const float2 *>(b.tw_y);
            if ((e = col(yc, kPassRlColY))) return e;
            ColPass zc{};
            zc.ncols = nb * g.Y * g.Hx; zc.Hx = g.Hx;
            zc.src = s1; zc.src_outer = g.Hp; zc.src_row = (int64_t)g.Y * g.Hp;
            zc.n_img = g.Z; zc.halo = g.hz;
            zc.dst = s1; zc.dst_outer = g.Hp; zc.dst_row = (int64_t)g.Y * g.Hp;
            zc.bdiv = g.Y; zc.src_b = zc.dst_b = (int64_t)g.Z * g.Y * g.Hp;
            zc.store_begin = g.hz; zc.store_count = g.Z;
            zc.mode = kColFull; zc.pad_mode = g.mode;
            zc.H = nullptr; zc.h_outer = 0; zc.h_row = 0; zc.conj_h = conj;
            zc.Hrow = Hrow;
            zc.plan = pz_plan; zc.tw = reinterpret_cast<const float2 *>(b.tw_z);
            return col(zc, kPassRlColZ);
        }
        if ((e = col(y_forward(s2, (int64_t)g.Py * g.Hp)))) return e;
        ColPass zp{};
        zp.ncols = nb * g.Py * g.Hx; zp.Hx = g.Hx;
        zp.src = s2; zp.src_outer = g.Hp; zp.src_row = (int64_t)g.Py * g.Hp;
        zp.n_img = g.Z; zp.halo = g.hz;
        zp.dst = s2; zp.dst_outer = g.Hp; zp.dst_row = (int64_t)g.Py * g.Hp;
        zp.bdiv = g.Py; zp.src_b = zp.dst_b = (int64_t)g.Z * g.Py * g.Hp; zp.spec_b = (int64_t)g.Pz * g.Py * g.Hp;
        zp.store_begin = g.hz; zp.store_count = g.Z;
        zp.mode = kColFull; zp.pad_mode = g.mode;
        zp.H = static_cast<const float2 *>(H); zp.h_outer = g.Hp; zp.h_row = Hrow ? 0 : (int64_t)g.Py * g.Hp;
        zp.conj_h = conj;
        zp.Hrow = Hrow;
        zp.spec_out = spec_out;
        zp.spec_row = (int64_t)g.Py * g.Hp;
        zp.plan = pz_plan; zp.tw = reinterpret_cast<const float2 *>(b.tw_z);
        if ((e = col(zp))) return e;
        return col(y_inverse(s2, (int64_t)g.Py * g.Hp));
    }

    // out = H x (conj = 0) or conj(H) x (conj = 1) on the image region.
    int apply(const void *H, int conj, const float *x, float *out, float2 *spec_out) {
        int e;
        if ((e = row(kRowRealIn, x, nullptr, 0, 0, 0, 0.f))) return e;
        if ((e = pair(H, conj, spec_out))) return e;
        return row(kRowRealOut, nullptr, out, 0, 0, 0, 0.f);
    }

    // Unnormalised inverse of a full spectrum [Pz][Py][Hp] onto the image
    // region (the geometry's Z, Y, X at offsets hz, hy, hx).
    int spectrum_to_real(const float2 *spec, float *out) {
        int e;
        if (g.ndim == 2) {
            if ((e = col(y_inverse(spec, 0)))) return e;
        } else {
            float2 *s2 = static_cast<float2 *>(b.s2);
            ColPass zi{};
            zi.ncols = g.Py * g.Hx; zi.Hx = g.Hx;
            zi.src = spec; zi.src_outer = g.Hp; zi.src_row = (int64_t)g.Py * g.Hp;
            zi.n_img = g.Pz;
            zi.dst = s2; zi.dst_outer = g.Hp; zi.dst_row = (int64_t)g.Py * g.Hp;
            zi.store_begin = g.hz; zi.store_count = g.Z;
            zi.mode = kColInv; zi.pad_mode = g.mode;
            zi.plan = pz_plan; zi.tw = reinterpret_cast<const float2 *>(b.tw_z);
            if ((e = col(zi))) return e;
            if ((e = col(y_inverse(s2, (int64_t)g.Py * g.Hp)))) return e;
        }
        return row(kRowRealOut, nullptr, out, 0, 0, 0, 0.f);
    }

    // The fused Richardson-Lucy iterations; start from `est_out`'s contents
    // when from_est, else from the constant 0.5.
    int iterations(const float *obs, float *est_out, int num_iter, int clip, float eps, bool from_est) {
        int e;
        if (from_est) e = row(kRowRealIn, est_out, nullptr, 0, 0, 0, eps);
        else e = row(kRowInit, nullptr, nullptr, 0, 0, 0, eps);
        if (e) return e;
        for (int it = 0; it < num_iter; ++it) {
            if ((e = pair(b.h_conv, 0, nullptr))) return e;
            if ((e = row(kRowRatio, obs, nullptr, 0, 0, 0, eps))) return e;
            if ((e = pair(b.h_corr, 1, nullptr))) return e;
            if ((e = row(kRowUpdate, nullptr, est_out, it == 0 && !from_est, it + 1 == num_iter, clip, eps))) return e;
        }
        return 0;
    }
};

// ---- elementwise kernels of the backward pass --------------------------

// acc += sum over nb volumes of x * conj(y) (+ u * conj(v) when u is given),
// over n complex values per volume (volumes n apart; volumes in order).
__global__ void spec_mac_kernel(float2 *__restrict__ acc, const float2 *__restrict__ x, const float2 *__restrict__ y,
                                const float2 *__restrict__ u, const float2 *__restrict__ v, int64_t n, int nb) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 a = acc[i];
        for (int b = 0; b < nb; ++b) {
            const int64_t j = i + b * n;
            const float2 p = x[j], q = y[j];
            a.x += p.x * q.x + p.y * q.y;
            a.y += p.y * q.x - p.x * q.y;
            if (u) {
                const float2 s = u[j], t = v[j];
                a.x += s.x * t.x + s.y * t.y;
                a.y += s.y * t.x - s.x * t.y;
            }
        }
        acc[i] = a;
    }
}

// out[s] = scale * full[lag(s) mod P], lag = s - centre per axis.
__global__ void gather_lags_kernel(const float *__restrict__ full, int Pz, int Py, int Px, int kz, int ky, int kx,
                                   int cz, int cy, int cx, float scale, float *__restrict__ out) {
    const int n = kz * ky * kx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int sx = i % kx, sy = (i / kx) % ky, sz = i / (kx * ky);
        const int z = ((sz - cz) % Pz + Pz) % Pz, y = ((sy - cy) % Py + Py) % Py, x = ((sx - cx) % Px + Px) % Px;
        out[i] = scale * full[((int64_t)z * Py + y) * Px + x];
    }
}

int ew_grid_rl(int64_t n) {
    const int64_t nb = (n + 255) / 256, cap = (int64_t)sms() * 16;
    return (int)(nb < cap ? (nb > 0 ? nb : 1) : cap);
}

// The full-grid geometry (no image region, no halo) used to bring an
// accumulated cross-spectrum back to lags.
RlGeom full_geom(const RlGeom &g) {
    RlGeom gf = g;
    gf.nb = 1;
    gf.Z = g.ndim == 3 ? g.Pz : 1;
    gf.Y = g.Py;
    gf.X = g.Px;
    gf.hz = gf.hy = gf.hx = 0;
    return gf;
}

}  // namespace

int rl_launch_iterations(const RlGeom &g, const RlBuffers &b, const float *obs, float *est_out,
                         int32_t num_iter, int32_t clip, float eps, void *stream, PassTimer *timer) {
    RlRunner run(g, b, stream, timer);
    if (!run.ok) return (int)cudaErrorInvalidValue;
    return run.iterations(obs, est_out, num_iter, clip, eps, false);
}

int rl_apply(const RlGeom &g, const RlBuffers &b, const void *H, int conj, const float *x, float *out,
             void *stream, PassTimer *timer) {
    RlRunner run(g, b, stream, timer);
    if (!run.ok) return (int)cudaErrorInvalidValue;
    return run.apply(H, conj, x, out, nullptr);
}

static_assert(sizeof(ColItem) == sizeof(RlColItem), "ColItem layout");
static_assert(sizeof(RowItem) == sizeof(RlRowItem), "RowItem layout");

// Batched iterations: per pass kind one launch per group of problems that
// share the transform length (groups built by the host), in the order of
// rl_launch_iterations.
int rl_batch_iterations(const RlBatchLaunch &L, int num_iter, int clip, float eps, void *stream, PassTimer *timer) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto rows = [&](int kind, int est_first, int last) -> int {
        for (int gi = 0; gi < L.n_rows; ++gi) {
            const RlBatchGroup &G = L.rows[gi];
            RowPass r{};
            r.Px = G.n;
            r.M = G.n / 2;
            r.Hx = r.M + 1;
            r.Hp = (r.Hx + 15) & ~15;
            r.pad_mode = L.mode;
            r.kind = kind;
            r.est_first = est_first;
            r.last = last;
            r.clip = clip;
            r.eps = eps;
            if (!fft_make_plan(r.M, &r.plan)) return (int)cudaErrorInvalidValue;
            r.tw = reinterpret_cast<const float2 *>(G.tw);
            r.items = static_cast<const RowItem *>(G.items);
            r.n_items = G.n_items;
            r.total_tiles = G.total_tiles;
            if (timer) timer->begin(kPassRlRow, stream);
            int e = launch_row(r, s);
            if (timer) timer->end(kPassRlRow, stream);
            if (e) return e;
        }
        return 0;
    };
    auto cols = [&](int h2) -> int {
        for (int gi = 0; gi < L.n_cols; ++gi) {
            const RlBatchGroup &G = L.cols[gi];
            ColPass c{};
            c.mode = kColFull;
            c.pad_mode = L.mode;
            c.conj_h = h2;
            c.use_h2 = h2;
            if (!fft_make_plan(G.n, &c.plan)) return (int)cudaErrorInvalidValue;
            c.tw = reinterpret_cast<const float2 *>(G.tw);
            c.items = static_cast<const ColItem *>(G.items);
            c.n_items = G.n_items;
            c.total_tiles = G.total_tiles;
            if (timer) timer->begin(kPassRlColFull, stream);
            int e = launch_col(c, s);
            if (timer) timer->end(kPassRlColFull, stream);
            if (e) return e;
        }
        return 0;
    };
    int e;
    if ((e = rows(kRowInit, 0, 0))) return e;
    for (int it = 0; it < num_iter; ++it) {
        if ((e = cols(0))) return e;
        if ((e = rows(kRowRatio, 0, 0))) return e;
        if ((e = cols(1))) return e;
        if ((e = rows(kRowUpdate, it == 0, it + 1 == num_iter))) return e;
    }
    return 0;
}

// Times one column pass (kind 0: forward * H * inverse over `lines` columns)
// or one row pass (kind 1: the ratio epilogue over `lines` rows) of length n
// on scratch buffers; average of `reps` launches after one warm-up, in ms.
// a: complex, n * (n/2 + 16) * lines / n elements at least (see the host),
// b: lines * n floats.
int rl_tune_pass(int kind, int n, int lines, void *a, void *b, const float2_ *tw, int reps, void *stream,
                 float *ms) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return (int)cudaErrorUnknown;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return (int)cudaErrorUnknown;
    }
    auto launch = [&]() -> int {
        if (kind == 0) {
            ColPass c{};
            c.ncols = lines; c.Hx = lines;
            c.src = static_cast<const float2 *>(a); c.src_outer = 0; c.src_row = lines;
            c.n_img = n; c.halo = 0;
            c.dst = static_cast<float2 *>(a); c.dst_outer = 0; c.dst_row = lines;
            c.store_begin = 0; c.store_count = n;
            c.mode = kColFull; c.pad_mode = LUCEM_PAD_CONSTANT;
            c.H = static_cast<const float2 *>(a); c.h_outer = 0; c.h_row = lines;
            if (!fft_make_plan(n, &c.plan)) return (int)cudaErrorInvalidValue;
            c.tw = reinterpret_cast<const float2 *>(tw);
            return launch_col(c, s);
        }
        RowPass r{};
        r.nrows = lines; r.X = n; r.Px = n; r.M = n / 2; r.Hx = n / 2 + 1; r.Hp = (r.Hx + 15) & ~15; r.hx = 0;
        r.pad_mode = LUCEM_PAD_CONSTANT; r.kind = kRowRatio; r.eps = 1e-6f;
        r.obs = static_cast<const float *>(b);
        r.s1 = static_cast<float2 *>(a);
        if (!fft_make_plan(r.M, &r.plan)) return (int)cudaErrorInvalidValue;
        r.tw = reinterpret_cast<const float2 *>(tw);
        return launch_row(r, s);
    };
    int e = launch();
    if (!e) e = (int)cudaEventRecord(e0, s);
    for (int i = 0; i < reps && !e; ++i) e = launch();
    if (!e) e = (int)cudaEventRecord(e1, s);
    if (!e) e = (int)cudaEventSynchronize(e1);
    if (!e) {
        float t = 0.f;
        e = (int)cudaEventElapsedTime(&t, e0, e1);
        *ms = t / (float)reps;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return e;
}

// Reverse mode through the unrolled iterations (clip off), checkpoints every K.
//   forward:  c = A e;  r = y / guard(c);  a = B r;  e' = e * a
//     (A: convolution with the PSF centred at k-1-k/2, transfer function
//      h_conv; B: correlation centred at k/2, conj(h_corr))
//   backward: abar = ebar * e;  rbar = B^T abar (h_corr);
//             cbar = -rbar y / d^2 where |c| >= eps, else 0;  ybar += rbar / d;
//             ebar = ebar * a + A^T cbar (conj(h_conv)).
//   PSF: dA/dp gives F(cbar) conj(F(e)), dB/dp gives F(r) conj(F(abar)); the
//   sums over iterations are brought back to lags s - centre by one inverse
//   transform on the full grid, scaled by 1 / (Pz Py Px).
int rl_backward(const RlGeom &g, const RlBuffers &b, const RlBwdBuffers &w, const float *y, int T, int K,
                float eps, const float *ebar_T, float *gpsf_conv, float *gpsf_corr, float *ybar, void *stream,
                PassTimer *timer) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RlRunner run(g, b, stream, timer);
    if (!run.ok) return (int)cudaErrorInvalidValue;
    // V: every volume of the batch (the state arrays hold nb volumes each);
    // nspec: one volume's spectrum (the cross-spectra are summed over volumes).
    const int nb = g.nb > 1 ? g.nb : 1;
    const int64_t V = (int64_t)nb * g.Z * g.Y * g.X;
    const size_t vb = (size_t)V * sizeof(float);
    const int64_t nspec = (int64_t)g.Pz * g.Py * g.Hp;
    const int sg = ew_grid_rl(nspec);
    int e;
    if (K < 1) K = 1;
    const int nseg = (T + K - 1) / K;
    float2 *spec_e = reinterpret_cast<float2 *>(w.spec_e), *spec_r = reinterpret_cast<float2 *>(w.spec_r);
    float2 *spec_abar = reinterpret_cast<float2 *>(w.spec_abar), *spec_cbar = reinterpret_cast<float2 *>(w.spec_cbar);
    float2 *pbar1 = reinterpret_cast<float2 *>(w.pbar1), *pbar2 = reinterpret_cast<float2 *>(w.pbar2);
    // Forward, keeping the estimate at the start of every segment.
    if ((e = launch_fill(w.ckpt, V, 0.5f, stream))) return e;
    for (int j = 0; j + 1 < nseg; ++j) {
        float *dst = w.ckpt + (int64_t)(j + 1) * V;
        if ((e = (int)cudaMemcpyAsync(dst, w.ckpt + (int64_t)j * V, vb, cudaMemcpyDeviceToDevice, s))) return e;
        if ((e = run.iterations(y, dst, K, 0, eps, true))) return e;
    }
    if ((e = (int)cudaMemcpyAsync(w.ebar, ebar_T, vb, cudaMemcpyDeviceToDevice, s))) return e;
    if ((e = (int)cudaMemsetAsync(pbar1, 0, nspec * sizeof(float2), s))) return e;
    if (pbar2 && (e = (int)cudaMemsetAsync(pbar2, 0, nspec * sizeof(float2), s))) return e;
    if (ybar && (e = (int)cudaMemsetAsync(ybar, 0, vb, s))) return e;
    for (int j = nseg - 1; j >= 0; --j) {
        const int k0 = j * K, k1 = T < k0 + K ? T : k0 + K;
        // Recompute the segment's estimates.
        if ((e = (int)cudaMemcpyAsync(w.seg, w.ckpt + (int64_t)j * V, vb, cudaMemcpyDeviceToDevice, s))) return e;
        for (int k = k0; k + 1 < k1; ++k) {
            float *next = w.seg + (int64_t)(k - k0 + 1) * V;
            if ((e = (int)cudaMemcpyAsync(next, next - V, vb, cudaMemcpyDeviceToDevice, s))) return e;
            if ((e = run.iterations(y, next, 1, 0, eps, true))) return e;
        }
        for (int k = k1 - 1; k >= k0; --k) {
            const float *ek = w.seg + (int64_t)(k - k0) * V;
            // c = A e_k (kept), r = y / guard(c) straight into the correlation,
            // a = B r: the ratio is fused into the row pass between them.
            if ((e = run.row(kRowRealIn, ek, nullptr, 0, 0, 0, eps))) return e;
            if ((e = run.pair(b.h_conv, 0, spec_e))) return e;
            if ((e = run.row(kRowRatioKeep, y, w.c, 0, 0, 0, eps))) return e;
            if ((e = run.pair(b.h_corr, 1, spec_r))) return e;
            // a out (kept) and abar = ebar * e_k in, in one row pass; rbar =
            // B^T abar; cbar (and ybar) fused into the row pass that starts
            // t = A^T cbar; ebar = ebar * a + t fused into the last one.
            if ((e = run.row(kRowAbar, ek, w.a, 0, 0, 0, eps, w.ebar))) return e;
            if ((e = run.pair(b.h_corr, 0, spec_abar))) return e;
            if ((e = run.row(kRowCbar, y, nullptr, 0, 0, 0, eps, w.c, ybar))) return e;
            if ((e = run.pair(b.h_conv, 1, spec_cbar))) return e;
            if ((e = run.row(kRowEbar, nullptr, nullptr, 0, 0, 0, eps, w.a, w.ebar))) return e;
            if (pbar2) {
                spec_mac_kernel<<<sg, 256, 0, s>>>(pbar1, spec_cbar, spec_e, nullptr, nullptr, nspec, nb);
                spec_mac_kernel<<<sg, 256, 0, s>>>(pbar2, spec_r, spec_abar, nullptr, nullptr, nspec, nb);
            } else {
                spec_mac_kernel<<<sg, 256, 0, s>>>(pbar1, spec_cbar, spec_e, spec_r, spec_abar, nspec, nb);
            }
            if ((e = (int)cudaGetLastError())) return e;
        }
    }
    const RlGeom gf = full_geom(g);
    RlBuffers bf = b;
    bf.s1 = w.full_s1;
    bf.s2 = w.full_s2;
    RlRunner full(gf, bf, stream, timer);
    if (!full.ok) return (int)cudaErrorInvalidValue;
    const float scale = 1.0f / ((float)g.Pz * (float)g.Py * (float)g.Px);
    const int kz = w.kdims[0], ky = w.kdims[1], kx = w.kdims[2];
    if ((e = full.spectrum_to_real(pbar1, w.full_real))) return e;
    gather_lags_kernel<<<ew_grid_rl(kz * ky * kx), 256, 0, s>>>(w.full_real, gf.Z, g.Py, g.Px, kz, ky, kx,
                                                               w.c_conv[0], w.c_conv[1], w.c_conv[2], scale,
                                                               gpsf_conv);
    if (pbar2) {
        if ((e = full.spectrum_to_real(pbar2, w.full_real))) return e;
        gather_lags_kernel<<<ew_grid_rl(kz * ky * kx), 256, 0, s>>>(w.full_real, gf.Z, g.Py, g.Px, kz, ky, kx,
                                                                   w.c_corr[0], w.c_corr[1], w.c_corr[2], scale,
                                                                   gpsf_corr);
    }
    return (int)cudaGetLastError();
}

// Gradients of out = A x (zero padding): gx = A^T gout (conj(h_conv)), and
// gpsf[s] = sum_y gout[y] x[y - (s - centre)], from F(gout) conj(F(x)).
int rl_convolve_backward(const RlGeom &g, const RlBuffers &b, const RlBwdBuffers &w, const float *x,
                         const float *gout, float *gx, float *gpsf, void *stream, PassTimer *timer) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    RlRunner run(g, b, stream, timer);
    if (!run.ok) return (int)cudaErrorInvalidValue;
    float2 *spec_x = reinterpret_cast<float2 *>(w.spec_e), *spec_g = reinterpret_cast<float2 *>(w.spec_cbar);
    float2 *pbar = reinterpret_cast<float2 *>(w.pbar1);
    int e;
    if ((e = run.apply(b.h_conv, 1, gout, gx ? gx : w.t, gpsf ? spec_g : nullptr))) return e;
    if (!gpsf) return 0;
    if ((e = run.apply(b.h_conv, 0, x, w.c, spec_x))) return e;
    const int64_t nspec = (int64_t)g.Pz * g.Py * g.Hp;
    if ((e = (int)cudaMemsetAsync(pbar, 0, nspec * sizeof(float2), s))) return e;
    spec_mac_kernel<<<ew_grid_rl(nspec), 256, 0, s>>>(pbar, spec_g, spec_x, nullptr, nullptr, nspec,
                                                      g.nb > 1 ? g.nb : 1);
    const RlGeom gf = full_geom(g);
    RlBuffers bf = b;
    bf.s1 = w.full_s1;
    bf.s2 = w.full_s2;
    RlRunner full(gf, bf, stream, timer);
    if (!full.ok) return (int)cudaErrorInvalidValue;
    if ((e = full.spectrum_to_real(pbar, w.full_real))) return e;
    const int kz = w.kdims[0], ky = w.kdims[1], kx = w.kdims[2];
    gather_lags_kernel<<<ew_grid_rl(kz * ky * kx), 256, 0, s>>>(
        w.full_real, gf.Z, g.Py, g.Px, kz, ky, kx, w.c_conv[0], w.c_conv[1], w.c_conv[2],
        1.0f / ((float)g.Pz * (float)g.Py * (float)g.Px), gpsf);
    return (int)cudaGetLastError();
}

int rl_launch_otf(const RlGeom &g, const double *psf_dev, const int32_t kdims[3],
                  const int32_t centre[3], double *work_a, double *work_b, void *h_out,
                  const double *twd_x, const double *twd_y, const double *twd_z, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int kz = kdims[0], ky = kdims[1], kx = kdims[2];
    double2 *A = reinterpret_cast<double2 *>(work_a);
    double2 *B = reinterpret_cast<double2 *>(work_b);
    const double scale = 1.0 / ((double)g.Pz * (double)g.Py * (double)g.Px);
    auto grid_for = [](int64_t total) {
        int64_t nb = (total + 255) / 256;
        int64_t cap = (int64_t)sms() * 32;
        return (int)(nb < cap ? (nb > 0 ? nb : 1) : cap);
    };
    int64_t ta = (int64_t)kz * ky * g.Hx;
    otf_x_kernel<<<grid_for(ta), 256, 0, s>>>(psf_dev, kz, ky, kx, centre[2], g.Px, g.Hx, g.Hp,
                                               reinterpret_cast<const double2 *>(twd_x), A);
    int64_t tb = (int64_t)kz * g.Py * g.Hx;
    otf_y_kernel<<<grid_for(tb), 256, 0, s>>>(A, kz, ky, centre[1], g.Py, g.Hx, g.Hp,
                                               reinterpret_cast<const double2 *>(twd_y), B);
    int64_t tz = (int64_t)g.Pz * g.Py * g.Hx;
    otf_z_kernel<<<grid_for(tz), 256, 0, s>>>(B, kz, centre[0], g.Pz, g.Py, g.Hx, g.Hp,
                                               reinterpret_cast<const double2 *>(twd_z), scale,
                                               static_cast<float2 *>(h_out));
    return (int)cudaGetLastError();
}

}  // namespace lucem
