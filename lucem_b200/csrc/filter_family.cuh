// filter_family.cuh -- the fused Gaussian-family tile kernels (see filter.cu
// for what they replace in the reference) and their launchers, templated on
// the input type.  Each input type is instantiated in its own translation unit
// (filter_family_u8.cu, _u16.cu, _f32.cu) so the three compile in parallel;
// filter.cu dispatches on the type.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "internal.h"
#include "tensor_ops.cuh"

namespace lucem {
namespace famk {

constexpr int kTH = kFamTile;  // output tile rows
constexpr int kTW = kFamTile;  // output tile columns
constexpr int kThreads = 256;
constexpr int kITP = 66;       // pitch of the transposed intermediate (even: 8-byte pairs)

inline int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// crates/lucem-ops/src/core/kernels/pad.rs:11-34.
template <int MODE>
__device__ __forceinline__ int pad_index(int p, int len) {
    if (p >= 0 && p < len) return p;
    if (MODE == LUCEM_PAD_CONSTANT) return -1;
    if (MODE == LUCEM_PAD_NEAREST) return p < 0 ? 0 : len - 1;
    if (MODE == LUCEM_PAD_WRAP) return ((p % len) + len) % len;
    if (MODE == LUCEM_PAD_REFLECT) {
        int period = 2 * len;
        int r = ((p % period) + period) % period;
        return r < len ? r : period - 1 - r;
    }
    int period = max(2 * len - 2, 1);  // mirror
    int r = ((p % period) + period) % period;
    return r < len ? r : period - r;
}

__device__ __forceinline__ int pad_index_rt(int p, int len, int mode) {
    if (p >= 0 && p < len) return p;
    switch (mode) {
    case LUCEM_PAD_CONSTANT: return -1;
    case LUCEM_PAD_NEAREST: return pad_index<LUCEM_PAD_NEAREST>(p, len);
    case LUCEM_PAD_WRAP: return pad_index<LUCEM_PAD_WRAP>(p, len);
    case LUCEM_PAD_MIRROR: return pad_index<LUCEM_PAD_MIRROR>(p, len);
    default: return pad_index<LUCEM_PAD_REFLECT>(p, len);
    }
}

// u8 / u16 / f32 -> f32 times `scale`.  Integers go through the float bit
// pattern 2^23 + v (exact for v < 2^23) on the FMA pipe instead of a
// conversion instruction: (2^23 + v) * s - 2^23 * s is v * s rounded once,
// the same value as float(v) * s.
__device__ __forceinline__ float to_f32_scaled(uint32_t v, float s) {
    return fmaf(__uint_as_float(0x4B000000u | v), s, -8388608.0f * s);
}
__device__ __forceinline__ float to_f32_scaled(uint16_t v, float s) { return to_f32_scaled((uint32_t)v, s); }
__device__ __forceinline__ float to_f32_scaled(uint8_t v, float s) { return to_f32_scaled((uint32_t)v, s); }
__device__ __forceinline__ float to_f32_scaled(float v, float s) { return v * s; }

template <typename T>
__device__ __forceinline__ float load_as_float(const T *p) { return static_cast<float>(__ldg(p)); }

// Two consecutive samples of one load.
template <typename T> struct Pair;
template <> struct Pair<uint8_t> { using type = uchar2; };
template <> struct Pair<uint16_t> { using type = ushort2; };
template <> struct Pair<float> { using type = float2; };

// Where one CTA tile sits.  Coordinates of the read box are absolute (slide
// or plane); the pad map applies at the read box's borders.
struct TileGeom {
    int plane;
    int rb_y, rb_x, rb_h, rb_w;   // read box
    int oy, ox;                   // output tile origin (absolute)
    int th, tw;                   // valid rows / cols of this tile
    // Batch of separate images: this tile's image and output (row pitches in
    // elements) replace FamParams' input and single output.  Null otherwise.
    const void *in;
    float *out;
    int64_t in_pitch, out_pitch;
};

// Axis-0 pass of one filter with kernel radius R over the staged tile A
// (pitch AWP): item = (column pair, 8 rows).  Every output is accumulated in
// tap order with packed f32x2 FMAs (two columns per instruction), taps
// (w, w) in registers 16 at a time.  Writes IT[c][y] (c from cstart).
template <int R>
__device__ __forceinline__ void vpass(const float *__restrict__ A, int AWP, int row0, int cstart, int ncols,
                                   const float2 *__restrict__ w, float *__restrict__ IT) {
    constexpr int NT = 2 * R + 1;
    const int npairs = ncols / 2;
    // q / npairs for q < 8 npairs <= 512 as a multiply and shift, exact
    // there (the rounding of the reciprocal adds less than 1 / npairs).
    const uint32_t inv = (65536u + (uint32_t)npairs - 1u) / (uint32_t)npairs;
    for (int q = threadIdx.x; q < npairs * 8; q += kThreads) {
        const int yc = (int)(((uint32_t)q * inv) >> 16), cp = q - yc * npairs;
        const float *col = A + (yc * 8 + row0) * AWP + cstart + 2 * cp;
        float2 acc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = make_float2(0.f, 0.f);
#pragma unroll
        for (int s0 = 0; s0 < NT; s0 += 8) {
            constexpr int kBlk = 8;
            float2 wv[kBlk];
#pragma unroll
            for (int u = 0; u < kBlk; ++u)
                if (s0 + u < NT) wv[u] = w[s0 + u];
#pragma unroll
            for (int m = 0; m < kBlk + 7; ++m) {
                if (s0 + m >= NT + 7) break;
                const float2 x = *reinterpret_cast<const float2 *>(col + (s0 + m) * AWP);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int u = m - j;
                    if (u >= 0 && u < kBlk && s0 + u < NT) acc[j] = __ffma2_rn(wv[u], x, acc[j]);
                }
            }
        }
        float *o0 = IT + (2 * cp) * kITP + yc * 8;
        float *o1 = o0 + kITP;
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            *reinterpret_cast<float2 *>(o0 + j) = make_float2(acc[j].x, acc[j + 1].x);
            *reinterpret_cast<float2 *>(o1 + j) = make_float2(acc[j].y, acc[j + 1].y);
        }
    }
}

// Axis-1 pass with kernel radius R: thread = (row pair yp, 8 columns from
// x0); reads IT[x0 + m][2 yp .. 2 yp + 1] as one 8-byte word per tap row.
template <int R>
__device__ __forceinline__ void hpass(const float *__restrict__ IT, int x0, int yp, const float2 *__restrict__ w,
                                   float2 *__restrict__ out) {
    constexpr int NT = 2 * R + 1;
    const float *row = IT + x0 * kITP + 2 * yp;
#pragma unroll
    for (int j = 0; j < 8; ++j) out[j] = make_float2(0.f, 0.f);
#pragma unroll
    for (int s0 = 0; s0 < NT; s0 += 8) {
        constexpr int kBlk = 8;
        float2 wv[kBlk];
#pragma unroll
        for (int u = 0; u < kBlk; ++u)
            if (s0 + u < NT) wv[u] = w[s0 + u];
#pragma unroll
        for (int m = 0; m < kBlk + 7; ++m) {
            if (s0 + m >= NT + 7) break;
            const float2 x = *reinterpret_cast<const float2 *>(row + (s0 + m) * kITP);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int u = m - j;
                if (u >= 0 && u < kBlk && s0 + u < NT) out[j] = __ffma2_rn(wv[u], x, out[j]);
            }
        }
    }
}

#define LUCEM_RADII(X) X(0) X(2) X(4) X(6) X(8) X(10) X(12) X(14) X(16) X(20) X(24) X(28) X(32)

__device__ __forceinline__ void vpass_r(int R, const float *A, int AWP, int row0, int cstart, int ncols,
                                        const float2 *w, float *IT) {
    switch (R) {
#define V(r) \
    case r: vpass<r>(A, AWP, row0, cstart, ncols, w, IT); break;
        LUCEM_RADII(V)
#undef V
    default: break;
    }
}

__device__ __forceinline__ void hpass_r(int R, const float *IT, int x0, int yp, const float2 *w, float2 *out) {
    switch (R) {
#define H(r) \
    case r: hpass<r>(IT, x0, yp, w, out); break;
        LUCEM_RADII(H)
#undef H
    default: break;
    }
}

// Eight consecutive outputs of row y from column x of a tile (two 16-byte
// stores where aligned and inside the tile).
__device__ __forceinline__ void store_row8(float *obase, int64_t opitch, const TileGeom &g, int y, int x,
                                           const float *v) {
    float *dst = obase + (int64_t)(g.oy + y) * opitch + g.ox + x;
    if ((x + 8 <= g.tw) && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0)) {
        reinterpret_cast<float4 *>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4 *>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (x + j < g.tw) dst[j] = v[j];
    }
}

// Tensor epilogue: the first three filters' responses per pixel through
// tens::apply into outs[0..2] (the ridge modes read their running maximum
// from outs[0] first, unless tensor_first).
template <int NOUT>
__device__ __forceinline__ void tensor_epilogue(const FamParams &p, const TileGeom &g, const float2 (&acc)[NOUT][8],
                                                int yp, int xc) {
    float *ob[3];
    int64_t op[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ob[k] = g.out ? g.out : p.outs[k].out + (int64_t)g.plane * p.outs[k].plane_stride;
        op[k] = g.out ? g.out_pitch : p.outs[k].row_pitch;
    }
    const bool ridge = p.tensor >= kTensorFrangi && p.tensor <= kTensorMeijering;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int y = 2 * yp + h, x = xc * 8;
        if (y >= g.th) continue;
        float prev[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) prev[j] = 0.0f;
        if (ridge && !p.tensor_first) {
            const float *src = ob[0] + (int64_t)(g.oy + y) * op[0] + g.ox + x;
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (x + j < g.tw) prev[j] = src[j];
        }
        float v0[8], v1[8], v2[8];
        int nout = 1;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float a = h ? acc[0][j].y : acc[0][j].x;
            const float b = h ? acc[1][j].y : acc[1][j].x;
            const float c = h ? acc[2][j].y : acc[2][j].x;
            nout = tens::apply(p.tensor, a, b, c, prev[j], p.tensor_p0, p.tensor_p1, p.tensor_black != 0, &v0[j],
                               &v1[j], &v2[j]);
        }
        store_row8(ob[0], op[0], g, y, x, v0);
        if (nout > 1) store_row8(ob[1], op[1], g, y, x, v1);
        if (nout > 2) store_row8(ob[2], op[2], g, y, x, v2);
    }
}

// One 64 x 64 output tile: stage tile + halo (cast fused), then per filter
// the axis-0 pass into IT and the axis-1 pass into registers, folded into
// every response that uses the filter; responses written once at the end.
// TENSOR: the tensor epilogue (FamParams::tensor) is compiled in; kernels
// that never take it (the tile walk, the batch) leave it out.
template <typename T, int NOUT, int RF = -1, bool STAGED = false, bool TENSOR = false>
__device__ void family_tile(const FamParams &p, const TileGeom &g, float *A, float *IT, bool preloaded = false) {
    const int tid = threadIdx.x;
    // RF >= 0: one filter whose two kernel radii are both RF, known at compile
    // time (strides and tap loops become constants).
    const int R0 = RF >= 0 ? RF : p.rmax0, R1 = RF >= 0 ? RF : p.rmax1;
    const int AWP = kTW + 2 * R1;   // even (R1 even)
    const int AH = kTH + 2 * R0;
    const int64_t ipitch = g.in ? g.in_pitch : p.in_row_pitch;
    const T *in = g.in ? static_cast<const T *>(g.in)
                       : static_cast<const T *>(p.in) + (int64_t)g.plane * p.in_plane_stride;

    // Phase 0: tile + halo -> A (f32).  A warp stages rows warp, warp + 8,
    // ...; each lane covers columns lane, lane + 32, ... of a row (no index
    // division), and every lane issues the loads of 4 rows before storing
    // any of them, so many global loads are in flight per warp.
    // preloaded: A already holds the window (copied ahead by the caller).
    if (!STAGED && !preloaded) {
        const int wy0 = g.oy - g.rb_y - R0, wx0 = g.ox - g.rb_x - R1;  // window origin in the read box
        const T *wbase = in + (int64_t)g.rb_y * ipitch + g.rb_x;
        const bool interior = wy0 >= 0 && wx0 >= 0 && wy0 + AH <= g.rb_h && wx0 + AWP <= g.rb_w;
        const T *w0 = wbase + (int64_t)wy0 * ipitch + wx0;
        const bool pairs_ok = (ipitch % 2 == 0) &&
                              (reinterpret_cast<uintptr_t>(w0) % (2 * sizeof(T)) == 0);
        const int lane = tid & 31, warp = tid >> 5;
        constexpr int kRows = NOUT == 1 ? 4 : 2;  // rows in flight per lane
        constexpr int kWarps = kThreads / 32;
        if (interior && pairs_ok) {
            // No pad map: two samples per load (AWP is even, <= 128).
            using V2 = typename Pair<T>::type;
            const int npr = AWP / 2;
            for (int r0 = warp; r0 < AH; r0 += kWarps * kRows) {
                V2 v[kRows][2];
#pragma unroll
                for (int k = 0; k < kRows; ++k) {
                    const int r = r0 + kWarps * k;
                    const V2 *src = reinterpret_cast<const V2 *>(w0 + (int64_t)r * ipitch);
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        if (r < AH && lane + 32 * h < npr) v[k][h] = __ldg(src + lane + 32 * h);
                }
#pragma unroll
                for (int k = 0; k < kRows; ++k) {
                    const int r = r0 + kWarps * k;
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        if (r < AH && lane + 32 * h < npr)
                            *reinterpret_cast<float2 *>(A + r * AWP + 2 * (lane + 32 * h)) =
                                make_float2(to_f32_scaled(v[k][h].x, p.in_scale), to_f32_scaled(v[k][h].y, p.in_scale));
                }
            }
        } else {
            // Pad map relative to the read box (border tiles, odd pitches):
            // the row map once per row, the column map per element.
            for (int r0 = warp; r0 < AH; r0 += kWarps * kRows) {
                float v[kRows][4];
#pragma unroll
                for (int k = 0; k < kRows; ++k) {
                    const int r = r0 + kWarps * k;
                    const int py = r < AH ? pad_index_rt(wy0 + r, g.rb_h, p.mode) : -1;
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const int c = lane + 32 * h;
                        v[k][h] = p.cval;
                        if (py >= 0 && c < AWP) {
                            const int px = pad_index_rt(wx0 + c, g.rb_w, p.mode);
                            if (px >= 0) v[k][h] = to_f32_scaled(__ldg(wbase + (int64_t)py * ipitch + px), p.in_scale);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < kRows; ++k) {
                    const int r = r0 + kWarps * k;
#pragma unroll
                    for (int h = 0; h < 4; ++h)
                        if (r < AH && lane + 32 * h < AWP) A[r * AWP + lane + 32 * h] = v[k][h];
                }
            }
        }
    }
    if constexpr (!STAGED) __syncthreads();

    // Axis-1 item of this thread: a warp covers 8 row pairs x 4 chunks of 8
    // columns (8-byte bank = 8 * chunk + pair: conflict-free).
    const int lane = tid & 31, wt = tid >> 5;
    const int yp = (wt & 3) * 8 + (lane & 7);    // row pair: rows 2 yp, 2 yp + 1
    const int xc = (wt >> 2) * 4 + (lane >> 3);  // columns xc * 8 .. + 7
    float2 acc[NOUT][8];
#pragma unroll
    for (int k = 0; k < NOUT; ++k)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[k][j] = make_float2(0.f, 0.f);

    // Identity terms (unsharp) read the staged input at the output pixel.
#pragma unroll
    for (int k = 0; k < NOUT; ++k) {
        if (k >= p.n_outputs) break;
        const FamOutput &o = p.outs[k];
        if (o.fa == -2 || o.fb == -2) {
            const float coef = o.fa == -2 ? o.alpha : o.beta;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float a0 = A[(2 * yp + R0) * AWP + xc * 8 + j + R1];
                const float a1 = A[(2 * yp + 1 + R0) * AWP + xc * 8 + j + R1];
                acc[k][j] = make_float2(acc[k][j].x + coef * a0, acc[k][j].y + coef * a1);
            }
        }
    }

    const int nf = RF >= 0 ? 1 : p.n_filters;
    for (int f = 0; f < nf; ++f) {
        const int r0 = RF >= 0 ? RF : p.r0[f], r1 = RF >= 0 ? RF : p.r1[f];
        const int ncols = kTW + 2 * r1;           // even
        const int cstart = R1 - r1;               // even
        if constexpr (RF >= 0) vpass<RF>(A, AWP, R0 - r0, cstart, ncols, reinterpret_cast<const float2 *>(p.taps0[f]), IT);
        else vpass_r(r0, A, AWP, R0 - r0, cstart, ncols, reinterpret_cast<const float2 *>(p.taps0[f]), IT);
        __syncthreads();
        if (p.mode == LUCEM_PAD_CONSTANT) {
            // A column outside the read box is cval itself in the reference's
            // intermediate (its axis-1 pass pads the axis-0 result with cval).
            for (int q = tid; q < ncols; q += kThreads) {
                const int rx = g.ox - g.rb_x - r1 + q;
                if (rx < 0 || rx >= g.rb_w)
                    for (int y = 0; y < kTH; ++y) IT[q * kITP + y] = p.cval;
            }
            __syncthreads();
        }
        float2 o[8];
        if constexpr (RF >= 0) hpass<RF>(IT, xc * 8, yp, reinterpret_cast<const float2 *>(p.taps1[f]), o);
        else hpass_r(r1, IT, xc * 8, yp, reinterpret_cast<const float2 *>(p.taps1[f]), o);
        // Fold this filter into every response that uses it.
#pragma unroll
        for (int k = 0; k < NOUT; ++k) {
            if (k >= p.n_outputs) break;
            const FamOutput &oo = p.outs[k];
            if (oo.combine == (int)Combine::kHypot) {
                if (oo.fa == f || oo.fb == f) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[k][j] = __ffma2_rn(o[j], o[j], acc[k][j]);
                }
            } else {
                // Two terms at most, added to an exact 0: the result does not
                // depend on which filter runs first.
                if (oo.fa == f) {
                    const float2 al = make_float2(oo.alpha, oo.alpha);
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[k][j] = __ffma2_rn(al, o[j], acc[k][j]);
                }
                if (oo.fb == f) {
                    const float2 be = make_float2(oo.beta, oo.beta);
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[k][j] = __ffma2_rn(be, o[j], acc[k][j]);
                }
            }
        }
        __syncthreads();  // IT is rewritten by the next filter
    }

    if constexpr (TENSOR && NOUT >= 3) {
        tensor_epilogue<NOUT>(p, g, acc, yp, xc);
        return;
    }
    // Epilogue: bias / sqrt, then two 32-byte row segments per thread.
#pragma unroll
    for (int k = 0; k < NOUT; ++k) {
        if (k >= p.n_outputs) break;
        const FamOutput &oo = p.outs[k];
        float *obase = g.out ? g.out : oo.out + (int64_t)g.plane * oo.plane_stride;
        const int64_t opitch = g.out ? g.out_pitch : oo.row_pitch;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int y = 2 * yp + h, x = xc * 8;
            if (y >= g.th) continue;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float a = h ? acc[k][j].y : acc[k][j].x;
                if (oo.combine == (int)Combine::kHypot) v[j] = sqrtf(fmaxf(a, 0.0f)) * oo.alpha;
                else v[j] = a + oo.bias;
            }
            float *dst = obase + (int64_t)(g.oy + y) * opitch + g.ox + x;
            const bool vec_ok = (x + 8 <= g.tw) && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0);
            if (vec_ok) {
                reinterpret_cast<float4 *>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
                reinterpret_cast<float4 *>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (x + j < g.tw) dst[j] = v[j];
            }
        }
    }
}

// CTAs per SM the plain-blur kernels (one filter of radius RF, RF >= 0)
// are compiled for: four where the tile code fits 64 registers without
// spilling (u16 input up to radius 8, u8 / f32 from radius 4 to 8; the
// image batch u16 only), else three; the general kernels two.  A 2048^2
// u16 blur at sigma 2 went from 34.5 to 31.8 us with four: its 1,024 tiles
// run in two rounds of 592 CTAs instead of three of 444.
template <typename T, int RF, bool BATCH>
constexpr int family_min_ctas() {
    return RF < 0 ? 2
                  : (RF <= 8 && (std::is_same<T, uint16_t>::value || (!BATCH && RF >= 4))) ? 4 : 3;
}

// Planes launch: B planes of [H, W], each its own read and owned box.
template <typename T, int NOUT, int RF = -1, bool TENSOR = false>
__global__ void __launch_bounds__(kThreads, family_min_ctas<T, RF, false>())
family_planes_kernel(const __grid_constant__ FamParams p, int tiles_y, int tiles_x) {
    extern __shared__ float4 smem4[];
    float *A = reinterpret_cast<float *>(smem4);
    float *IT = A + (kTH + 2 * p.rmax0) * (kTW + 2 * p.rmax1);
    const int per_plane = tiles_y * tiles_x;
    const int total = per_plane * p.B;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        TileGeom g{};
        g.plane = t / per_plane;
        int r = t - g.plane * per_plane;
        int ty = r / tiles_x, tx = r - ty * tiles_x;
        g.rb_y = 0; g.rb_x = 0; g.rb_h = p.H; g.rb_w = p.W;
        g.oy = ty * kTH; g.ox = tx * kTW;
        g.th = min(kTH, p.H - g.oy); g.tw = min(kTW, p.W - g.ox);
        family_tile<T, NOUT, RF, false, TENSOR>(p, g, A, IT);
        __syncthreads();
    }
}

// Asynchronous global -> shared copies (cp.async, completion waited for by
// the issuing thread, then a block barrier makes them visible).
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Tile tg of a work list (global index): the item owning it, then its place
// in the item's own box.  The item is searched from *hint (the previous
// tile's item: tiles are taken in increasing order, so it is that item or one
// a few entries on), by a short forward scan, else by binary search.
__device__ __forceinline__ TileGeom work_geom(const FamWork *__restrict__ work, int n_work, int tg, int *hint) {
    int lo = *hint;
    bool found = false;
    if (lo >= 0 && lo < n_work && work[lo].tile_begin <= tg) {
        for (int k = 0; k < 8; ++k) {
            if (lo + 1 >= n_work || work[lo + 1].tile_begin > tg) {
                found = true;
                break;
            }
            ++lo;
        }
    } else {
        lo = 0;
    }
    if (!found) {
        int hi = n_work - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (work[mid].tile_begin <= tg) lo = mid; else hi = mid - 1;
        }
    }
    *hint = lo;
    const FamWork w = work[lo];
    const int local = tg - w.tile_begin;
    const int tiles_x = (w.own_w + kTW - 1) / kTW;
    const int ty = local / tiles_x, tx = local - ty * tiles_x;
    TileGeom g{};
    g.plane = w.channel;
    g.rb_y = w.read_y; g.rb_x = w.read_x; g.rb_h = w.read_h; g.rb_w = w.read_w;
    g.oy = w.own_y + ty * kTH; g.ox = w.own_x + tx * kTW;
    g.th = min(kTH, w.own_y + w.own_h - g.oy); g.tw = min(kTW, w.own_x + w.own_w - g.ox);
    return g;
}

// Starts the copy of tile g's raw window (tile + halo, inside its read box)
// into `raw` (pitch AWP elements) when no pad map is needed and the window's
// rows are 16- or 4-byte aligned; returns false (nothing issued) otherwise.
// The answer is the same in every thread.
template <typename T>
__device__ __forceinline__ bool prefetch_window(const FamParams &p, const TileGeom &g, T *raw) {
    const int R0 = p.rmax0, R1 = p.rmax1, AWP = kTW + 2 * R1, AH = kTH + 2 * R0;
    const int wy0 = g.oy - g.rb_y - R0, wx0 = g.ox - g.rb_x - R1;
    if (wy0 < 0 || wx0 < 0 || wy0 + AH > g.rb_h || wx0 + AWP > g.rb_w) return false;
    const int64_t ipitch = g.in ? g.in_pitch : p.in_row_pitch;
    const T *base = g.in ? static_cast<const T *>(g.in)
                         : static_cast<const T *>(p.in) + (int64_t)g.plane * p.in_plane_stride;
    const T *w0 = base + (int64_t)(g.rb_y + wy0) * ipitch + (g.rb_x + wx0);
    const size_t row_bytes = (size_t)AWP * sizeof(T), pitch_bytes = (size_t)ipitch * sizeof(T);
    const uintptr_t a = reinterpret_cast<uintptr_t>(w0);
    const char *src = reinterpret_cast<const char *>(w0);
    char *dst = reinterpret_cast<char *>(raw);
    if (a % 16 == 0 && pitch_bytes % 16 == 0 && row_bytes % 16 == 0) {
        const int per_row = (int)(row_bytes / 16), n = AH * per_row;
        for (int i = threadIdx.x; i < n; i += kThreads) {
            const int r = i / per_row, c = i - r * per_row;
            cp_async16(dst + (size_t)r * row_bytes + 16 * c, src + (size_t)r * pitch_bytes + 16 * c);
        }
        return true;
    }
    if (a % 4 == 0 && pitch_bytes % 4 == 0 && row_bytes % 4 == 0) {
        const int per_row = (int)(row_bytes / 4), n = AH * per_row;
        for (int i = threadIdx.x; i < n; i += kThreads) {
            const int r = i / per_row, c = i - r * per_row;
            cp_async4(dst + (size_t)r * row_bytes + 4 * c, src + (size_t)r * pitch_bytes + 4 * c);
        }
        return true;
    }
    return false;
}

// Work-list launch: tiles of uneven blocks of a [C, H, W] slide.  With a
// counter the CTAs are persistent and take tiles from it; without one each
// CTA walks tiles blockIdx.x, +gridDim.x, ...  With `raw` room (prefetch),
// a CTA starts the copy of its next tile's window before computing the
// current one, so the loads of one tile overlap the filters of the previous
// (its first tile, and tiles that need the pad map, load as they go).
template <typename T, int NOUT>
__global__ void __launch_bounds__(kThreads, 2)
family_work_kernel(const __grid_constant__ FamParams p, const FamWork *__restrict__ work, int n_work,
                   int n_tiles, int tile_base, int *counter, int prefetch) {
    extern __shared__ float4 smem4[];
    const int AWP = kTW + 2 * p.rmax1, AH = kTH + 2 * p.rmax0;
    float *A = reinterpret_cast<float *>(smem4);
    float *IT = A + AH * AWP;
    T *raw = reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(IT + AWP * kITP + 15) & ~(uintptr_t)15);
    // Thread 0 takes the next tile and writes its geometry here; the block
    // reads it after the barrier (callers make sure every thread has read
    // the previous one first).
    __shared__ int next_tile;
    __shared__ TileGeom next_geom;
    int hint = 0;  // thread 0's item search start
    auto fetch = [&](int cur) {
        if (threadIdx.x == 0) {
            const int tn = counter ? atomicAdd(counter, 1) : (cur < 0 ? (int)blockIdx.x : cur + (int)gridDim.x);
            next_tile = tn;
            if (tn < n_tiles) next_geom = work_geom(work, n_work, tn + tile_base, &hint);
        }
        __syncthreads();
        return next_tile;
    };
    int t = fetch(-1);
    TileGeom g = next_geom;
    bool staged = false;  // tile t's window is in raw (copies issued)
    while (t < n_tiles) {
        if (staged) {
            cp_async_wait_all();
            __syncthreads();
            using V2 = typename Pair<T>::type;
            const V2 *r2 = reinterpret_cast<const V2 *>(raw);
            float2 *a2 = reinterpret_cast<float2 *>(A);
            for (int i = threadIdx.x; i < AWP * AH / 2; i += kThreads) {
                const V2 v = r2[i];
                a2[i] = make_float2(to_f32_scaled(v.x, p.in_scale), to_f32_scaled(v.y, p.in_scale));
            }
        }
        __syncthreads();  // raw converted; every thread holds g
        const int tn = fetch(t);
        const bool next_staged = prefetch && tn < n_tiles && prefetch_window<T>(p, next_geom, raw);
        family_tile<T, NOUT>(p, g, A, IT, staged);
        __syncthreads();
        t = tn;
        g = next_geom;
        staged = next_staged;
    }
    cp_async_wait_all();
}


// Tile t of a batch: the image owning it (the last item whose tile_begin
// <= t, searched from *hint as work_geom does), then its place in that
// image, which is its own read box.
__device__ __forceinline__ TileGeom batch_geom(const FamImage *__restrict__ items, int n_items, int t, int *hint) {
    int lo = *hint;
    bool found = false;
    if (lo >= 0 && lo < n_items && items[lo].tile_begin <= t) {
        for (int k = 0; k < 8; ++k) {
            if (lo + 1 >= n_items || items[lo + 1].tile_begin > t) {
                found = true;
                break;
            }
            ++lo;
        }
    } else {
        lo = 0;
    }
    if (!found) {
        int hi = n_items - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].tile_begin <= t) lo = mid; else hi = mid - 1;
        }
    }
    *hint = lo;
    const FamImage it = items[lo];
    const int local = t - it.tile_begin;
    const int tiles_x = (it.W + kTW - 1) / kTW;
    const int ty = local / tiles_x, tx = local - ty * tiles_x;
    TileGeom g{};
    g.plane = 0;
    g.rb_y = 0; g.rb_x = 0; g.rb_h = it.H; g.rb_w = it.W;
    g.oy = ty * kTH; g.ox = tx * kTW;
    g.th = min(kTH, it.H - g.oy); g.tw = min(kTW, it.W - g.ox);
    g.in = it.in;
    g.out = it.out;
    g.in_pitch = it.in_pitch;
    g.out_pitch = it.out_pitch;
    return g;
}

// Batch of separate 2-D images sharing one filter set.  CTAs walk tiles
// blockIdx.x, +gridDim.x, ...; with `raw` room (prefetch) a CTA copies its
// next tile's window ahead while filtering the current one, as the tile
// walk does.
template <typename T, int RF = -1>
__global__ void __launch_bounds__(kThreads, family_min_ctas<T, RF, true>())
family_batch_kernel(const __grid_constant__ FamParams p, const FamImage *__restrict__ items, int n_items,
                    int n_tiles, int prefetch) {
    extern __shared__ float4 smem4[];
    const int AWP = kTW + 2 * p.rmax1, AH = kTH + 2 * p.rmax0;
    float *A = reinterpret_cast<float *>(smem4);
    float *IT = A + AH * AWP;
    T *raw = reinterpret_cast<T *>(reinterpret_cast<uintptr_t>(IT + AWP * kITP + 15) & ~(uintptr_t)15);
    __shared__ TileGeom next_geom;
    int hint = 0;  // thread 0's item search start
    int t = blockIdx.x;
    if (t >= n_tiles) return;
    if (threadIdx.x == 0) next_geom = batch_geom(items, n_items, t, &hint);
    __syncthreads();
    TileGeom g = next_geom;
    bool staged = false;
    while (true) {
        if (staged) {
            cp_async_wait_all();
            __syncthreads();
            using V2 = typename Pair<T>::type;
            const V2 *r2 = reinterpret_cast<const V2 *>(raw);
            float2 *a2 = reinterpret_cast<float2 *>(A);
            for (int i = threadIdx.x; i < AWP * AH / 2; i += kThreads) {
                const V2 v = r2[i];
                a2[i] = make_float2(to_f32_scaled(v.x, p.in_scale), to_f32_scaled(v.y, p.in_scale));
            }
        }
        __syncthreads();  // raw converted; every thread holds g
        const int tn = t + (int)gridDim.x;
        if (threadIdx.x == 0 && tn < n_tiles) next_geom = batch_geom(items, n_items, tn, &hint);
        __syncthreads();
        const bool next_staged = prefetch && tn < n_tiles && prefetch_window<T>(p, next_geom, raw);
        family_tile<T, 1, RF>(p, g, A, IT, staged);
        __syncthreads();
        if (tn >= n_tiles) break;
        t = tn;
        g = next_geom;
        staged = next_staged;
    }
    cp_async_wait_all();
}

// The window copies ahead (a raw buffer in shared memory) only when a plan
// asks for them: on the 512-image batch (sides 64..1024, one filter) the
// autotuner measured them slower for radii 4, 8 and 16.
template <typename T, int RF = -1>
int dispatch_batch(const FamParams &p, size_t smem, const FamImage *items, int n_items, int n_tiles,
                   cudaStream_t s) {
    const size_t raw = ((size_t)(kTW + 2 * p.rmax1) * (kTH + 2 * p.rmax0) * sizeof(T) + 15) & ~(size_t)15;
    const bool want = p.plan ? ((p.plan - 1) & kPlanAhead) != 0 : false;
    const int prefetch = want && smem + raw + 16 + 1024 <= 227 * 1024 ? 1 : 0;
    if (prefetch) smem += raw + 16;
    cudaFuncSetAttribute(family_batch_kernel<T, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, family_batch_kernel<T, RF>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const int slots = sm_count() * per_sm;
    const int grid = n_tiles < slots ? n_tiles : slots;
    family_batch_kernel<T, RF><<<grid, kThreads, smem, s>>>(p, items, n_items, n_tiles, prefetch);
    return (int)cudaGetLastError();
}

template <typename T>
int dispatch_batch_r(const FamParams &p, size_t smem, const FamImage *items, int n_items, int n_tiles,
                     cudaStream_t s) {
    if (p.n_filters == 1 && p.r0[0] == p.r1[0] && p.rmax0 == p.r0[0] && p.rmax1 == p.r1[0]) {
        switch (p.r0[0]) {
#define RFCASE(r) \
    case r: return dispatch_batch<T, r>(p, smem, items, n_items, n_tiles, s);
            RFCASE(2) RFCASE(4) RFCASE(6) RFCASE(8) RFCASE(10) RFCASE(12) RFCASE(16)
#undef RFCASE
        default: break;
        }
    }
    return dispatch_batch<T>(p, smem, items, n_items, n_tiles, s);
}

// ---- TMA staging for the plain 2-D blur ------------------------------------
//
// Used when a launch has at least 12 tiles per SM (4 per resident CTA), so
// that the next tile's copy has a tile's compute to hide behind: measured
// 14-19% faster at 4096^2 and 8192^2, 8% slower at 2048^2 (2.3 tiles per CTA).
//
// Interior tiles of a plain blur (one filter, radius RF on both axes) load
// their (64 + 2 RF)^2 window with one tensor copy (cp.async.bulk.tensor,
// issued by one thread, completion on an mbarrier) into a raw buffer, which
// is converted to f32 in shared memory.  CTAs are persistent and the copy of
// the next tile is issued before the current tile is computed.  Border tiles
// (pad maps) and any wait that gives up use the load path of family_tile.
// No multicast: every copy reads this GPU's own input.

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase: polls until the phase completes or
// `limit_ns` nanoseconds of %globaltimer have passed (limit_ns < 0: no
// polling at all).  Uniform over the block: every thread returns the same
// answer (true only if every thread saw the phase complete).
__device__ __forceinline__ bool mbar_wait_all(uint32_t mbar, uint32_t phase, int64_t limit_ns) {
    bool done = false;
    if (limit_ns >= 0) {
        const uint64_t t0 = global_ns();
        for (;;) {
            uint32_t ok = 0;
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                         : "=r"(ok) : "r"(mbar), "r"(phase) : "memory");
            if (ok) {
                done = true;
                break;
            }
            if ((int64_t)(global_ns() - t0) >= limit_ns) break;
        }
    }
    return __syncthreads_and(done) != 0;
}

constexpr int64_t kTmaWaitDefaultNs = 1000000000;  // one second
constexpr int64_t kTmaDrainNs = 2000000000;        // before exit, for a copy given up on

template <typename T, int RF>
__global__ void __launch_bounds__(kThreads, 3)
family_planes_tma_kernel(const __grid_constant__ FamParams p, const __grid_constant__ CUtensorMap tmap, int tiles_y,
                         int tiles_x) {
    constexpr int AWP = kTW + 2 * RF, AH = kTH + 2 * RF;
    constexpr uint32_t kBytes = (uint32_t)(AWP * AH * sizeof(T));
    extern __shared__ float4 smem4[];
    float *A = reinterpret_cast<float *>(smem4);
    float *IT = A + AH * AWP;
    // raw window, 128-byte aligned, then the mbarrier
    uintptr_t rp = reinterpret_cast<uintptr_t>(IT + AWP * kITP);
    rp = (rp + 127) & ~(uintptr_t)127;
    T *raw = reinterpret_cast<T *>(rp);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(rp + ((kBytes + 15) & ~15u));
    const uint32_t mb = smem_u32(mbar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const int per_plane = tiles_y * tiles_x, total = per_plane * p.B;
    auto geom = [&](int t) {
        TileGeom g{};
        g.plane = t / per_plane;
        const int r = t - g.plane * per_plane, ty = r / tiles_x, tx = r - ty * tiles_x;
        g.rb_y = 0; g.rb_x = 0; g.rb_h = p.H; g.rb_w = p.W;
        g.oy = ty * kTH; g.ox = tx * kTW;
        g.th = min(kTH, p.H - g.oy); g.tw = min(kTW, p.W - g.ox);
        return g;
    };
    auto interior = [&](const TileGeom &g) {
        return g.ox >= RF && g.oy >= RF && g.ox - RF + AWP <= p.W && g.oy - RF + AH <= p.H;
    };
    auto issue = [&](const TileGeom &g) {
        if (threadIdx.x == 0) {
            // Order this CTA's earlier generic reads of raw before the async write.
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mb), "r"(kBytes) : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
                ::"r"(smem_u32(raw)), "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(g.ox - RF), "r"(g.oy - RF),
                "r"(g.plane), "r"(mb)
                : "memory");
        }
    };
    const int64_t limit = p.wait_ns == 0 ? kTmaWaitDefaultNs : p.wait_ns;
    bool tma = true;
    uint32_t phase = 0;
    // A copy given up on is still in flight into `raw`: its phase is waited
    // for (with kTmaDrainNs) before the CTA exits.
    bool lost = false;
    uint32_t lost_phase = 0;
    int t = blockIdx.x;
    bool pending = false;
    if (t < total && interior(geom(t))) {
        issue(geom(t));
        pending = true;
    }
    for (; t < total; t += gridDim.x) {
        const TileGeom g = geom(t);
        bool staged = false;
        if (pending) {
            if (mbar_wait_all(mb, phase, limit)) {
                const int n2 = AWP * AH / 2;
                using V2 = typename Pair<T>::type;
                const V2 *r2 = reinterpret_cast<const V2 *>(raw);
                float2 *a2 = reinterpret_cast<float2 *>(A);
                for (int i = threadIdx.x; i < n2; i += kThreads) {
                    const V2 v = r2[i];
                    a2[i] = make_float2(to_f32_scaled(v.x, p.in_scale), to_f32_scaled(v.y, p.in_scale));
                }
                staged = true;
            } else {
                tma = false;  // never reuse raw after a copy that did not arrive
                lost = true;
                lost_phase = phase;
                if (threadIdx.x == 0 && p.wait_status) atomicAdd(p.wait_status, 1);
            }
            phase ^= 1u;
            __syncthreads();
        }
        const int tn = t + gridDim.x;
        pending = tma && tn < total && interior(geom(tn));
        if (pending) issue(geom(tn));
        if (staged) family_tile<T, 1, RF, true>(p, g, A, IT);
        else family_tile<T, 1, RF, false>(p, g, A, IT);
        __syncthreads();
    }
    // No CTA leaves with a tensor copy still writing into its shared memory:
    // wait (bounded) for the one given up on; count it again if even that
    // wait runs out.
    if (lost && !mbar_wait_all(mb, lost_phase, kTmaDrainNs) && threadIdx.x == 0 && p.wait_status)
        atomicAdd(p.wait_status, 1);
}

// Tensor map of the input planes for family_planes_tma_kernel, when every
// alignment rule of the tiled copy holds: 16-byte base, row and plane
// strides multiples of 16 bytes, the window's inner extent a multiple of 16
// bytes, and every window's x origin (64 k - RF) a multiple of 16 bytes.
// Returns false (no map) otherwise.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiled encode_fn() {
    static const EncodeTiled fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiled>(f);
        cudaGetLastError();
        return (EncodeTiled) nullptr;
    }();
    return fn;
}

template <typename T>
bool make_plane_map(const FamParams &p, int rf, CUtensorMap *map) {
    const size_t es = sizeof(T);
    const int awp = kTW + 2 * rf, ah = kTH + 2 * rf;
    if (reinterpret_cast<uintptr_t>(p.in) % 16 != 0) return false;
    if ((size_t)p.W * es % 16 != 0 || p.in_row_pitch != p.W || p.in_plane_stride != (int64_t)p.H * p.W) return false;
    if ((size_t)awp * es % 16 != 0 || ((size_t)rf * es) % 16 != 0 || awp > 256 || ah > 256) return false;
    if (p.W < awp || p.H < ah) return false;
    // Only while the raw buffer still leaves room for 3 CTAs per SM (the
    // radius-16 window would drop to 2, measured 5% slower than the loads).
    const size_t smem = (size_t)(ah * awp + awp * kITP) * sizeof(float) + 128 + (((size_t)awp * ah * es + 15) & ~(size_t)15) + 16;
    if (3 * (smem + 1024) > 227 * 1024) return false;
    EncodeTiled fn = encode_fn();
    if (!fn) return false;
    const CUtensorMapDataType dt = sizeof(T) == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : sizeof(T) == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint64_t dims[3] = {(cuuint64_t)p.W, (cuuint64_t)p.H, (cuuint64_t)p.B};
    const cuuint64_t strides[2] = {(cuuint64_t)p.W * es, (cuuint64_t)p.H * p.W * es};
    const cuuint32_t box[3] = {(cuuint32_t)awp, (cuuint32_t)ah, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(map, dt, 3, const_cast<void *>(p.in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

template <typename T, int RF>
int dispatch_planes_tma(const FamParams &p, const CUtensorMap &map, int total, int ty, int tx, cudaStream_t s) {
    constexpr int AWP = kTW + 2 * RF, AH = kTH + 2 * RF;
    const size_t smem = (size_t)(AH * AWP + AWP * kITP) * sizeof(float) + 128 +
                        (((size_t)AWP * AH * sizeof(T) + 15) & ~(size_t)15) + 16;
    cudaFuncSetAttribute(family_planes_tma_kernel<T, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, family_planes_tma_kernel<T, RF>, kThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const int slots = sm_count() * per_sm;
    family_planes_tma_kernel<T, RF><<<total < slots ? total : slots, kThreads, smem, s>>>(p, map, ty, tx);
    return (int)cudaGetLastError();
}

template <typename T, int NOUT, int RF = -1, bool TENSOR = false>
int dispatch_planes(const FamParams &p, size_t smem, int grid, int ty, int tx, cudaStream_t s) {
    cudaFuncSetAttribute(family_planes_kernel<T, NOUT, RF, TENSOR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    family_planes_kernel<T, NOUT, RF, TENSOR><<<grid, kThreads, smem, s>>>(p, ty, tx);
    return (int)cudaGetLastError();
}

// Persistent walks (a counter) get the raw-window buffer for the next
// tile's copies when two CTAs per SM still fit with it; the grid is then the
// resident CTAs, at most `grid`.
template <typename T, int NOUT>
int dispatch_work(const FamParams &p, size_t smem, int grid, const FamWork *work, int n_work,
                  int n_tiles, int tile_base, int *counter, cudaStream_t s) {
    const size_t raw = ((size_t)(kTW + 2 * p.rmax1) * (kTH + 2 * p.rmax0) * sizeof(T) + 15) & ~(size_t)15;
    const int bits = p.plan ? p.plan - 1 : 0;
    const bool fits = (p.plan ? 1 : 2) * (smem + raw + 16 + 1024) <= 227 * 1024;
    const int prefetch = counter && (p.plan ? (bits & kPlanAhead) != 0 : true) && fits ? 1 : 0;
    if (prefetch) smem += raw + 16;
    cudaFuncSetAttribute(family_work_kernel<T, NOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (counter) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, family_work_kernel<T, NOUT>, kThreads, smem);
        if (per_sm < 1) per_sm = 1;
        if (bits & kPlanOneCta) per_sm = 1;
        if (grid > sm_count() * per_sm) grid = sm_count() * per_sm;
    }
    family_work_kernel<T, NOUT><<<grid, kThreads, smem, s>>>(p, work, n_work, n_tiles, tile_base, counter, prefetch);
    return (int)cudaGetLastError();
}

template <typename T>
int dispatch_planes_n(const FamParams &p, size_t smem, int grid, int ty, int tx, cudaStream_t s) {
    // A single filter with equal radii along both axes (a plain 2-D blur) runs
    // a kernel compiled for that radius.
    if (p.n_outputs == 1 && p.n_filters == 1 && p.r0[0] == p.r1[0] && p.rmax0 == p.r0[0] && p.rmax1 == p.r1[0]) {
        switch (p.r0[0]) {
#define RFCASE(r)                                                                          \
    case r: {                                                                              \
        CUtensorMap map;                                                                   \
        const bool ahead = p.plan ? ((p.plan - 1) & kPlanAhead) != 0                     \
                                  : ty * tx * p.B >= 12 * sm_count();                      \
        if (ahead && make_plane_map<T>(p, r, &map))                                        \
            return dispatch_planes_tma<T, r>(p, map, ty * tx * p.B, ty, tx, s);            \
        return dispatch_planes<T, 1, r>(p, smem, grid, ty, tx, s);                         \
    }
            RFCASE(2) RFCASE(4) RFCASE(6) RFCASE(8) RFCASE(10) RFCASE(12) RFCASE(16)
#undef RFCASE
        default: break;
        }
    }
    if (p.tensor != kTensorNone) return dispatch_planes<T, kFamMaxOutputs, -1, true>(p, smem, grid, ty, tx, s);
    return p.n_outputs == 1 ? dispatch_planes<T, 1>(p, smem, grid, ty, tx, s)
                            : dispatch_planes<T, kFamMaxOutputs>(p, smem, grid, ty, tx, s);
}

template <typename T>
int dispatch_work_n(const FamParams &p, size_t smem, int grid, const FamWork *work, int n_work, int n_tiles,
                    int tile_base, int *counter, cudaStream_t s) {
    return p.n_outputs == 1 ? dispatch_work<T, 1>(p, smem, grid, work, n_work, n_tiles, tile_base, counter, s)
                            : dispatch_work<T, kFamMaxOutputs>(p, smem, grid, work, n_work, n_tiles, tile_base,
                                                               counter, s);
}

// Per input type: one launch of the family kernels (the bodies of
// launch_family_planes / _batch / _work for T), instantiated in
// filter_family_<type>.cu.
template <typename T>
int planes_t(const FamParams &p, void *stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int ty = (p.H + kTH - 1) / kTH, tx = (p.W + kTW - 1) / kTW;
    int64_t total = (int64_t)ty * tx * p.B;
    if (total == 0) return 0;
    size_t smem = family_smem_bytes(p.rmax0, p.rmax1);
    int grid = (int)(total < (int64_t)sm_count() * 64 ? total : (int64_t)sm_count() * 64);
    return dispatch_planes_n<T>(p, smem, grid, ty, tx, s);
}

template <typename T>
int batch_t(const FamParams &p, const FamImage *items_dev, int32_t n_items, int32_t n_tiles, void *stream) {
    if (n_tiles == 0) return 0;
    const size_t smem = family_smem_bytes(p.rmax0, p.rmax1);
    return dispatch_batch_r<T>(p, smem, items_dev, n_items, n_tiles, static_cast<cudaStream_t>(stream));
}

template <typename T>
int work_t(const FamParams &p, const FamWork *work_dev, int32_t n_work, int32_t n_tiles_total, int32_t tile_base,
           int32_t *counter_dev, int32_t persistent_ctas, void *stream) {
    if (n_tiles_total == 0) return 0;
    size_t smem = family_smem_bytes(p.rmax0, p.rmax1);
    int grid = counter_dev ? persistent_ctas : n_tiles_total;
    return dispatch_work_n<T>(p, smem, grid, work_dev, n_work, n_tiles_total, tile_base, counter_dev,
                              static_cast<cudaStream_t>(stream));
}

#define LUCEM_FAMILY_DECLARE(T, SFX)                                                                             \
    int planes_##SFX(const FamParams &p, void *stream);                                                         \
    int batch_##SFX(const FamParams &p, const FamImage *items_dev, int32_t n_items, int32_t n_tiles,             \
                    void *stream);                                                                              \
    int work_##SFX(const FamParams &p, const FamWork *work_dev, int32_t n_work, int32_t n_tiles_total,          \
                   int32_t tile_base, int32_t *counter_dev, int32_t persistent_ctas, void *stream);
LUCEM_FAMILY_DECLARE(uint8_t, u8)
LUCEM_FAMILY_DECLARE(uint16_t, u16)
LUCEM_FAMILY_DECLARE(float, f32)
#undef LUCEM_FAMILY_DECLARE

}  // namespace famk
}  // namespace lucem
