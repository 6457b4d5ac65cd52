// rl_pass.cuh -- the Richardson-Lucy pass kernels' shared definitions: pass
// descriptors (ColPass, RowPass and their batch items), pad maps and the
// register-resident column and row pass kernels with their launchers.
// rl.cu drives them; the power-of-two launchers are instantiated per length
// in rl_fast_*.cu (one translation unit each, so they compile in parallel).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fft.cuh"
#include "fft_fast.cuh"
#include "internal.h"

namespace lucem {
namespace rlp {
using fft::cadd;
using fft::cmul;
using fft::csub;

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
    int period = max(2 * len - 2, 1);
    int r = ((p % period) + period) % period;
    return r < len ? r : period - r;
}

__device__ __forceinline__ int pad_index_rt(int p, int len, int mode) {
    switch (mode) {
    case LUCEM_PAD_CONSTANT: return pad_index<LUCEM_PAD_CONSTANT>(p, len);
    case LUCEM_PAD_NEAREST: return pad_index<LUCEM_PAD_NEAREST>(p, len);
    case LUCEM_PAD_WRAP: return pad_index<LUCEM_PAD_WRAP>(p, len);
    case LUCEM_PAD_MIRROR: return pad_index<LUCEM_PAD_MIRROR>(p, len);
    default: return pad_index<LUCEM_PAD_REFLECT>(p, len);
    }
}

enum ColMode : int { kColFwd = 0, kColInv = 1, kColFull = 2 };

// One transform along a strided axis over many columns.  Column c maps to
// (outer = c / Hx, kx = c % Hx); element (row, c) sits at
// outer*outer_stride + row*row_stride + kx.  Forward output rows are in the
// plan's digit-reversed order and inverse input rows are expected in it.
struct ColPass {
    int32_t ncols, Hx;
    const float2 *src;
    int64_t src_outer, src_row;
    int32_t n_img, halo;          // forward load: row j <- src row pad(j - halo, n_img)
    float2 *dst;
    int64_t dst_outer, dst_row;
    int32_t store_begin, store_count;
    int32_t mode;                 // ColMode
    int32_t pad_mode;
    const float2 *H;              // transfer function (kColFull)
    int64_t h_outer, h_row;
    int32_t conj_h;
    float2 *spec_out;             // kColFull: also store the forward spectrum here, or null:
    int64_t spec_row;             // [outer * h_outer + row * spec_row + kx] (the dense layout)
    const float2 *Hrow;           // kColFull, separable transfer function: the factor along the
                                  // transformed axis (natural order); H then holds the other
                                  // axes' product and h_row is 0.  Null: H is dense.
    FftPlan plan;
    const float2 *tw;             // e^{-2 pi i m / n}, m < n
    int32_t C, CP;
    // Volumes sharing one transfer function (bdiv > 0): outer index o splits
    // into volume v = o / bdiv and o' = o % bdiv; src, dst and spec_out are
    // offset by v times src_b, dst_b, spec_b and o' takes the place of o.
    // bdiv == 0: one volume.
    int32_t bdiv;
    int64_t src_b, dst_b, spec_b;
    // Batch mode (items != null): the launch covers several problems of the
    // same transform length; tile t belongs to the last item whose
    // tile_begin <= t, and that item's fields replace the ones above.
    const struct ColItem *items;
    int32_t n_items, total_tiles, use_h2;
};

// One problem of a batched column pass (the per-problem fields of ColPass).
struct ColItem {
    const float2 *src;
    float2 *dst;
    const float2 *H, *H2;         // H2: the second transfer function (use_h2)
    float2 *spec_out;
    int64_t src_outer, src_row, dst_outer, dst_row, h_outer, h_row;
    int32_t ncols, Hx, n_img, halo, store_begin, store_count;
    int32_t tile_begin, pad_;
};

__device__ __forceinline__ ColItem col_view(const ColPass &p) {
    ColItem v;
    v.src = p.src; v.dst = p.dst; v.H = p.H; v.H2 = p.H; v.spec_out = p.spec_out;
    v.src_outer = p.src_outer; v.src_row = p.src_row; v.dst_outer = p.dst_outer; v.dst_row = p.dst_row;
    v.h_outer = p.h_outer; v.h_row = p.h_row;
    v.ncols = p.ncols; v.Hx = p.Hx; v.n_img = p.n_img; v.halo = p.halo;
    v.store_begin = p.store_begin; v.store_count = p.store_count;
    v.tile_begin = 0; v.pad_ = 0;
    return v;
}

// Largest i with tile_begin(i) <= t (items sorted by tile_begin).
template <class Item>
__device__ __forceinline__ int find_item(const Item *items, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].tile_begin <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Element offsets of column `outer` (before kx and the row term): source,
// destination, transfer function and spectrum output.
struct ColOffsets {
    int64_t src, dst, h, spec;
};
__device__ __forceinline__ ColOffsets col_offsets(const ColPass &p, const ColItem &q, int outer) {
    int v = 0, o = outer;
    if (p.bdiv > 0) {
        v = outer / p.bdiv;
        o = outer - v * p.bdiv;
    }
    ColOffsets r;
    r.src = v * p.src_b + o * q.src_outer;
    r.dst = v * p.dst_b + o * q.dst_outer;
    r.h = o * q.h_outer;
    r.spec = v * p.spec_b + o * q.h_outer;
    return r;
}

// The problem and local tile of global tile t.
__device__ __forceinline__ ColItem col_tile(const ColPass &p, int t, int *local) {
    if (p.items == nullptr) {
        *local = t;
        return col_view(p);
    }
    ColItem v = p.items[find_item(p.items, p.n_items, t)];
    if (p.use_h2) v.H = v.H2;
    *local = t - v.tile_begin;
    return v;
}

// Fast column pass for power-of-two lengths N = N1 * N2 (fft_fast.cuh):
// each thread loads its N2 values straight from global memory (lanes along
// columns: coalesced), transforms in registers with one shared-memory
// exchange per direction, multiplies by H in registers and stores back.
// PR (chosen at launch for zero padding to at least twice the data):
// bit 1, the input rows N/2 .. N-1 are zero (not loaded, first forward
// stage pruned); bit 2, only the rows below N/2 are stored (last inverse
// stage pruned).
// Rows t + N1 i (i < N2; i < N2 / 2 when the upper half is zero) of one
// column, extended by the pass's pad map: row j holds source row
// pad(j - halo) for j < n_img + 2 halo, zero beyond.  Zero padding takes a
// branch of its own outside the unrolled loop (one unsigned range check per
// row): the pad map's mode switch per element made up 15% of the 128-point
// pass's instructions.
template <int N1, int N2, bool ZERO_HI>
__device__ __forceinline__ void col_load_rows(const ColPass &p, const ColItem &q, const float2 *src, int t, bool ok,
                                              float2 *v) {
    const int src_row = (int)q.src_row;
    if (p.pad_mode == LUCEM_PAD_CONSTANT) {
#pragma unroll
        for (int i = 0; i < N2; ++i) {
            if (ZERO_HI && i >= N2 / 2) continue;  // rows >= N/2: zero, never read
            const int sr = t + N1 * i - q.halo;
            v[i] = (ok && (unsigned)sr < (unsigned)q.n_img) ? src[sr * src_row] : make_float2(0.f, 0.f);
        }
        return;
    }
    const int n_ext = q.n_img + 2 * q.halo;
#pragma unroll
    for (int i = 0; i < N2; ++i) {
        if (ZERO_HI && i >= N2 / 2) continue;
        const int row = t + N1 * i;
        const int srow = row < n_ext ? pad_index_rt(row - q.halo, q.n_img, p.pad_mode) : -1;
        v[i] = (ok && srow >= 0) ? src[srow * src_row] : make_float2(0.f, 0.f);
    }
}

// The input rows of global tile gt held by thread (c, t) (col_load_rows).
template <int N1, int N2, int C, bool ZERO_HI>
__device__ __forceinline__ void col_load_input(const ColPass &p, int gt, int t, int c, float2 *v) {
    int tile;
    const ColItem q = col_tile(p, gt, &tile);
    const int col = tile * C + c;
    const bool ok = col < q.ncols;
    int outer = 0, kx = 0;
    if (ok) {
        outer = col / q.Hx;
        kx = col - outer * q.Hx;
    }
    const float2 *src = q.src + (col_offsets(p, q, outer).src + kx);
    col_load_rows<N1, N2, ZERO_HI>(p, q, src, t, ok, v);
}

// PR bit 4 (with bit 1, forward and full modes): the next tile's input rows
// are loaded into registers before the current tile's transforms, so their
// memory latency overlaps the arithmetic.
template <int N1, int N2, int C, bool SEP, int PR, int MODE>
__global__ void __launch_bounds__(N1 * C, (N2 > 32 ? 1 : 65536 / (N1 * C * 128))) col_fast_kernel(const __grid_constant__ ColPass p) {
    constexpr bool kZeroHi = (PR & 1) != 0, kLoOnly = (PR & 2) != 0;
    constexpr bool kPrefetch = (PR & 4) != 0 && kZeroHi && MODE != kColInv;
    // MODE: the pass's ColMode (p.mode), fixed at compile time.
    using L = fftc::ColLayout<N1, N2, C>;
    using F = fftc::TwoStep<N1, N2, L>;
    constexpr int N = N1 * N2;
    extern __shared__ float4 smem4[];
    float2 *tf = reinterpret_cast<float2 *>(smem4);
    float2 *ti = tf + N;
    float2 *xb = ti + N;
    // Separable full pass: the axis factor (N complex, natural order) staged
    // once per CTA after the exchange buffer (launch_col_fast sizes it).
    float2 *hrs = xb + L::kBuf;
    const int tid = threadIdx.x, c = tid % C, t = tid / C;
    F::build_tables(tf, ti, p.tw, 1);
    if (SEP && MODE == kColFull)
        for (int i = tid; i < N; i += N1 * C) hrs[i] = p.Hrow[i];
    __syncthreads();
    const int ntiles = p.items ? p.total_tiles : (p.ncols + C - 1) / C;
    float2 nx[kPrefetch ? N2 / 2 : 1];
    if constexpr (kPrefetch) {
        if (blockIdx.x < ntiles) col_load_input<N1, N2, C, true>(p, blockIdx.x, t, c, nx);
    }
    for (int gt = blockIdx.x; gt < ntiles; gt += gridDim.x) {
        int tile;
        const ColItem q = col_tile(p, gt, &tile);
        // Element offsets within one column fit 32 bits (checked by the host).
        const int src_row = (int)q.src_row, dst_row = (int)q.dst_row, h_row = (int)q.h_row;
        const int col = tile * C + c;
        const bool ok = col < q.ncols;
        int outer = 0, kx = 0;
        if (ok) {
            outer = col / q.Hx;
            kx = col - outer * q.Hx;
        }
        const ColOffsets off = col_offsets(p, q, outer);
        const float2 *src = q.src + (off.src + kx);
        float2 v[N2];
        if (MODE == kColInv) {
#pragma unroll
            for (int j = 0; j < N2; ++j) v[j] = ok ? src[F::freq(t, j) * src_row] : make_float2(0.f, 0.f);
            F::template inverse<kLoOnly>(v, t, c, xb, ti);
        } else {
            const float2 *h = q.H + (off.h + kx);
            // Short transforms prefetch the transfer function with the data
            // (one memory round trip per tile instead of two).
            constexpr bool kPrefetchH = N2 <= 16;
            float2 hv[kPrefetchH ? N2 : 1];
            // SEP: separable transfer function (ColPass::Hrow), chosen at launch.
            float2 hc = make_float2(0.f, 0.f);
            // Null H with SEP: the transformed axis's factor is the whole
            // transfer function (no column factor).
            if (SEP && MODE == kColFull && ok && q.H) hc = h[0];
            if (kPrefetchH && MODE == kColFull && !SEP) {
#pragma unroll
                for (int j = 0; j < (kPrefetchH ? N2 : 1); ++j)
                    hv[j] = ok ? h[F::freq(t, j) * h_row] : make_float2(0.f, 0.f);
            }
            if constexpr (kPrefetch) {
#pragma unroll
                for (int i = 0; i < N2 / 2; ++i) v[i] = nx[i];
                if (gt + (int)gridDim.x < ntiles) col_load_input<N1, N2, C, true>(p, gt + gridDim.x, t, c, nx);
            } else {
                col_load_rows<N1, N2, kZeroHi>(p, q, src, t, ok, v);
            }
            F::template forward<kZeroHi>(v, t, c, xb, tf);
            if (MODE == kColFull && q.spec_out != nullptr && ok) {
                float2 *so = q.spec_out + (off.spec + kx);
#pragma unroll
                for (int j = 0; j < N2; ++j) so[F::freq(t, j) * (int)p.spec_row] = v[j];
            }
            if (MODE == kColFwd) {
                float2 *dst = q.dst + (off.dst + kx);
                if (ok) {
#pragma unroll
                    for (int j = 0; j < N2; ++j) dst[F::freq(t, j) * dst_row] = v[j];
                }
                continue;
            }
#pragma unroll
            for (int j = 0; j < N2; ++j) {
                float2 hj;
                // Separable: the row factor here, the column's constant factor
                // after the inverse, on the stored values only (it commutes).
                if constexpr (SEP) hj = hrs[F::freq(t, j)];
                else if constexpr (kPrefetchH) hj = hv[j];
                else hj = ok ? h[F::freq(t, j) * h_row] : make_float2(0.f, 0.f);
                if (p.conj_h) hj.y = -hj.y;
                v[j] = fftc::mul(v[j], hj);
            }
            F::template inverse<kLoOnly>(v, t, c, xb, ti);
            if constexpr (SEP) {
                if (q.H) {
                    if (p.conj_h) hc.y = -hc.y;
#pragma unroll
                    for (int i = 0; i < N2; ++i)
                        if (!(kLoOnly && i >= N2 / 2)) v[i] = fftc::mul(v[i], hc);
                }
            }
        }
        float2 *dst = q.dst + (off.dst + kx);
        if (ok) {
            constexpr int kRows = kLoOnly ? N / 2 : N;  // rows computed
            if (q.store_begin == 0 && q.store_count == kRows) {
                // Every computed row is stored: no per-row range checks.
#pragma unroll
                for (int i = 0; i < N2; ++i)
                    if (!(kLoOnly && i >= N2 / 2)) dst[(t + N1 * i) * dst_row] = v[i];
            } else {
#pragma unroll
                for (int i = 0; i < N2; ++i) {
                    if (kLoOnly && i >= N2 / 2) continue;  // not computed, not stored
                    const int row = t + N1 * i - q.store_begin;
                    if (row >= 0 && row < q.store_count) dst[row * dst_row] = v[i];
                }
            }
        }
    }
}

// Row pass kinds: the RL iteration's three (start from the constant 0.5,
// ratio, update) and the plain transforms (a real array in, or out).
// The reverse pass adds four fused kinds:
//   RatioKeep  c in: store c (est), r = y / guard(c) out (y from obs);
//   Cbar       rbar in: cbar = -rbar y / guard(c)^2 (0 where guarded) out,
//              ybar += rbar / guard(c) when aux2 is given (c from aux);
//   Abar       a in: store a (est), abar = ebar * e out (ebar from aux, e from obs);
//   Ebar       t in: ebar = ebar * a + t in place (ebar aux2, a aux), nothing out.
enum RowKind : int {
    kRowInit = 0, kRowRatio = 1, kRowUpdate = 2, kRowRealIn = 3, kRowRealOut = 4, kRowRatioKeep = 5, kRowCbar = 6,
    kRowAbar = 7, kRowEbar = 8
};

// The x axis: C2R, the Richardson-Lucy epilogue on the image columns, the x
// extension and R2C, for C rows per tile.
struct RowPass {
    int32_t nrows, X, Px, M, Hx, Hp, hx;
    int32_t pad_mode;
    int32_t kind;                 // RowKind
    const float *obs;             // [nrows][X]        (ratio; real input of RealIn)
    float *est;                   // [nrows][X]        (update; real output of RealOut)
    int32_t est_first, last, clip;
    float eps;
    float2 *s1;                   // [nrows][Hp]
    FftPlan plan;                 // M-point
    const float2 *tw;             // table of length Px
    int32_t C, CP;
    const float *aux;             // [nrows][X]: c (Cbar)
    float *aux2;                  // [nrows][X]: ybar, accumulated (Cbar; may be null)
    // Batch mode (items != null): problems of the same Px; the item's fields
    // replace nrows, X, hx, obs, est and s1.
    const struct RowItem *items;
    int32_t n_items, total_tiles;
};

struct RowItem {
    float2 *s1;
    const float *obs;
    float *est;
    int32_t nrows, X, hx, tile_begin;
};

__device__ __forceinline__ RowItem row_tile(const RowPass &p, int t, int *local) {
    if (p.items == nullptr) {
        *local = t;
        RowItem v;
        v.s1 = p.s1; v.obs = p.obs; v.est = p.est;
        v.nrows = p.nrows; v.X = p.X; v.hx = p.hx; v.tile_begin = 0;
        return v;
    }
    const RowItem v = p.items[find_item(p.items, p.n_items, t)];
    *local = t - v.tile_begin;
    return v;
}

// Fast row pass for packed lengths M = N1 * N2 (powers of two): R rows per
// CTA, lanes along the row (coalesced), the M-point transforms in registers.
// ZP (chosen at launch): the real row's data and extension fit the first
// half (X + 2 hx <= Px / 2), so the packed samples m >= M/2 are zero going
// into the forward transform and unused coming out of the inverse one.
template <int N1, int N2, int R, bool ZP, int KIND>
__global__ void __launch_bounds__(N1 * R, 65536 / (N1 * R * 128)) row_fast_kernel(const __grid_constant__ RowPass p) {
    // KIND >= 0: the row kind fixed at compile time (the ratio and update
    // passes of every iteration); -1: kind at run time.
    const int kind = KIND >= 0 ? KIND : p.kind;
    using L = fftc::RowLayout<N1, N2, R>;
    using F = fftc::TwoStep<N1, N2, L>;
    constexpr int M = N1 * N2, Px = 2 * M;
    constexpr int SP = M + 1;  // spectrum row pitch (complex)
    constexpr int U = (L::kBuf > R * SP ? L::kBuf : R * SP);
    extern __shared__ float4 smem4[];
    float2 *tws = reinterpret_cast<float2 *>(smem4);  // W_Px^m, m < Px
    float2 *tf = tws + Px;                              // W_M tables (fft_fast.cuh)
    float2 *ti = tf + M;
    float2 *xb = ti + M;                                // exchange / spectrum / real rows
    const int tid = threadIdx.x, t = tid % N1, r = tid / N1;
    for (int i = tid; i < Px; i += N1 * R) tws[i] = p.tw[i];
    F::build_tables(tf, ti, p.tw, 2);  // W_M^m = W_Px^{2m}
    __syncthreads();
    const int ntiles = p.items ? p.total_tiles : (p.nrows + R - 1) / R;
    const bool emit_last = !(kind == kRowUpdate && p.last) && kind != kRowRealOut && KIND != kRowEbar;
    for (int gt = blockIdx.x; gt < ntiles; gt += gridDim.x) {
        int tile;
        const RowItem pi = row_tile(p, gt, &tile);
        const int row = tile * R + r;
        const bool ok = row < pi.nrows;
        float2 *spec = xb + r * SP;
        float2 v[N2];
        if (kind != kRowInit && kind != kRowRealIn) {
            const float2 *s1 = pi.s1 + (int64_t)(ok ? row : 0) * p.Hp;
            // The half spectrum straight into the inverse transform's layout
            // (slot j of thread t holds bin freq(t, j); lanes along t:
            // coalesced), every load issued before any use.  The merge
            //   Z[k] = (X[k] + X*[M-k]) + i (X[k] - X*[M-k]) W_Px^{-k}
            // takes X[M-k] from the mirror thread N1 - t of the same row
            // (a shuffle within the warp), thread 0 from its own slots and
            // X[M] (one more load).
#pragma unroll
            for (int j = 0; j < N2; ++j) v[j] = ok ? s1[F::freq(t, j)] : make_float2(0.f, 0.f);
            const float2 xM = (ok && t == 0) ? s1[M] : make_float2(0.f, 0.f);
            const unsigned lane = threadIdx.x & 31u, src = (lane & ~(unsigned)(N1 - 1)) | ((N1 - t) & (N1 - 1));
            float2 z[N2];
#pragma unroll
            for (int j = 0; j < N2; ++j) {
                const int jm = F::mirror_slot(j), j0 = F::mirror_slot0(j);
                float2 xm;
                xm.x = __shfl_sync(0xffffffffu, v[jm].x, src);
                xm.y = __shfl_sync(0xffffffffu, v[jm].y, src);
                if (t == 0) xm = j == 0 ? xM : v[j0];
                const int k = F::freq(t, j);
                const float2 xk = v[j];
                const float2 xmc = fftc::conjf2(xm);
                const float2 e = fftc::add(xk, xmc), d = fftc::mul(fftc::sub(xk, xmc), fftc::conjf2(tws[k]));
                z[j] = make_float2(e.x - d.y, e.y + d.x);
            }
#pragma unroll
            for (int j = 0; j < N2; ++j) v[j] = z[j];
            F::template inverse<ZP>(v, t, r, xb, ti);
        }
        // v[i] = (x[2m], x[2m+1]), m = t + N1 i.  Epilogue on the image
        // columns, 8 values of m at a time: all loads of a chunk are issued
        // before its stores (the image pointers do not alias).
        {
            const int64_t gbase = (int64_t)(ok ? row : 0) * pi.X;
            const float *__restrict__ obs = pi.obs;
            float *__restrict__ est = pi.est;
            constexpr int CH = N2 < 8 ? N2 : 8;
#pragma unroll
            for (int i0 = 0; i0 < N2; i0 += CH) {
                float in[2 * CH];
#pragma unroll
                for (int q = 0; q < 2 * CH; ++q) {
                    const int xi = 2 * (t + N1 * (i0 + q / 2)) + (q & 1) - pi.hx;
                    const bool inside = ok && xi >= 0 && xi < pi.X;
                    in[q] = 0.0f;
                    if ((kind == kRowRatio || kind == kRowRealIn || KIND == kRowRatioKeep || KIND == kRowCbar ||
                         KIND == kRowAbar) &&
                        inside)
                        in[q] = obs[gbase + xi];
                    if (kind == kRowUpdate && !p.est_first && inside) in[q] = est[gbase + xi];
                }
#pragma unroll
                for (int q = 0; q < 2 * CH; ++q) {
                    const int i = i0 + q / 2;
                    const int xi = 2 * (t + N1 * i) + (q & 1) - pi.hx;
                    const bool inside = xi >= 0 && xi < pi.X;
                    const float val = (q & 1) ? v[i].y : v[i].x;
                    float nv = 0.0f;
                    if (inside) {
                        if (kind == kRowInit) {
                            nv = 0.5f;
                        } else if (kind == kRowRealIn) {
                            nv = in[q];
                        } else if (kind == kRowRealOut) {
                            nv = val;
                        } else if (kind == kRowRatio) {
                            const float d = fabsf(val) < p.eps ? p.eps : val;
                            nv = in[q] / d;
                        } else if (KIND == kRowRatioKeep) {
                            const float d = fabsf(val) < p.eps ? p.eps : val;
                            nv = in[q] / d;
                            if (ok) est[gbase + xi] = val;
                        } else if (KIND == kRowCbar) {
                            const float ci = p.aux[gbase + xi];
                            const bool gd = fabsf(ci) < p.eps;
                            const float d = gd ? p.eps : ci;
                            nv = gd ? 0.0f : -val * in[q] / (d * d);
                            if (p.aux2 && ok) p.aux2[gbase + xi] += val / d;
                        } else if (KIND == kRowAbar) {
                            if (ok) est[gbase + xi] = val;
                            nv = p.aux[gbase + xi] * in[q];
                        } else if (KIND == kRowEbar) {
                            nv = fmaf(p.aux2[gbase + xi], p.aux[gbase + xi], val);
                            if (ok) p.aux2[gbase + xi] = nv;
                        } else {
                            const float old = p.est_first ? 0.5f : in[q];
                            nv = old * val;
                            if (p.last && p.clip) nv = fminf(fmaxf(nv, -1.0f), 1.0f);
                        }
                    }
                    if (q & 1) v[i].y = nv; else v[i].x = nv;
                }
                if ((kind == kRowUpdate || kind == kRowRealOut) && ok) {
#pragma unroll
                    for (int q = 0; q < 2 * CH; ++q) {
                        const int i = i0 + q / 2;
                        const int xi = 2 * (t + N1 * i) + (q & 1) - pi.hx;
                        if (xi >= 0 && xi < pi.X) est[gbase + xi] = (q & 1) ? v[i].y : v[i].x;
                    }
                }
            }
        }
        if (!emit_last) continue;
        if (pi.hx > 0) {
            // Extension along x by the pad map: positions outside
            // [hx, hx + X) take image samples, past X + 2 hx zero.
            float *real = reinterpret_cast<float *>(spec);
#pragma unroll
            for (int i = 0; i < N2; ++i) {
                const int m = t + N1 * i;
                real[2 * m] = v[i].x;
                real[2 * m + 1] = v[i].y;
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < N2; ++i) {
                const int m = t + N1 * i;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int pos = 2 * m + e;
                    if (pos >= pi.hx && pos < pi.hx + pi.X) continue;
                    float nv = 0.0f;
                    if (pos < pi.X + 2 * pi.hx) {
                        int q = pad_index_rt(pos - pi.hx, pi.X, p.pad_mode);
                        if (q >= 0) nv = real[q + pi.hx];
                    }
                    if (e) v[i].y = nv; else v[i].x = nv;
                }
            }
            __syncthreads();
        }
        F::template forward<ZP>(v, t, r, xb, tf);
        // Split, in registers: X[k] = 1/2 (Z[k] + Z*[M-k]) - i/2 W_Px^k
        // (Z[k] - Z*[M-k]) with Z[M] = Z[0]; Z[M-k] from the mirror thread
        // (thread 0: its own slots), X[M] from Z[0] by thread 0.
        {
            const unsigned lane = threadIdx.x & 31u, src = (lane & ~(unsigned)(N1 - 1)) | ((N1 - t) & (N1 - 1));
            float2 *s1 = pi.s1 + (int64_t)(ok ? row : 0) * p.Hp;
            float2 xM = make_float2(0.f, 0.f);
#pragma unroll
            for (int j = 0; j < N2; ++j) {
                const int jm = F::mirror_slot(j), j0 = F::mirror_slot0(j);
                float2 zm;
                zm.x = __shfl_sync(0xffffffffu, v[jm].x, src);
                zm.y = __shfl_sync(0xffffffffu, v[jm].y, src);
                if (t == 0) zm = v[j0];
                const int k = F::freq(t, j);
                const float2 zk = v[j];
                const float2 zmc = fftc::conjf2(zm);
                const float2 e = fftc::add(zk, zmc), d = fftc::mul(fftc::sub(zk, zmc), tws[k]);
                if (j == 0 && t == 0) {
                    // X[M] = 1/2 (Z[0] + Z*[0]) - i/2 W_Px^M (Z[0] - Z*[0]).
                    const float2 zkc = fftc::conjf2(zk);
                    const float2 e2 = fftc::add(zk, zkc), d2 = fftc::mul(fftc::sub(zk, zkc), tws[M]);
                    xM = make_float2(0.5f * (e2.x + d2.y), 0.5f * (e2.y - d2.x));
                }
                if (ok) s1[k] = make_float2(0.5f * (e.x + d.y), 0.5f * (e.y - d.x));
            }
            if (ok && t == 0) s1[M] = xM;
        }
    }
    (void)U;
}

inline int sms() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

template <int N1, int N2, int C>
int launch_col_fast(const ColPass &p, cudaStream_t s) {
    using L = fftc::ColLayout<N1, N2, C>;
    constexpr int N = N1 * N2;
    // Twiddle tables, the exchange buffer and (separable full pass) the axis factor.
    const size_t hrow = (p.Hrow && p.mode == kColFull) ? (size_t)N : 0;
    size_t smem = ((size_t)2 * N + (size_t)L::kBuf + hrow) * sizeof(float2);
    int ntiles = p.items ? p.total_tiles : (p.ncols + C - 1) / C;
    int per_sm = (int)((200 * 1024) / (smem + 1024));
    per_sm = per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
    int grid = ntiles < sms() * per_sm ? ntiles : sms() * per_sm;
    // Pruning needs the zero rows / the unstored rows to be the upper half of
    // every column (single problems only: a batch's items differ).
    const int N_ = N1 * N2;
    int pr = 0;
    if (!p.items && p.mode != kColInv && p.n_img + 2 * p.halo <= N_ / 2) pr |= 1;
    if (!p.items && p.mode != kColFwd && p.store_begin >= 0 && p.store_begin + p.store_count <= N_ / 2) pr |= 2;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, N1 * C, smem, s>>>(p);
    };
    // One instantiation per pass mode; pruning only where the mode allows it
    // (forward: the zero input half; inverse: the unstored output half;
    // forward * H * inverse: both or neither).
    if (p.mode == kColFwd) {
        if (pr & 1) go(col_fast_kernel<N1, N2, C, false, 1, kColFwd>);
        else go(col_fast_kernel<N1, N2, C, false, 0, kColFwd>);
    } else if (p.mode == kColInv) {
        if (pr & 2) go(col_fast_kernel<N1, N2, C, false, 2, kColInv>);
        else go(col_fast_kernel<N1, N2, C, false, 0, kColInv>);
    } else if (p.Hrow) {
        // The 128-point separable full pass loads the next tile ahead (PR
        // bit 4): 238 against 246 us per launch on the 64x512x512 volume.
        // The same prefetch in the forward pass measured slower; the other
        // lengths keep the plain loads.
        if (pr == 3) {
            if constexpr (N1 * N2 == 128) go(col_fast_kernel<N1, N2, C, true, 7, kColFull>);
            else go(col_fast_kernel<N1, N2, C, true, 3, kColFull>);
        } else {
            go(col_fast_kernel<N1, N2, C, true, 0, kColFull>);
        }
    } else {
        if (pr == 3) go(col_fast_kernel<N1, N2, C, false, 3, kColFull>);
        else go(col_fast_kernel<N1, N2, C, false, 0, kColFull>);
    }
    return (int)cudaGetLastError();
}

template <int N1, int N2, int R>
int launch_row_fast(const RowPass &p, cudaStream_t s) {
    using L = fftc::RowLayout<N1, N2, R>;
    constexpr int M = N1 * N2;
    constexpr int U = L::kBuf > R * (M + 1) ? L::kBuf : R * (M + 1);
    size_t smem = ((size_t)2 * M + 2 * (size_t)M + (size_t)U) * sizeof(float2);
    int ntiles = p.items ? p.total_tiles : (p.nrows + R - 1) / R;
    int per_sm = (int)((200 * 1024) / (smem + 1024));
    per_sm = per_sm < 1 ? 1 : (per_sm > 8 ? 8 : per_sm);
    int grid = ntiles < sms() * per_sm ? ntiles : sms() * per_sm;
    // Pruning for single problems only (a batch's items differ in X).
    const bool zp = !p.items && p.X + 2 * p.hx <= p.Px / 2;
    auto go = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, N1 * R, smem, s>>>(p);
    };
    // The two passes of every iteration get kernels compiled for their kind.
    if (p.kind == kRowRatio) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowRatio>);
        else go(row_fast_kernel<N1, N2, R, false, kRowRatio>);
    } else if (p.kind == kRowUpdate) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowUpdate>);
        else go(row_fast_kernel<N1, N2, R, false, kRowUpdate>);
    } else if (p.kind == kRowRatioKeep) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowRatioKeep>);
        else go(row_fast_kernel<N1, N2, R, false, kRowRatioKeep>);
    } else if (p.kind == kRowCbar) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowCbar>);
        else go(row_fast_kernel<N1, N2, R, false, kRowCbar>);
    } else if (p.kind == kRowAbar) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowAbar>);
        else go(row_fast_kernel<N1, N2, R, false, kRowAbar>);
    } else if (p.kind == kRowEbar) {
        if (zp) go(row_fast_kernel<N1, N2, R, true, kRowEbar>);
        else go(row_fast_kernel<N1, N2, R, false, kRowEbar>);
    } else {
        if (zp) go(row_fast_kernel<N1, N2, R, true, -1>);
        else go(row_fast_kernel<N1, N2, R, false, -1>);
    }
    return (int)cudaGetLastError();
}

// Per-length launchers of the register-resident passes (rl_fast_*.cu).
int launch_col_64_256(int n, const ColPass &p, cudaStream_t s);
int launch_col_512(const ColPass &p, cudaStream_t s);
int launch_col_1024(const ColPass &p, cudaStream_t s);
int launch_col_2048(const ColPass &p, cudaStream_t s);
int launch_row_64_256(int m, const RowPass &p, cudaStream_t s);
int launch_row_512(const RowPass &p, cudaStream_t s);
int launch_row_1024(const RowPass &p, cudaStream_t s);

}  // namespace rlp
}  // namespace lucem
