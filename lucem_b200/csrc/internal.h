// internal.h -- shared declarations of the lucem_b200 implementation (host
// C++ and CUDA).  Not part of the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "lucem_b200.h"

namespace lucem {

// Kernels index with 32-bit integers: crates/lucem-core/src/compute/limits.rs:12.
constexpr int64_t kMaxDeviceElements = 0xFFFFFFFFll;

// ---- separable filters -------------------------------------------------

// Largest radius the fused 2-D family kernel takes per axis (65 taps); wider
// filters run as per-axis passes.  The kernel is compiled for the even radii
// 0, 2, ..., 16, 20, 24, 28, 32; a filter of another radius runs at the next
// one up with zero taps at both ends (fam_kernel_radius).
constexpr int kFamMaxRadius = 32;
constexpr int kFamTile = 64;  // output tile side of the family kernels
constexpr int kFamMaxTaps = 2 * kFamMaxRadius + 1;
constexpr int kFamMaxFilters = 8;
constexpr int kFamMaxOutputs = 4;
constexpr int kFamTapStride = 66;  // tap pairs per filter axis (>= 2 * kFamMaxRadius + 1)

inline int fam_kernel_radius(int r) {
    if (r <= 0) return 0;
    if (r <= 16) return (r + 1) & ~1;
    return (r + 3) & ~3;
}

struct float2_ { float x, y; };

enum class Combine : int32_t { kLinear = 0, kHypot = 1 };

struct FamOutput {
    float *out;        // f32 [B, H, W] (plane/row strides below)
    int64_t plane_stride;
    int64_t row_pitch;
    int32_t combine;   // Combine
    int32_t fa, fb;    // filter indices (fb < 0: single term)
    float alpha, beta, bias;
    // fa or fb == -2 names the input sample itself (unsharp).
};

// Launch-setting bits of FamParams::plan (plan = 1 + bits).
constexpr int32_t kPlanAhead = 1;   // copy the next tile's window ahead (tensor copy / cp.async)
constexpr int32_t kPlanOneCta = 2;  // one persistent CTA per SM (else as many as fit)

// Epilogue modes of FamParams::tensor (tensor_ops.cuh); 0: none, the
// linear outputs.
enum TensorMode : int32_t {
    kTensorNone = 0,
    kTensorDet = 1,        // out0 = a c - b^2
    kTensorEigvals = 2,    // out0 = l1, out1 = l2 (l1 >= l2)
    kTensorShapeIndex = 3, // out0 = shape index of (l1, l2)
    kTensorFrangi = 4,     // out0 = max(out0, frangi(l1, l2)); p0 = 1/(2 beta^2), p1 = 1/(2 c^2)
    kTensorSato = 5,       // out0 = max(out0, sato(l1 sigma^2, l2 sigma^2)); p0 = sigma^2
    kTensorMeijering = 6,  // out0 = max(out0, meijering(l1, l2))
    kTensorOuter = 7,      // (a, b) = (g_r, g_c): out0 = a a, out1 = a b, out2 = b b
    kTensorScaledSum = 8,  // out0 = p0 (a + p1 b), each step rounded (LoG / DoG responses)
    kTensorScaledDet = 9,  // out0 = p0 (a c - b^2) (determinant-of-Hessian response)
    kTensorCannyGrad = 10, // (a, b) = (g_r, g_c): out0 = |g|, out1 = the direction sector 0..3 (as f32)
};

// One launch of the fused 2-D family kernel over B planes of [H, W] (or over
// work items of a slide, see FamWork).
struct FamParams {
    const void *in;
    int64_t in_plane_stride;
    int64_t in_row_pitch;
    int32_t B, H, W;
    int32_t mode;
    float cval;
    float in_scale;
    int32_t n_filters;
    int32_t n_outputs;
    int32_t rmax0, rmax1;          // largest kernel radius per axis over the filters
    int32_t r0[kFamMaxFilters];    // kernel radius (fam_kernel_radius), axis 0 (rows)
    int32_t r1[kFamMaxFilters];    // kernel radius, axis 1 (columns)
    FamOutput outs[kFamMaxOutputs];
    // Taps as (w, w) pairs for the packed f32x2 FMA, 2 r + 1 per filter axis,
    // zero padded from the filter's own radius to its kernel radius.
    float2_ taps0[kFamMaxFilters][kFamTapStride];
    float2_ taps1[kFamMaxFilters][kFamTapStride];
    // Bounded waits of the TMA-staged blur: give up on a tensor copy after
    // wait_ns nanoseconds (0: the default, one second; -1: at once, without
    // polling), count each give-up in *wait_status (may be null).
    int32_t *wait_status;
    // Launch settings: 0 = the built-in heuristics; else 1 + kPlan* bits,
    // chosen by the autotuner.
    int32_t plan;
    int64_t wait_ns;
    // Tensor epilogue (tensor_ops.cuh TensorMode; 0: none): the first three
    // filters' responses (a, b, c) are combined per pixel into outs[0..2]
    // instead of the linear outputs.  tensor_black: the ridge modes' dark
    // ridges; tensor_first: the ridge modes start their running maximum at 0
    // instead of reading the output.
    int32_t tensor, tensor_black, tensor_first;
    float tensor_p0, tensor_p1;
};

// One tile of a batched walk: the read box of one channel and the owned box
// inside it (absolute slide coordinates).
struct FamWork {
    int32_t channel;
    int32_t read_y, read_x, read_h, read_w;
    int32_t own_y, own_x, own_h, own_w;
    int32_t tile_begin;   // first CTA tile index of this item in the flattened list
};

// One image of a batch of separate 2-D images (lucem_gaussian_batch).
struct FamImage {
    const void *in;               // [H][in_pitch] of the input dtype
    float *out;                   // [H][out_pitch]
    int64_t in_pitch, out_pitch;  // elements
    int32_t H, W;
    int32_t tile_begin;           // first 64x64 tile of this image in the batch
    int32_t pad_;
};

// Launchers (filter.cu).  All return cudaGetLastError() as int.
int launch_family_planes(const FamParams &p, int in_dtype, void *stream);
// Tiles [tile_base, tile_base + n_tiles) of the work list (global tile
// indices); with counter_dev the launch is persistent (persistent_ctas CTAs).
// Every 64x64 tile of n_items images with the same filter set (p's filters,
// one output: combine, alpha, bias from p.outs[0]; its pointer unused).
int launch_family_batch(const FamParams &p, int in_dtype, const FamImage *items_dev, int32_t n_items,
                        int32_t n_tiles, void *stream);
int launch_family_work(const FamParams &p, int in_dtype, const FamWork *work_dev, int32_t n_work,
                       int32_t n_tiles, int32_t tile_base, int32_t *counter_dev,
                       int32_t persistent_ctas, void *stream);
int family_tile_dims(int *th, int *tw);
size_t family_smem_bytes(int rmax0, int rmax1);

// Generic 1-D correlation along one axis of an [outer, len, inner] view.
int launch_correlate_1d(const void *in, int in_dtype, float in_scale, float *out, int64_t outer,
                        int64_t len, int64_t inner, const float *w_dev, int32_t size, int32_t left,
                        int32_t mode, float cval, void *stream);
// Halo part of the adjoint of launch_correlate_1d (f32 in): out[pad(p)] +=
// scale * sum_t w[t] g[p + left - t] over the extended positions p outside
// [0, len).  No-op for the constant mode.
int launch_adjoint_fold(const float *g, float scale, float *out, int64_t outer, int64_t len, int64_t inner,
                        const float *w_dev, int32_t size, int32_t left, int32_t mode, void *stream);
// out = alpha*a + beta*b + bias (b may be null: beta ignored).
int launch_linear_comb(const float *a, const float *b, float *out, int64_t n, float alpha,
                       float beta, float bias, void *stream);
// acc += d*d
int launch_add_sq(const float *d, float *acc, int64_t n, void *stream);
// out = sqrt(max(acc,0)) * scale
int launch_sqrt_scale(const float *acc, float *out, int64_t n, float scale, void *stream);
// out = (float)in * scale (u8/u16/f32 -> f32)
int launch_cast(const void *in, int in_dtype, float scale, float *out, int64_t n, void *stream);
int launch_fill(float *out, int64_t n, float v, void *stream);
// tens::apply (tensor_ops.cuh) per element: (a, b, c) -> o0 (o1, o2), mode a
// TensorMode; c may be null (outer products); first: the ridge modes'
// running maximum starts at 0 instead of o0.
int launch_tensor_elementwise(const float *a, const float *b, const float *c, float *o0, float *o1, float *o2,
                              int64_t n, int mode, float p0, float p1, int black, int first, void *stream);

// features.cu: resampling on the resize grid (order 0 nearest, 1 bilinear;
// the input sampled at (m0 oy + m2, m4 ox + m5), pad map outside).
int launch_resample(const float *in, int H, int W, float *out, int OH, int OW, float m0, float m2, float m4,
                    float m5, int order, int mode, float cval, void *stream);
// features.cu: Canny's non-maximum suppression (nms, and the maximum of mag
// as non-negative float bits in *max_bits, to be zeroed first), its default
// thresholds on the device (thr[0] low, thr[1] high), and its hysteresis by
// connected components: edges = 1 on the components of (nms >= low) that
// hold a pixel with nms >= high (labels: H W scratch); the thresholds from
// thr when it is not null, else low / high.
int launch_canny_nms(const float *mag, const float *sector, float *nms, int H, int W, unsigned int *max_bits,
                     void *stream);
int launch_canny_thresholds(const unsigned int *max_bits, int quantiles, double *thr, void *stream);
int launch_canny_hysteresis(const float *nms, int H, int W, const double *thr, double low, double high,
                            uint32_t *labels, uint32_t *edges, void *stream);
// features.cu: scale-space maxima of the blob detectors.
struct BlobCandidate {
    float response;
    int32_t s, y, x;
};
// Upper bound of the maxima of an ns x H x W stack (no two are neighbours).
int64_t blob_candidate_bound(int ns, int64_t H, int64_t W);
// Appends the strict 3x3x3 maxima above `threshold` outside the border to
// out (at most cap written) and counts them in *count (to be zeroed first).
int launch_blob_candidates(const float *cube, int ns, int H, int W, int border, double threshold,
                           BlobCandidate *out, int64_t cap, unsigned long long *count, void *stream);

// ---- Gaussian planning shared by the entry points (api.cpp) ---------------

// One 1-D pass of a separable Gaussian (crates/lucem-ops/src/filter/gaussian.rs:204-219).
struct GaussPass {
    int axis;
    double sigma;
    uint32_t order;
    int64_t radius;
};

// Every check lucem_gaussian_blur makes, then its pass list.
lucem_status gaussian_blur_plan(const lucem_tensor *in, const double *sigmas, int32_t n_sigmas,
                                const lucem_gaussian_settings *settings, const lucem_tensor *out,
                                std::vector<GaussPass> *passes);
// True when the last two passes are the two innermost axes (ascending) and
// both fit the fused 2-D kernel.
bool gaussian_fuse_last_two(const lucem_tensor *in, const std::vector<GaussPass> &passes);
// f32 taps of one pass.
std::vector<float> gaussian_pass_taps(const GaussPass &p);
// Fused 2-D launch parameters for one separable filter over the last two
// axes of `view` into `out`.
void gaussian_fused_params(FamParams *fp, const lucem_tensor *view, int mode, double cval, float scale,
                           const GaussPass &rows, const GaussPass &cols, float *out);
// Records `msg` as the calling thread's last error and returns `st`.
lucem_status set_error(lucem_status st, const char *msg);

// ---- per-kernel timing ---------------------------------------------------

enum PassKind : int {
    kPassRlRow = 0,      // row pass: C2R, RL epilogue, R2C
    kPassRlColFwd,       // column pass, forward transform
    kPassRlColFull,      // column pass, forward * H * inverse
    kPassRlColInv,       // column pass, inverse transform
    kPassRlOtf,          // transfer-function build
    kPassFamily,         // fused 2-D Gaussian family
    kPassCorrelate,      // per-axis correlation
    kPassElementwise,    // combine / cast / fill
    kPassRlColY,         // separable PSF: y convolution on the row spectra (forward * Hy * inverse)
    kPassRlColZ,         // separable PSF: z convolution on the row spectra (forward * Hz * inverse)
    kPassFft,            // general complex FFT along one axis
    kPassCount
};
const char *pass_name(int kind);

// Brackets launches with events when a workspace has timing enabled.
struct PassTimer {
    virtual ~PassTimer() = default;
    virtual void begin(int kind, void *stream) = 0;
    virtual void end(int kind, void *stream) = 0;
};

// ---- FFT / Richardson-Lucy ---------------------------------------------

constexpr int kFftMaxStages = 16;

struct FftPlan {
    int32_t n;
    int32_t nstages;
    int32_t radix[kFftMaxStages];
};

bool fft_make_plan(int64_t n, FftPlan *plan);
int64_t fft_good_length(int64_t n, bool even);

// One axis pass of the general complex FFT (spectral.cu): every line (O, k),
// O < n_outer, k < inner, of length n.  Element `row` of line (O, k) sits at
// base(O) + k + row * rs with base(O) = (O / odiv) os_hi + (O % odiv) os_lo
// (odiv <= 1: O os_hi), for the source (s_*) and the destination (d_*).
// Source: split (sre, sim; sim null: zero imaginary part) or interleaved sc.
// Destination: split (dre, dim; dim null: imaginary part dropped) or dc.
// src_rows / dst_rows: rows read (the rest zero) / written.  Options: pre
// (per input row), mid (between a forward and a backward transform, the
// Bluestein filter), post (per output row), twiddle W_twiddle_n^(m2 row) with
// m2 = k / tw_div (four-step), conjugation in / out, scale, clip to [-1, 1]
// (split real output).  C, CP: set by the launcher.
constexpr int kFftLinesMax = 8192;  // longest line transformed in shared memory
struct FftLines {
    const float *sre, *sim;
    const float2_ *sc;
    float *dre, *dim;
    float2_ *dc;
    int64_t n_outer, inner;
    int32_t s_odiv, d_odiv;
    int64_t s_os_hi, s_os_lo, s_rs;
    int64_t d_os_hi, d_os_lo, d_rs;
    int32_t n, src_rows, dst_rows, inverse;
    FftPlan plan;
    const float2_ *tw, *pre, *mid, *post, *tw_big;
    int32_t twiddle_n;
    int64_t tw_div;
    float scale;
    int32_t conj_in, conj_out, clip;
    int32_t C, CP;
};
int launch_fft_lines(FftLines p, void *stream);
int launch_dft_direct(const FftLines &p, void *stream);
int launch_wiener_filter(const float2_ *y, const float2_ *h, const float2_ *l, float2_ *x, int64_t n, float balance,
                         float eps, void *stream);
int launch_complex_mul(const float *ar, const float *ai, const float *br, const float *bi, float *outr, float *outi,
                       int64_t n, int conj_b, void *stream);
int launch_centre_kernel(const float *k, int kh, int kw, float2_ *out, int H, int W, void *stream);

// spectral_ops.cu: per-axis spectral filters, Butterworth, phase
// correlation and unsupervised Wiener on the FFTs above.
constexpr int kRedBlocks = 148 * 8;  // most blocks of one reduction launch
constexpr int kCandBlocks = 148;     // blocks per candidate of the phase-correlation refinement sums
struct float4_ { float x, y, z, w; };
// Axes of a C-contiguous array of < 2^32 elements: bin k_d = (e / inner[d])
// % len[d]; off[d]: the axis's table in a concatenated f32 table (phase: the
// cos table, then the sin table).
struct SpecAxes {
    int32_t ndim, phase;
    uint32_t len[8], inner[8], off[8];
};
// Device state of one phase correlation: shift per axis, the peak's
// cross-correlation value and flat index.
struct PcState {
    double shift[8];
    double peak_re, peak_im;
    uint32_t max_idx, pad_;
};
// Device state of one unsupervised Wiener chain.
struct UwState {
    double balance, img_var;
    uint64_t rng;
};
int launch_spectral_axes(float *re, float *im, int64_t n, const float *tab, const SpecAxes &a, void *stream);
int launch_butterworth(float2_ *X, int64_t n, const SpecAxes &a, double cutoff, double order, int high_pass,
                       void *stream);
int launch_phase_cross_power(const float2_ *A, const float2_ *B, float2_ *R, int64_t n, int normalize, void *stream);
int launch_phase_argmax(const float2_ *X, int64_t n, const SpecAxes &a, float *pv, uint32_t *pi, PcState *st,
                        void *stream);
int launch_phase_refine_axis(const float2_ *R, int64_t n, const SpecAxes &a, int ax, int radius, double step,
                             double2 *oth, double2 *axt, double2 *part, PcState *st, void *stream);
int launch_phase_error_terms(const float *ref, const float *mov, const float2_ *A, const float2_ *B, int64_t n,
                             const SpecAxes &a, const PcState *st, int want_cc, double *part, double *out,
                             void *stream);
int launch_uw_setup(const float *in, const float2_ *Y, const float2_ *H, const float2_ *L, float4_ *P, int64_t n,
                    uint64_t seed, double *part, UwState *st, double2 *mean, void *stream);
int launch_uw_iteration(const float2_ *Y, const float2_ *H, const float4_ *P, int64_t n, int accumulate,
                        double2 *mean, double *part, UwState *st, double *chain, int it, void *stream);
int launch_uw_mean(const double2 *mean, int64_t n, double inv_count, float2_ *X, void *stream);


// Geometry of one RL problem on its FFT grid.  Axes are (z, y, x); 2-D inputs
// have Z = Pz = 1.
struct RlGeom {
    int32_t ndim;
    int32_t Z, Y, X;         // image
    int32_t Pz, Py, Px;      // grid
    int32_t hz, hy, hx;      // extension halo per axis (0 for zero padding)
    int32_t Hx;              // Px/2 + 1
    int32_t Hp;              // spectrum row pitch (complex elements)
    int32_t mode;
    int32_t nb;              // volumes sharing the PSF, stored one after another (0 or 1: one)
};

struct RlBuffers {
    void *s1;      // complex [Z][Y][Hp]
    void *s2;      // complex [Z][Py][Hp] (3-D only)
    const void *h_conv;  // complex [Pz][Py][Hp]
    const void *h_corr;  // complex [Pz][Py][Hp] (may equal h_conv)
    // Separable PSF: h_conv / h_corr hold the product of the factors of all
    // axes but the last transformed one ([Py][Hp] in 3-D, [Hp] in 2-D) and
    // hrow_* that factor ([Pz] in 3-D, [Py] in 2-D).  Null: dense transfer
    // functions.
    const void *hrow_conv, *hrow_corr;
    // Separable 3-D PSF, per-axis factors: y ([Py]) and x times 1/(Pz Py Px)
    // ([Hp]).  With them a convolution without a spectrum output runs as a
    // y convolution and a z convolution on s1 (no s2 round trip).  Null
    // otherwise.
    const void *hy_conv, *hy_corr, *hx_conv, *hx_corr;
    const float2_ *tw_x, *tw_y, *tw_z;  // twiddle tables e^{-2 pi i k / n}, n = Px, Py, Pz
};

int rl_launch_iterations(const RlGeom &g, const RlBuffers &b, const float *obs, float *est_out,
                         int32_t num_iter, int32_t clip, float eps, void *stream, PassTimer *timer);
// out = H x (conj 0) or conj(H) x (conj 1) over the image region, zero
// padding (the geometry's mode must be constant).  Uses b.s1 / b.s2.
int rl_apply(const RlGeom &g, const RlBuffers &b, const void *H, int conj, const float *x, float *out,
             void *stream, PassTimer *timer);

// Scratch of the reverse passes (device pointers; V = Z*Y*X floats per
// volume, S = Pz*Py*Hp complex per spectrum).
struct RlBwdBuffers {
    float *ckpt;                  // ceil(T/K) volumes
    float *seg;                   // K volumes
    float *c, *r, *a, *abar, *rbar, *cbar, *t, *ebar;  // one volume each
    float2_ *spec_e, *spec_r, *spec_abar, *spec_cbar;  // one spectrum each
    float2_ *pbar1, *pbar2;       // PSF cross-spectrum accumulators (pbar2: even sides only)
    void *full_s1, *full_s2;      // complex [Pz][Py][Hp] (full-grid inverse)
    float *full_real;             // [Pz][Py][Px]
    int32_t kdims[3], c_conv[3], c_corr[3];
};

// Reverse mode of rl_launch_iterations (clip off, zero padding): from
// d loss / d (estimate after T iterations) `ebar_T`, writes the PSF gradient
// at the convolution centre (gpsf_conv) and, when the two centres differ,
// the correlation's share at its centre (gpsf_corr; null otherwise), and
// d loss / d obs into ybar (optional).  Checkpoints every K iterations.
int rl_backward(const RlGeom &g, const RlBuffers &b, const RlBwdBuffers &w, const float *y, int T, int K,
                float eps, const float *ebar_T, float *gpsf_conv, float *gpsf_corr, float *ybar, void *stream,
                PassTimer *timer);
// Gradients of out = conv(psf, x): gx (optional) and gpsf (optional, at the
// convolution centre).  Uses w.c, w.t, w.spec_e, w.spec_cbar, w.pbar1, full_*.
int rl_convolve_backward(const RlGeom &g, const RlBuffers &b, const RlBwdBuffers &w, const float *x,
                         const float *gout, float *gx, float *gpsf, void *stream, PassTimer *timer);
// ---- batched 2-D Richardson-Lucy -------------------------------------------

// Tiles per launch unit of the column pass (columns) and of the row pass
// (rows) for a transform length; the host uses them to lay out work lists.
int col_tile_width(int n);
int row_tile_rows(int M);

// One problem of a batched column pass (device layout of the kernels' item).
struct RlColItem {
    const float2_ *src;
    float2_ *dst;
    const float2_ *H, *H2;        // convolution / correlation transfer functions
    float2_ *spec_out;
    int64_t src_outer, src_row, dst_outer, dst_row, h_outer, h_row;
    int32_t ncols, Hx, n_img, halo, store_begin, store_count;
    int32_t tile_begin, pad_;
};
// One problem of a batched row pass.
struct RlRowItem {
    float2_ *s1;
    const float *obs;
    float *est;
    int32_t nrows, X, hx, tile_begin;
};
// Problems that share a transform length n: their items (device array,
// sorted by tile_begin) and the length's twiddle table.
struct RlBatchGroup {
    int32_t n;
    const void *items;
    int32_t n_items, total_tiles;
    const float2_ *tw;
};
struct RlBatchLaunch {
    int32_t mode;
    const RlBatchGroup *rows;     // grouped by Px
    int32_t n_rows;
    const RlBatchGroup *cols;     // grouped by Py
    int32_t n_cols;
};
int rl_tune_pass(int kind, int n, int lines, void *a, void *b, const float2_ *tw, int reps, void *stream,
                 float *ms);
int rl_batch_iterations(const RlBatchLaunch &L, int num_iter, int clip, float eps, void *stream, PassTimer *timer);

// OTF of the normalised PSF `psf_dev` (f64 [kz][ky][kx]) centred at `centre`,
// scaled by 1/(Pz*Py*Px), into complex [Pz][Py][Hp] (f32).  Work buffers are
// f64 complex of size kz*ky*Hp and kz*Py*Hp.
int rl_launch_otf(const RlGeom &g, const double *psf_dev, const int32_t kdims[3],
                  const int32_t centre[3], double *work_a, double *work_b, void *h_out,
                  const double *twd_x, const double *twd_y, const double *twd_z, void *stream);

}  // namespace lucem
