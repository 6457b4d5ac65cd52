/*
 * lucem_b200.h -- C ABI of the B200 (sm_100a) implementation of lucem-ops'
 * separable Gaussian family and Richardson-Lucy deconvolution.
 *
 * This is the layer a Rust `extern "C"` block in lucem-core binds in place of
 * the CubeCL launches for these operations.  Every entry point cites the
 * reference interface it replaces (paths inside neuro-kitchen/lucem).
 *
 * Conventions
 *  - Tensors are C-contiguous device arrays described by lucem_tensor (data
 *    pointer, element type, dims), as lucem-core's DeviceArray
 *    (crates/lucem-core/src/memory/array.rs:21-27).  The caller owns them.
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *    Launches are asynchronous on it; only functions that say so synchronise.
 *  - Scratch comes from a lucem_workspace: named slots that only grow, as
 *    lucem-core's Workspace (crates/lucem-core/src/memory/workspace.rs:10-52).
 *    A workspace serves one thread of work at a time.
 *  - A context is bound to one device; constant data (Gaussian taps, PSF
 *    transfer functions) lives in its mutex-guarded cache, as DeviceCache
 *    (crates/lucem-core/src/memory/cache.rs:19-44).
 *  - Return codes mirror OpsError / CoreError
 *    (crates/lucem-ops/src/error.rs:9-59, crates/lucem-core/src/error.rs:8-38);
 *    lucem_last_error_message() gives the text of the calling thread's last
 *    error.  No C++ exception crosses this boundary.
 *  - Element counts are capped at 2^32-1 per buffer, as
 *    crates/lucem-core/src/compute/limits.rs:12.
 *  - Empty inputs return LUCEM_OK with no work, as the reference does.
 */
#ifndef LUCEM_B200_H
#define LUCEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUCEM_B200_ABI_VERSION 1
#define LUCEM_MAX_DIMS 8

typedef enum lucem_status {
    LUCEM_OK = 0,
    LUCEM_ERR_SHAPE_MISMATCH = 1,       /* OpsError::ShapeMismatch */
    LUCEM_ERR_ALIASED_BUFFERS = 2,      /* OpsError::AliasedBuffers */
    LUCEM_ERR_INVALID_DIMENSION = 3,    /* OpsError::InvalidDimension */
    LUCEM_ERR_UNKNOWN_PAD_MODE = 4,     /* OpsError::UnknownPadMode */
    LUCEM_ERR_INVALID_ORIGIN = 5,       /* OpsError::InvalidOrigin */
    LUCEM_ERR_INVALID_WEIGHTS = 6,      /* OpsError::InvalidWeights */
    LUCEM_ERR_INVALID_PARAMETER = 7,    /* OpsError::InvalidParameter */
    LUCEM_ERR_EMPTY_INPUT = 8,          /* OpsError::EmptyInput */
    LUCEM_ERR_AXIS_OUT_OF_BOUNDS = 9,   /* CoreError::AxisOutOfBounds */
    LUCEM_ERR_REPEATED_AXIS = 10,       /* CoreError::RepeatedAxis */
    LUCEM_ERR_TOO_MANY_ELEMENTS = 11,   /* CoreError::TooManyElements */
    LUCEM_ERR_OUT_OF_DEVICE_MEMORY = 12,/* CoreError::OutOfDeviceMemory */
    LUCEM_ERR_UNSUPPORTED_DTYPE = 13,   /* element type not accepted by the op */
    LUCEM_ERR_CUDA = 14,                /* a CUDA runtime call failed */
    LUCEM_ERR_DEVICE_TIMEOUT = 15,      /* a bounded device wait gave up */
    LUCEM_ERR_INVALID_HANDLE = 16       /* NULL / foreign context or workspace */
} lucem_status;

/* LUCEM_U32: label and edge maps only (lucem_canny's output); every other
 * entry point refuses it as an unsupported element type. */
typedef enum lucem_dtype { LUCEM_U8 = 1, LUCEM_U16 = 2, LUCEM_F32 = 3, LUCEM_U32 = 4 } lucem_dtype;

/* crates/lucem-ops/src/core/pad.rs:84-88 (same ids). */
typedef enum lucem_pad_mode {
    LUCEM_PAD_REFLECT = 0,  /* d c b a | a b c d | d c b a */
    LUCEM_PAD_CONSTANT = 1, /* k k k k | a b c d | k k k k */
    LUCEM_PAD_NEAREST = 2,  /* a a a a | a b c d | d d d d */
    LUCEM_PAD_MIRROR = 3,   /*   d c b | a b c d | c b a   */
    LUCEM_PAD_WRAP = 4      /* a b c d | a b c d | a b c d */
} lucem_pad_mode;

typedef struct lucem_tensor {
    void *data;     /* device pointer, C-contiguous */
    int32_t dtype;  /* lucem_dtype */
    int32_t ndim;   /* 0..LUCEM_MAX_DIMS */
    int64_t dims[LUCEM_MAX_DIMS];
} lucem_tensor;

typedef struct lucem_ctx lucem_ctx;
typedef struct lucem_workspace lucem_workspace;

/* ---- library, context, workspace ------------------------------------- */

int32_t lucem_abi_version(void);
/* Text of the calling thread's last error ("" if none). */
const char *lucem_last_error_message(void);
/* crates/lucem-core/src/device.rs:23-189 (ComputeTarget + client) reduced to
 * "one CUDA device": binds `device`, reads its SM count. */
lucem_status lucem_ctx_create(int32_t device, lucem_ctx **out);
void lucem_ctx_destroy(lucem_ctx *ctx);
/* crates/lucem-core/src/memory/workspace.rs:21-52. */
lucem_status lucem_workspace_create(lucem_ctx *ctx, lucem_workspace **out);
void lucem_workspace_destroy(lucem_workspace *ws);
size_t lucem_workspace_capacity_bytes(const lucem_workspace *ws);
/* Per-kernel device timing, the analogue of the pipeline's EvalTimings
 * (engine/lucem-pipeline/src/eval.rs:59-71): while enabled, every kernel the
 * workspace's calls launch is bracketed by CUDA events.  lucem_workspace_timings
 * synchronises on those events and reports, per kernel kind, the launches and
 * the summed device milliseconds since timing was (re)enabled; names are
 * written as NUL-terminated strings of at most 31 chars in a [cap][32] array. */
lucem_status lucem_workspace_set_timing(lucem_workspace *ws, int32_t enable);
lucem_status lucem_workspace_timings(lucem_workspace *ws, char *names, double *ms, int64_t *launches,
                                     int32_t cap, int32_t *n_out);
/* Bounded device waits.  No counterpart in the reference (it has no device
 * waits).  The TMA-staged plain 2-D blur (the fused kernel for launches of at
 * least 12 tiles per SM) waits for each tile's tensor copy at most `ns`
 * nanoseconds (default one second; 0: give up at once, for tests), then loads
 * that tile directly: results are the same either way.  A CTA never exits
 * with a copy still in flight into its shared memory (it waits for it, at
 * most two seconds more).  lucem_workspace_wait_status synchronises `stream`,
 * returns the number of waits that gave up since the last call in *gave_up
 * and clears it; LUCEM_ERR_DEVICE_TIMEOUT when that number is not zero. */
lucem_status lucem_workspace_set_wait_limit(lucem_workspace *ws, int64_t ns);
lucem_status lucem_workspace_wait_status(lucem_workspace *ws, void *stream, int64_t *gave_up);
/* Parses a pad-mode name with the reference's aliases
 * (crates/lucem-ops/src/core/pad.rs:46-56); LUCEM_ERR_UNKNOWN_PAD_MODE else. */
lucem_status lucem_pad_mode_parse(const char *name, int32_t *mode_out);

/* ---- host-side helpers (no device work) ------------------------------ */

/* crates/lucem-ops/src/filter/gaussian.rs:22-63: writes 2*radius+1 f64 taps. */
lucem_status lucem_gaussian_kernel_1d(double sigma, uint32_t order, int64_t radius, double *out);
/* crates/lucem-ops/src/filter/gaussian.rs:83-85: floor(truncate*sigma+0.5). */
int64_t lucem_gaussian_radius(double truncate, double sigma);
/* crates/lucem-ops/src/core/kernels/pad.rs:11-34 (-1 = constant fill). */
int64_t lucem_pad_index(int64_t p, int64_t len, int32_t mode);

/* ---- Gaussian family ------------------------------------------------- */

/* crates/lucem-ops/src/filter/gaussian.rs:133-156 (GaussianBlur), plus the
 * input scale of uint_to_unit_float (crates/lucem-ops/src/core/elementwise.rs
 * :205-230) for integer inputs: value = (float)raw * input_scale. */
typedef struct lucem_gaussian_settings {
    const uint32_t *orders; int32_t n_orders;   /* broadcast per axis; {0} when n_orders == 0 */
    int32_t mode;                               /* lucem_pad_mode */
    double cval;
    double truncate;                            /* 4.0 */
    const int64_t *radii; int32_t n_radii;      /* None when n_radii == 0 */
    const int64_t *axes; int32_t n_axes;        /* None (all axes) when axes == NULL */
    int32_t has_channel_axis; int64_t channel_axis;
    double input_scale;                         /* 1.0 */
} lucem_gaussian_settings;
void lucem_gaussian_settings_default(lucem_gaussian_settings *s);

/* crates/lucem-ops/src/filter/gaussian.rs:176-237 gaussian_blur_into.
 * in: u8 | u16 | f32 (the cast is fused into the load); out: f32, same dims. */
lucem_status lucem_gaussian_blur(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                 int32_t n_sigmas, const lucem_gaussian_settings *settings,
                                 lucem_tensor *out, lucem_workspace *ws, void *stream);

/* The adjoint (transpose) of lucem_gaussian_blur's linear map in -> out with
 * the same sigmas and settings: grad_in = A^T grad_out, where out = A in + b
 * (b: the cval term of the constant mode).  It is the backward pass of
 * gaussian_blur for reverse-mode differentiation; the reference has no
 * counterpart (its filters are not differentiable).  f32 gradient in and
 * out; every pad mode (halo reads fold back onto the samples they came from). */
lucem_status lucem_gaussian_blur_adjoint(lucem_ctx *ctx, const lucem_tensor *grad_out, const double *sigmas,
                                         int32_t n_sigmas, const lucem_gaussian_settings *settings,
                                         lucem_tensor *grad_in, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/gaussian.rs:66-118 (Gaussian1d, gaussian_1d_into).
 * radius < 0 means None. */
typedef struct lucem_gaussian_1d_settings {
    int64_t axis; uint32_t order; int32_t mode; double cval; double truncate; int64_t radius;
} lucem_gaussian_1d_settings;
void lucem_gaussian_1d_settings_default(lucem_gaussian_1d_settings *s);
lucem_status lucem_gaussian_1d(lucem_ctx *ctx, const lucem_tensor *in, double sigma,
                               const lucem_gaussian_1d_settings *settings, lucem_tensor *out,
                               void *stream);

/* crates/lucem-ops/src/filter/convolve.rs:17-92 (Correlate1d, correlate_1d):
 * host f64 weights, cast to f32 and cached per context. */
typedef struct lucem_correlate_1d_settings {
    int64_t axis; int32_t mode; double cval; int32_t origin;
} lucem_correlate_1d_settings;
lucem_status lucem_correlate_1d(lucem_ctx *ctx, const lucem_tensor *in, const double *weights,
                                int64_t n_weights, const lucem_correlate_1d_settings *settings,
                                lucem_tensor *out, void *stream);

/* crates/lucem-ops/src/filter/gaussian.rs:374-390 difference_of_gaussians_into. */
lucem_status lucem_difference_of_gaussians(lucem_ctx *ctx, const lucem_tensor *in,
                                           const double *low_sigmas, int32_t n_low,
                                           const double *high_sigmas, int32_t n_high,
                                           const lucem_gaussian_settings *settings,
                                           lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/gaussian.rs:255-288 gaussian_laplace_into. */
lucem_status lucem_gaussian_laplace(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                    int32_t n_sigmas, int32_t mode, double cval, double truncate,
                                    lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/gaussian.rs:307-356 gaussian_grad_mag_into. */
lucem_status lucem_gaussian_grad_mag(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                     int32_t n_sigmas, int32_t mode, double cval, double truncate,
                                     lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/gaussian.rs:407-421 unsharp_mask_into. */
lucem_status lucem_unsharp_mask(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                int32_t n_sigmas, double amount,
                                const lucem_gaussian_settings *settings, lucem_tensor *out,
                                lucem_workspace *ws, void *stream);

/* Several Gaussian-family responses of one input in one fused pass: the input
 * tile is read once and every response is written from shared memory.  Each
 * response is what the named reference function returns for the same input:
 *   LUCEM_RESP_GAUSSIAN   gaussian_blur(sigma)            (gaussian.rs:176)
 *   LUCEM_RESP_DOG        difference_of_gaussians(sigma, sigma2) (:374)
 *   LUCEM_RESP_LAPLACE    gaussian_laplace(sigma)         (:255)
 *   LUCEM_RESP_GRAD_MAG   gaussian_grad_mag(sigma)        (:307)
 *   LUCEM_RESP_UNSHARP    unsharp_mask(sigma, amount)     (:407)
 * Sigmas are isotropic over the filtered axes (the last two).  This is the
 * per-tile function a lucem-pipeline tile walk calls
 * (engine/lucem-pipeline/src/custom.rs:233-251) when an Op list holds several
 * Gaussian-family ops (engine/lucem-pipeline/src/ops.rs:795-800). */
typedef enum lucem_response_kind {
    LUCEM_RESP_GAUSSIAN = 0, LUCEM_RESP_DOG = 1, LUCEM_RESP_LAPLACE = 2,
    LUCEM_RESP_GRAD_MAG = 3, LUCEM_RESP_UNSHARP = 4
} lucem_response_kind;
typedef struct lucem_response {
    int32_t kind; double sigma; double sigma2; double amount; lucem_tensor out;
} lucem_response;
lucem_status lucem_gaussian_family(lucem_ctx *ctx, const lucem_tensor *in,
                                   const lucem_response *responses, int32_t n_responses,
                                   int32_t mode, double cval, double truncate, double input_scale,
                                   lucem_workspace *ws, void *stream);

/* Allocation-free lucem_gaussian_blur.  No counterpart in the reference.
 * For callers that cannot allocate device memory: a host runtime whose device
 * memory all comes from its own pool under a fixed budget (a cudaMalloc behind
 * its back would escape that accounting or fail because the pool already holds
 * the memory), or a service that must not grow its footprint or synchronise
 * the device with cudaMalloc/cudaFree while it works.  Same arguments, checks
 * and results as lucem_gaussian_blur, minus the context and workspace: the
 * intermediate buffers and taps live in one static device array of the library
 * (2 x 4,194,304 floats + 16,384 taps, about 32 MiB, held by every GPU that
 * loads the library until exit).  Inputs of more than 4,194,304 elements are
 * refused with LUCEM_ERR_TOO_MANY_ELEMENTS.  The first call on a device looks
 * up the array's device address (once per device, on the current device);
 * make that first call before any stream capture.  Every call shares the
 * array: calls that overlap on the GPU race, so serialise them.  No
 * cudaMalloc, cudaFree or allocating library routine is called. */
lucem_status lucem_gaussian_blur_noalloc(const lucem_tensor *in, const double *sigmas, int32_t n_sigmas,
                                         const lucem_gaussian_settings *settings, lucem_tensor *out,
                                         void *stream);

/* ---- tiling and batched tiles ---------------------------------------- */

/* crates/lucem-core/src/tiling.rs:13-49 Block ([z, y, x]). */
typedef struct lucem_block {
    int64_t index;
    int64_t origin[3], size[3];
    int64_t read_origin[3], read_size[3];
} lucem_block;
/* crates/lucem-core/src/tiling.rs:54-78 schedule: writes at most `cap` blocks,
 * sets *n_out to the full count. */
lucem_status lucem_schedule(const int64_t dims[3], const int64_t block[3], const int64_t halo[3],
                            lucem_block *out, int64_t cap, int64_t *n_out);

/* Runs lucem_gaussian_family on every block of every channel of a [C, H, W]
 * slide, as the tile walk does (engine/lucem-pipeline/src/custom.rs:199-251):
 * each block's read part is filtered with the pad mode applied at the read
 * part's borders and only the owned part is written, into [C, H, W] outputs.
 * blocks[] come from lucem_schedule over [1, H, W]; every channel is walked.
 * persistent != 0: one persistent launch walks the whole work list (uneven
 * edge tiles included); persistent == 0: one launch per block and channel (the
 * plain per-tile drop-in). */
lucem_status lucem_gaussian_family_tiles(lucem_ctx *ctx, const lucem_tensor *slide,
                                         const lucem_block *blocks, int64_t n_blocks,
                                         const lucem_response *responses, int32_t n_responses,
                                         int32_t mode, double cval, double truncate,
                                         double input_scale, int32_t persistent,
                                         lucem_workspace *ws, void *stream);

/* ---- Richardson-Lucy ------------------------------------------------- */

/* crates/lucem-ops/src/restore/deconvolve.rs:19-41 (RichardsonLucy) plus the
 * FFT grid.  grid[d] == 0 picks the smallest length with factors 2, 3, 5, 7
 * (even along x) that holds the padded correlation: n + k/2 for
 * LUCEM_PAD_CONSTANT, n + 2*(k/2) for the other modes. */
typedef struct lucem_rl_settings {
    int32_t num_iter;          /* 30 */
    int32_t clip;              /* 1 */
    int32_t has_filter_epsilon; double filter_epsilon; /* None -> 1e-12, floor 1e-15 */
    int32_t mode;              /* LUCEM_PAD_REFLECT; LUCEM_PAD_CONSTANT = zero padding */
    int64_t grid[3];           /* per axis of the input; 0 = automatic */
} lucem_rl_settings;
void lucem_rl_settings_default(lucem_rl_settings *s);

/* crates/lucem-ops/src/restore/deconvolve.rs:45-162 richardson_lucy_into,
 * computed with FFT convolution for 2-D and 3-D f32 inputs.  Every pad mode
 * of the reference is honoured (the correlation input is extended by k/2
 * samples per axis with the pad map; zero padding needs no extension).  The
 * PSF is copied to the host once per call to normalise it (as the reference
 * does at :77), so the call synchronises the stream once before the
 * iterations are queued; its transfer function is cached in the workspace. */
lucem_status lucem_richardson_lucy(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                   const lucem_rl_settings *settings, lucem_tensor *out,
                                   lucem_workspace *ws, void *stream);
/* Reverse mode through lucem_richardson_lucy (the reference's
 * richardson_lucy is not differentiable; no counterpart there): given
 * d loss / d out, writes d loss / d psf (through the PSF normalisation;
 * optional, NULL to skip) and d loss / d in (optional).  The iterations are
 * recomputed from checkpoints kept every `checkpoint_every` iterations
 * (device memory: ceil(T/k) + k + 8 volumes and 5 spectra).  Zero padding
 * (LUCEM_PAD_CONSTANT) and clip off only.  Synchronises the stream (PSF in,
 * PSF gradient out). */
lucem_status lucem_richardson_lucy_backward(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                            const lucem_rl_settings *settings, const lucem_tensor *grad_out,
                                            int32_t checkpoint_every, lucem_tensor *grad_psf,
                                            lucem_tensor *grad_in, lucem_workspace *ws, void *stream);
/* The forward model of richardson_lucy as an operator: out = psf (*) x, the
 * convolution centred at k-1-k/2 per axis, zero padding, the PSF as given
 * (not normalised), 2-D or 3-D f32 on the FFT grid (grid NULL or 0 =
 * automatic).  The reference computes it inside richardson_lucy as
 * correlate with the flipped PSF (crates/lucem-ops/src/restore/deconvolve.rs:120). */
lucem_status lucem_fft_convolve(lucem_ctx *ctx, const lucem_tensor *x, const lucem_tensor *psf, int32_t mode,
                                const int64_t *grid, lucem_tensor *out, lucem_workspace *ws, void *stream);
/* Its reverse mode (no counterpart in the reference): grad_x = A^T grad_out
 * and grad_psf, each optional (NULL to skip). */
lucem_status lucem_fft_convolve_backward(lucem_ctx *ctx, const lucem_tensor *x, const lucem_tensor *psf,
                                         int32_t mode, const int64_t *grid, const lucem_tensor *grad_out,
                                         lucem_tensor *grad_x, lucem_tensor *grad_psf, lucem_workspace *ws,
                                         void *stream);
/* A batch of separate 2-D images of any sizes, each blurred as
 * lucem_gaussian_blur would with the isotropic sigma of its set
 * (set_sigmas[set_ids[i]]), the same mode, cval, truncate and input scale for
 * all: the batched counterpart of calling gaussian_blur_into per image
 * (crates/lucem-ops/src/filter/gaussian.rs:176-237).  Per sigma set, one
 * persistent launch walks the 64x64 tiles of all its images.  ins: n tensors
 * of one dtype (u8, u16 or f32); outs: n f32 tensors of the same shapes.  The
 * image list is uploaded on the first call with a given list (the stream is
 * synchronised then); later calls with the same list only launch.  Kernel
 * radius at most 32 (sigma 8 at truncate 4). */
lucem_status lucem_gaussian_batch(lucem_ctx *ctx, int32_t n, const lucem_tensor *ins, lucem_tensor *outs,
                                  const int32_t *set_ids, int32_t n_sets, const double *set_sigmas, int32_t mode,
                                  double cval, double truncate, double input_scale, lucem_workspace *ws,
                                  void *stream);

/* ---- Batched 2-D Richardson-Lucy --------------------------------------
 * Many 2-D problems of different sizes and PSFs (the reference runs
 * richardson_lucy once per image, crates/lucem-ops/src/restore/
 * deconvolve.rs:45-149).  A plan is built once: each problem gets an FFT
 * grid from a short list of lengths (m * 2^k, m in {1,3,5,7,9,15,21,25,27},
 * the cheapest by the autotuned or default pass costs), its transfer
 * functions and spectrum, and the problems are grouped by length.  A run then
 * issues, per pass of every iteration, one launch per length group (each
 * launch walks the work list of all its problems), and nothing else: no
 * allocation, synchronisation or host copy, so a run can be captured in a
 * CUDA graph.  per_problem = 1 runs the same kernels one problem at a time
 * (the per-image baseline).  Arrays obs, psfs and outs hold n tensors each;
 * the plan keeps their device pointers (they must stay valid).  create
 * synchronises `stream` and allocates the plan's device memory. */
typedef struct lucem_rl_batch lucem_rl_batch;
lucem_status lucem_rl_batch_create(lucem_ctx *ctx, int32_t n, const lucem_tensor *obs, const lucem_tensor *psfs,
                                   const lucem_rl_settings *settings, lucem_tensor *outs, lucem_workspace *ws,
                                   void *stream, lucem_rl_batch **out);
lucem_status lucem_rl_batch_run(lucem_rl_batch *batch, int32_t per_problem, lucem_workspace *timing_ws,
                                void *stream);
/* grids: 2 per problem (Py, Px); launches per row / column pass. */
lucem_status lucem_rl_batch_info(const lucem_rl_batch *batch, int64_t *grids, int32_t *n_row_launches,
                                 int32_t *n_col_launches);
void lucem_rl_batch_destroy(lucem_rl_batch *batch);

/* ---- Autotuning of FFT lengths (no counterpart in the reference) -------
 * Measures the column pass (kind 0) and row pass (kind 1) at each length
 * (2/3/5/7-smooth) on scratch data and records ns per transformed element in
 * the context; batched plans then choose grid lengths by these costs.  The
 * table can be saved to and loaded from a text file. */
lucem_status lucem_autotune_fft(lucem_ctx *ctx, const int64_t *lengths, int32_t n, lucem_workspace *ws,
                                void *stream);
lucem_status lucem_autotune_query(lucem_ctx *ctx, int32_t kind, int64_t length, double *ns_per_element);
lucem_status lucem_autotune_save(lucem_ctx *ctx, const char *path);
/* Launch settings of the Gaussian family kernels, as the reference tunes its
 * CubeCL launches (crates/lucem-core/src/compute/tune.rs:1-27: candidates
 * benchmarked once per device and problem-size key, the fastest reused).
 * While enabled, the first plain 2-D blur, persistent tile walk or image
 * batch set of each key -- kernel kind, SM count, element type, filter
 * count, largest radius, power-of-two class of the tile count -- times its
 * candidate settings on the call's own data (copying the next tile's window
 * ahead by tensor copy or cp.async or not; one or as many persistent CTAs
 * per SM as fit; every candidate computes the same result), keeps the
 * fastest and launches with it; later calls of the key reuse it.  Tuning synchronises the stream and
 * is skipped during stream capture.  Disabled (the default), cached plans
 * are still used and other keys take the built-in heuristics.  Plans are
 * saved and loaded with the FFT costs ("plan <key> <code>" lines). */
lucem_status lucem_autotune_enable(lucem_ctx *ctx, int32_t enable);
/* The cached plans: keys as NUL-terminated strings of at most 63 chars in a
 * [cap][64] array, codes in plans (1 + bits: 1 copy ahead, 2 one CTA per
 * SM); *n_out = the number cached. */
lucem_status lucem_autotune_plans(lucem_ctx *ctx, char *keys, int32_t *plans, int32_t cap, int32_t *n_out);
lucem_status lucem_autotune_load(lucem_ctx *ctx, const char *path);

/* ---- CUDA graphs of launch-only calls ------------------------------------
 * begin/end bracket a capture of `stream` (not the legacy default stream);
 * only calls that launch without synchronising or allocating may run inside:
 * lucem_rl_batch_run, and the filter entry points once a first call with the
 * same arguments has cached their taps and work lists. */
typedef struct lucem_graph lucem_graph;
lucem_status lucem_graph_begin(void *stream);
lucem_status lucem_graph_end(void *stream, lucem_graph **out);
lucem_status lucem_graph_launch(lucem_graph *graph, void *stream);
void lucem_graph_destroy(lucem_graph *graph);

/* ---- spectral operators -------------------------------------------- */

/* crates/lucem-ops/src/core/fft.rs:55-100 fft_nd_into: N-D forward
 * (inverse = 0, unnormalised) or inverse (inverse scaled by 1/len per axis)
 * DFT over every axis of a split complex f32 array (re_in, im_in) into
 * (re_out, im_out), axes in order, ping/pong through the workspace.  The
 * reference evaluates each axis as a direct O(len^2) DFT (dft_axis_kernel,
 * core/kernels/fft.rs:9-47); here: shared-memory Stockham transforms for
 * 2,3,5,7-smooth lengths up to 8192, four-step beyond, Bluestein for other
 * lengths up to 4096, a direct DFT above that.  0-D or empty arrays are
 * copied. */
lucem_status lucem_fft_nd(lucem_ctx *ctx, const lucem_tensor *re_in, const lucem_tensor *im_in,
                          lucem_tensor *re_out, lucem_tensor *im_out, int32_t inverse, lucem_workspace *ws,
                          void *stream);
/* crates/lucem-ops/src/core/fft.rs:14-53 fft_1d_into: the same along one
 * axis (negative axes count from the end).  The workspace may be NULL except
 * for smooth lengths above 8192 (four-step scratch). */
lucem_status lucem_fft_1d(lucem_ctx *ctx, const lucem_tensor *re_in, const lucem_tensor *im_in,
                          lucem_tensor *re_out, lucem_tensor *im_out, int32_t axis, int32_t inverse,
                          lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/core/fft.rs:104-138 complex_mul_into: out = a * b, or
 * a * conj(b) when conj_b, split complex f32. */
lucem_status lucem_complex_mul(const lucem_tensor *a_re, const lucem_tensor *a_im, const lucem_tensor *b_re,
                               const lucem_tensor *b_im, lucem_tensor *out_re, lucem_tensor *out_im, int32_t conj_b,
                               void *stream);

/* crates/lucem-ops/src/restore/deconvolve.rs:163-183 WienerDeconvolve. */
typedef struct lucem_wiener_settings {
    double balance;            /* 0.1; regularisation weight, finite and >= 0 */
    int32_t clip;              /* 1: clamp the result to [-1, 1] */
} lucem_wiener_settings;
void lucem_wiener_settings_default(lucem_wiener_settings *s);
/* crates/lucem-ops/src/restore/deconvolve.rs:210-295 wiener_deconvolve_into:
 * X = conj(H) Y / max(|H|^2 + balance |L|^2, 1e-12) with Y the FFT of the
 * 2-D f32 input, H that of the PSF centred at (kh/2, kw/2) on the image grid
 * (circular), L that of the discrete Laplacian; out = Re(IFFT(X)), clipped
 * when asked.  Same checks and error kinds as the reference; every FFT is
 * lucem_fft_nd's. */
lucem_status lucem_wiener_deconvolve(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                     const lucem_wiener_settings *settings, lucem_tensor *out, lucem_workspace *ws,
                                     void *stream);

/* crates/lucem-ops/src/filter/spectral.rs:21-63 fourier_gaussian_into: the
 * split complex f32 spectrum (re, im) times exp(-2 pi^2 sigma_d^2 f_d^2) per
 * axis d in place (f_d: the bin's signed normalised frequency); `values`
 * broadcast per axis (1 or ndim values).  All axes in one pass over the
 * array, applied in axis order with the reference's f32 products. */
lucem_status lucem_fourier_gaussian(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *sigmas,
                                    int32_t n_sigmas, void *stream);
/* crates/lucem-ops/src/filter/spectral.rs:66-108 fourier_box_into: times
 * sinc(pi size_d f_d) per axis (1 where |pi size_d f_d| < 1e-12). */
lucem_status lucem_fourier_box(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *sizes,
                               int32_t n_sizes, void *stream);
/* crates/lucem-ops/src/filter/spectral.rs:112-164 fourier_shift_into: times
 * exp(-i 2 pi shift_d f_d) per axis. */
lucem_status lucem_fourier_shift(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *shifts,
                                 int32_t n_shifts, void *stream);
/* crates/lucem-ops/src/filter/spectral.rs:168-213 butterworth: N-D f32 input
 * -> out = Re(IFFT(FFT(in) w)), w = 1 / (1 + (|f| / cutoff_ratio)^(2 order))
 * (low pass) or 1 - that (high_pass); cutoff_ratio in (0, 0.5].  The
 * reference builds w on the host; here it is evaluated per bin in FP64 inside
 * the product kernel. */
lucem_status lucem_butterworth(lucem_ctx *ctx, const lucem_tensor *in, double cutoff_ratio, int32_t high_pass,
                               double order, lucem_tensor *out, lucem_workspace *ws, void *stream);

/* crates/lucem-ops/src/register/phase.rs:18-37 PhaseCorrelation. */
typedef struct lucem_phase_correlation_settings {
    int64_t upsample_factor;   /* 1: integer-pixel; > 1: 1/upsample_factor pixel */
    int32_t normalize_phase;   /* 1: R / |R| (phase correlation); 0: plain cross-correlation */
} lucem_phase_correlation_settings;
void lucem_phase_correlation_settings_default(lucem_phase_correlation_settings *s);
/* crates/lucem-ops/src/register/phase.rs:39-48 PhaseCorrelationResult. */
typedef struct lucem_phase_correlation_result {
    double shift[LUCEM_MAX_DIMS]; /* per axis, the shift registering `moving` onto `reference` */
    double error;                 /* translation-invariant normalised RMS error in [0, 1] */
    double phasediff;             /* global phase difference at the peak, radians */
} lucem_phase_correlation_result;
/* crates/lucem-ops/src/register/phase.rs:51-255 phase_correlation: N-D f32
 * reference and moving images of one shape.  Cross-power spectrum of their
 * FFTs, the |cc|^2 argmax of its inverse (first index on ties), then (when
 * upsample_factor > 1) the reference's coordinate-wise candidate search,
 * two passes, each candidate's sum over the whole spectrum an FP64
 * reduction on the device, and the snap to the 1/upsample_factor grid.
 * Synchronises on `stream` (the result is host data). */
lucem_status lucem_phase_correlation(lucem_ctx *ctx, const lucem_tensor *reference, const lucem_tensor *moving,
                                     const lucem_phase_correlation_settings *settings,
                                     lucem_phase_correlation_result *result, lucem_workspace *ws, void *stream);

/* crates/lucem-ops/src/restore/deconvolve.rs:330-354 UnsupervisedWiener. */
typedef struct lucem_unsupervised_wiener_settings {
    int64_t num_iter;          /* 30 */
    int64_t burnin;            /* 10; < num_iter */
    int32_t clip;              /* 1: clamp the result to [-1, 1] */
    uint64_t seed;             /* 0: the balance jitter's PCG seed */
} lucem_unsupervised_wiener_settings;
void lucem_unsupervised_wiener_settings_default(lucem_unsupervised_wiener_settings *s);
/* crates/lucem-ops/src/restore/deconvolve.rs:357-509 unsupervised_wiener:
 * 2-D f32 input and PSF; the empirical-Bayes chain of the reference (balance
 * from 0.05, per iteration the residual, prior and trace sums at the current
 * balance, the variance update and the PCG jitter), the posterior mean of the
 * spectrum after the burn-in, out = Re(IFFT(mean)) (clipped when asked).
 * Every sum is an FP64 reduction on the device and the balance update runs on
 * the device, so the chain needs no host round trip; `balance_chain` (host,
 * num_iter doubles, may be NULL) receives the balances.  Synchronises on
 * `stream` when balance_chain is given. */
lucem_status lucem_unsupervised_wiener(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                       const lucem_unsupervised_wiener_settings *settings, lucem_tensor *out,
                                       double *balance_chain, lucem_workspace *ws, void *stream);

/* ---- Gaussian-consumer operators ------------------------------------------
 * 2-D input (u8, u16 or f32), f32 outputs of its shape.  Each scale's three
 * Hessian filters (Gaussian derivatives of orders (2,0), (1,1), (0,2),
 * truncate 4) run from one staged tile in one launch of the fused family
 * kernel, with the per-pixel tensor math in its epilogue; filters of radius
 * above 32 take per-axis passes and the same math elementwise. */

/* crates/lucem-ops/src/feature/structure.rs:16-54 hessian_matrix. */
lucem_status lucem_hessian_matrix(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                  lucem_tensor *hrr, lucem_tensor *hrc, lucem_tensor *hcc, lucem_workspace *ws,
                                  void *stream);
/* crates/lucem-ops/src/feature/structure.rs:57-83 hessian_det: H_rr H_cc - H_rc^2. */
lucem_status lucem_hessian_det(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                               lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/feature/structure.rs:86-97 hessian_eigvals: l1 >= l2. */
lucem_status lucem_hessian_eigvals(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                   lucem_tensor *eig1, lucem_tensor *eig2, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/feature/structure.rs:164-191 shape_index (Koenderink). */
lucem_status lucem_shape_index(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                               lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/feature/structure.rs:102-147 structure_tensor: Sobel
 * gradients, their outer products and a Gaussian window of sigma.  Both
 * gradients and the three products in one launch (into the workspace), then
 * the three windows. */
lucem_status lucem_structure_tensor(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                    lucem_tensor *arr, lucem_tensor *arc, lucem_tensor *acc, lucem_workspace *ws,
                                    void *stream);
/* crates/lucem-ops/src/feature/structure.rs:150-161 structure_tensor_eigvals
 * (f32 components in, l1 >= l2 out). */
lucem_status lucem_structure_tensor_eigvals(const lucem_tensor *arr, const lucem_tensor *arc, const lucem_tensor *acc,
                                            lucem_tensor *eig1, lucem_tensor *eig2, void *stream);

/* crates/lucem-ops/src/filter/ridge.rs:13-40 RidgeFilter. */
typedef struct lucem_ridge_settings {
    const double *sigmas; int32_t n_sigmas; /* NULL: {1, 3, 5, 7, 9} */
    int32_t black_ridges;                   /* 1: dark ridges on a bright background */
    int32_t mode;                           /* lucem_pad_mode (reflect) */
    double cval;
    double beta;                            /* 0.5 (Frangi) */
    double gamma;                           /* 15 (Frangi) */
} lucem_ridge_settings;
void lucem_ridge_settings_default(lucem_ridge_settings *s);
/* crates/lucem-ops/src/filter/ridge.rs:87-133 frangi_into: per scale the
 * Hessian eigenvalues, the vesselness and the running maximum, in the
 * scale's one launch. */
lucem_status lucem_frangi(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                          lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/ridge.rs:148-185 sato_into. */
lucem_status lucem_sato(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                        lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/filter/ridge.rs:199-235 meijering_into. */
lucem_status lucem_meijering(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                             lucem_tensor *out, lucem_workspace *ws, void *stream);

/* crates/lucem-ops/src/feature/canny.rs:17-45 Canny. */
typedef struct lucem_canny_settings {
    double sigma;               /* 1; Gaussian pre-smoothing, >= 0 */
    int32_t has_low;            /* 0: low threshold 0.1 max |grad| */
    double low_threshold;
    int32_t has_high;           /* 0: high threshold 0.2 max |grad| */
    double high_threshold;
    int32_t use_quantiles;      /* 1: thresholds are fractions of max |grad| */
    int32_t mode;               /* lucem_pad_mode (reflect) */
    double cval;
} lucem_canny_settings;
void lucem_canny_settings_default(lucem_canny_settings *s);
/* crates/lucem-ops/src/feature/canny.rs:47-165 canny: 2-D input -> u32 edge
 * map (1 on edges).  The Gaussian blur and the Sobel gradients are fused
 * family launches (the magnitude and the quantised direction in the second
 * one's epilogue); one kernel does the non-maximum suppression and the
 * maximum magnitude; the hysteresis, done by the reference as a host BFS
 * from the strong pixels, is 8-connected component labelling of the pixels
 * at or above the low threshold on the device (union-find), keeping the
 * components that hold a pixel at or above the high threshold: the same
 * edge set.  With both thresholds left to their defaults the call is
 * asynchronous (the thresholds are computed on the device from the maximum);
 * with one or both given it synchronises once to read the maximum, unless
 * both are values (not quantiles). */
lucem_status lucem_canny(lucem_ctx *ctx, const lucem_tensor *in, const lucem_canny_settings *settings,
                         lucem_tensor *out, lucem_workspace *ws, void *stream);

/* crates/lucem-ops/src/transform/pyramid.rs:98-133 Pyramid. */
typedef struct lucem_pyramid_settings {
    double downscale;      /* 2; > 1 */
    double sigma;          /* < 0: the default 2 downscale / 6 */
    int32_t order;         /* 1: bilinear; 0: nearest (orders 2..5, the spline prefilter, are refused) */
    int32_t mode;          /* lucem_pad_mode (reflect) */
    double cval;
} lucem_pyramid_settings;
void lucem_pyramid_settings_default(lucem_pyramid_settings *s);
/* crates/lucem-ops/src/transform/pyramid.rs:135-168 pyramid_reduce: 2-D f32
 * (or u8/u16) input [H, W] -> f32 out [ceil(H / downscale), ceil(W /
 * downscale)]: the Gaussian blur (one fused launch, into the workspace),
 * then the resize's resampling (transform/warp.rs:207-251, orders 0 and 1). */
lucem_status lucem_pyramid_reduce(lucem_ctx *ctx, const lucem_tensor *in, const lucem_pyramid_settings *settings,
                                  lucem_tensor *out, lucem_workspace *ws, void *stream);
/* crates/lucem-ops/src/transform/pyramid.rs:171-208 pyramid_expand: the
 * resampling up to out's shape, then the Gaussian blur.  The reference's
 * default shape is ceil(H * downscale) x ceil(W * downscale). */
lucem_status lucem_pyramid_expand(lucem_ctx *ctx, const lucem_tensor *in, const lucem_pyramid_settings *settings,
                                  lucem_tensor *out, lucem_workspace *ws, void *stream);
/* One band of crates/lucem-ops/src/transform/pyramid.rs:239-266
 * laplacian_pyramid: out = fine - pyramid_expand(coarse, fine's shape). */
lucem_status lucem_laplacian_band(lucem_ctx *ctx, const lucem_tensor *fine, const lucem_tensor *coarse,
                                  const lucem_pyramid_settings *settings, lucem_tensor *out, lucem_workspace *ws,
                                  void *stream);

/* crates/lucem-ops/src/feature/blobs.rs:33-112 BlobDetector. */
typedef struct lucem_blob_settings {
    double min_sigma;        /* 1 */
    double max_sigma;        /* 30 */
    int64_t num_sigma;       /* 10 (LoG, DoH) */
    double sigma_ratio;      /* 1.6 (DoG) */
    double threshold;        /* 0.1, absolute */
    double overlap;          /* 0.5, in [0, 1] */
    int32_t log_scale;       /* 0: linear scale spacing (LoG, DoH) */
    int64_t exclude_border;  /* 1 */
} lucem_blob_settings;
void lucem_blob_settings_default(lucem_blob_settings *s);
/* crates/lucem-ops/src/feature/blobs.rs:16-30 Blob. */
typedef struct lucem_blob {
    int64_t y, x;
    double sigma;
    double response;
} lucem_blob;
/* crates/lucem-ops/src/feature/blobs.rs:204-236 blobs_log, :238-287
 * blobs_dog, :289-345 blobs_doh: 2-D input.  Each scale's response
 * (-sigma^2 LoG, DoG / (ratio - 1), sigma^4 det H) is one fused family
 * launch into a scale stack kept on the device; one kernel marks the
 * 3 x 3 x 3 maxima above the threshold (the reference's tie rule and
 * border); the host sorts them (response descending, then y, x) and drops
 * those overlapping a stronger blob by more than `overlap`.  Writes up to
 * `cap` blobs to `out` and their total number to *n_out (call again with a
 * larger `out` when *n_out > cap).  Synchronises on `stream`. */
lucem_status lucem_blobs_log(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream);
lucem_status lucem_blobs_dog(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream);
lucem_status lucem_blobs_doh(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream);

/* The grid lucem_richardson_lucy uses (host only), before any autotuning of
 * the context: per axis the requested length, or the cheapest m * 2^k
 * (m in {1,3,5,7,9,15,21,25,27}) at least the padding's need, by length
 * times pass cost (the register-resident power-of-two kernels 1, the
 * Stockham kernels 5 for columns and 2.7 for rows). */
lucem_status lucem_rl_grid(const int64_t *dims, const int64_t *kdims, int32_t ndim, int32_t mode,
                           const int64_t *requested, int64_t *grid_out);
/* Smallest 2/3/5/7-smooth length >= n (even when `even`): the shortest
 * length the FFT kernels support (host only). */
int64_t lucem_fft_good_length(int64_t n, int32_t even);

#ifdef __cplusplus
}
#endif
#endif
