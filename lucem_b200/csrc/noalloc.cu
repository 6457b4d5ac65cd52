// noalloc.cu -- lucem_gaussian_blur_noalloc: the N-D separable Gaussian blur
// of lucem_gaussian_blur with no device allocation at all.
//
// Who needs it: callers whose device memory is owned by someone else -- a
// host runtime that hands out every byte from its own pool under a fixed
// budget, or a long-running service that must not grow its footprint or
// synchronise the device with cudaMalloc/cudaFree in the middle of work.
// lucem_gaussian_blur takes its intermediate buffers from a workspace that
// grows with cudaMalloc and caches taps with cudaMalloc; this variant takes
// both from one file-scope device array instead.
//
// The array: g_scratch below, 2 intermediate buffers of kScratchElems floats
// (16 MiB each) plus a taps area, 32 MiB + 64 KiB in all.  Every GPU that
// loads the library holds it until the process exits.  Inputs with more than
// kScratchElems elements are rejected (LUCEM_ERR_TOO_MANY_ELEMENTS); the
// caller still provides the input and output tensors.
//
// Set-up: the first call on a device (with that device current) resolves the
// array's device address with cudaGetSymbolAddress, once per device; that
// first call should come before any stream capture on the device.  The address
// is kept for the life of the process: after a cudaDeviceReset the array is
// reloaded elsewhere and this entry point must not be called again.
//
// Taps reach the array through kernel parameters (put_taps below), so a call
// makes no host-to-device copy.
//
// Sharing: every call uses the same array and it keeps the previous call's
// contents.  Nothing here needs to start at zero (each pass overwrites what
// it reads next), but calls whose work overlaps on the GPU (different
// streams, or different host threads) race on the array: serialise them.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.h"

namespace {

constexpr int64_t kScratchElems = int64_t(4) << 20;  // floats per intermediate buffer
constexpr int64_t kTapsCap = 16384;                   // floats of taps (all passes of one call)

static __device__ __align__(256) float g_scratch[2 * kScratchElems + kTapsCap];

struct DeviceScratch {
    bool ready = false;
    float *base = nullptr;  // device address of g_scratch on that device
};

std::mutex g_mu;
DeviceScratch g_devices[128];

// Device address of g_scratch on the current device (resolved once per device).
lucem_status scratch_base(float **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= 128) return lucem::set_error(LUCEM_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch &d = g_devices[dev];
    if (!d.ready) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString(e));
        }
        d.base = static_cast<float *>(p);
        d.ready = true;
    }
    *out = d.base;
    return LUCEM_OK;
}

// Taps travel to the device inside the parameters of a small kernel, not
// through a host-to-device copy: a launch copies its parameters when it is
// issued (and a captured launch keeps its own copy), so no host buffer has to
// outlive the call and nothing is staged through pageable memory.
constexpr int kTapsPerLaunch = 1000;  // 4,004 bytes of parameters
struct TapsChunk {
    int32_t n;
    float w[kTapsPerLaunch];
};

__global__ void put_taps_kernel(float *__restrict__ dst, const TapsChunk chunk) {
    for (int i = threadIdx.x; i < chunk.n; i += blockDim.x) dst[i] = chunk.w[i];
}

int put_taps(float *dst, const std::vector<float> &w, cudaStream_t s) {
    for (size_t off = 0; off < w.size(); off += kTapsPerLaunch) {
        TapsChunk c;
        c.n = (int32_t)std::min(w.size() - off, (size_t)kTapsPerLaunch);
        std::memcpy(c.w, w.data() + off, (size_t)c.n * sizeof(float));
        put_taps_kernel<<<1, 256, 0, s>>>(dst + off, c);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}

int64_t numel_of(const lucem_tensor *t) {
    int64_t n = 1;
    for (int i = 0; i < t->ndim; ++i) n *= t->dims[i];
    return n;
}

}  // namespace

extern "C" lucem_status lucem_gaussian_blur_noalloc(const lucem_tensor *in, const double *sigmas,
                                                    int32_t n_sigmas, const lucem_gaussian_settings *settings,
                                                    lucem_tensor *out, void *stream) {
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    const lucem_gaussian_settings *s = settings ? settings : &def;
    std::vector<lucem::GaussPass> passes;
    lucem_status st = lucem::gaussian_blur_plan(in, sigmas, n_sigmas, s, out, &passes);
    if (st) return st;
    const int64_t n = numel_of(in);
    if (n == 0) return LUCEM_OK;
    if (n > kScratchElems) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "gaussian_blur_noalloc takes at most %lld elements (its static scratch), got %lld: use "
                 "lucem_gaussian_blur",
                 (long long)kScratchElems, (long long)n);
        return lucem::set_error(LUCEM_ERR_TOO_MANY_ELEMENTS, msg);
    }
    const bool fuse = lucem::gaussian_fuse_last_two(in, passes);
    const size_t n_generic = fuse ? passes.size() - 2 : passes.size();
    int64_t taps_needed = 0;
    for (size_t i = 0; i < n_generic; ++i) taps_needed += 2 * passes[i].radius + 1;
    if (taps_needed > kTapsCap) {
        char msg[256];
        snprintf(msg, sizeof msg, "gaussian_blur_noalloc holds at most %lld taps per call, needs %lld",
                 (long long)kTapsCap, (long long)taps_needed);
        return lucem::set_error(LUCEM_ERR_INVALID_PARAMETER, msg);
    }
    float *base = nullptr;
    if ((st = scratch_base(&base))) return st;
    float *bufs[2] = {base, base + kScratchElems};
    float *taps = base + 2 * kScratchElems;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    float *dst_final = static_cast<float *>(out->data);

    if (passes.empty()) {
        int e = lucem::launch_cast(in->data, in->dtype, (float)s->input_scale, dst_final, n, stream);
        return e ? lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString((cudaError_t)e)) : LUCEM_OK;
    }
    // The reference's pass order (separable::run): generic passes alternate
    // between the two scratch buffers, the last pass writes the output.
    const void *src = in->data;
    int src_dtype = in->dtype;
    float src_scale = (float)s->input_scale;
    int ping = 0;
    int64_t tap_off = 0;
    for (size_t i = 0; i < n_generic; ++i) {
        const lucem::GaussPass &p = passes[i];
        const std::vector<float> w = lucem::gaussian_pass_taps(p);
        if (int e = put_taps(taps + tap_off, w, cs))
            return lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
        const bool last = !fuse && i + 1 == n_generic;
        float *dst = last ? dst_final : bufs[ping];
        int64_t outer = 1, inner = 1;
        for (int d = 0; d < p.axis; ++d) outer *= in->dims[d];
        for (int d = p.axis + 1; d < in->ndim; ++d) inner *= in->dims[d];
        const int size = (int)(2 * p.radius + 1);
        int e = lucem::launch_correlate_1d(src, src_dtype, src_scale, dst, outer, in->dims[p.axis], inner,
                                           taps + tap_off, size, size / 2, s->mode, (float)s->cval, stream);
        if (e) return lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
        tap_off += size;
        src = dst;
        src_dtype = LUCEM_F32;
        src_scale = 1.0f;
        ping ^= 1;
    }
    if (fuse) {
        lucem::FamParams fp;
        lucem_tensor view = *in;
        view.data = const_cast<void *>(src);
        view.dtype = src_dtype;
        lucem::gaussian_fused_params(&fp, &view, s->mode, s->cval, src_scale, passes[passes.size() - 2],
                                     passes[passes.size() - 1], dst_final);
        int e = lucem::launch_family_planes(fp, src_dtype, stream);
        if (e) return lucem::set_error(LUCEM_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    }
    return LUCEM_OK;
}
