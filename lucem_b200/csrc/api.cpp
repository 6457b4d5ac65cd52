// api.cpp -- the C ABI (include/lucem_b200.h): argument checks with the
// reference's error semantics, pass planning, the workspace and constant
// cache, and the host drivers of the filter and Richardson-Lucy kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cfloat>
#include <cstdarg>
#include <cstdio>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "internal.h"

using namespace lucem;

// ---------------------------------------------------------------------------
// Errors: thread-local message + status, as OpsError's Display text
// (crates/lucem-ops/src/error.rs:9-59).

namespace {

thread_local std::string g_last_error;

lucem_status fail(lucem_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

lucem_status ok() {
    return LUCEM_OK;
}

lucem_status cuda_fail(int err, const char *what) {
    return fail(LUCEM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(static_cast<cudaError_t>(err)));
}

#define CUDA_TRY(expr, what)                                                  \
    do {                                                                      \
        int _e = static_cast<int>(expr);                                      \
        if (_e != 0) return cuda_fail(_e, what);                              \
    } while (0)

std::string dims_str(const lucem_tensor *t) {
    std::string s = "[";
    for (int i = 0; i < t->ndim; ++i) {
        if (i) s += ", ";
        s += std::to_string(t->dims[i]);
    }
    return s + "]";
}

int64_t numel(const lucem_tensor *t) {
    int64_t n = 1;
    for (int i = 0; i < t->ndim; ++i) n *= t->dims[i];
    return n;
}

size_t dtype_size(int dt) {
    switch (dt) {
    case LUCEM_U8: return 1;
    case LUCEM_U16: return 2;
    case LUCEM_F32: return 4;
    default: return 0;
    }
}

lucem_status check_tensor_cap(const char *name, const lucem_tensor *t, int skip_leading);

lucem_status check_tensor(const char *name, const lucem_tensor *t) { return check_tensor_cap(name, t, 0); }

// As check_tensor, with the element cap applied to the trailing dims after
// `skip_leading` dims (a stack of planes whose kernels index each plane with
// 64-bit plane offsets).
lucem_status check_tensor_cap(const char *name, const lucem_tensor *t, int skip_leading) {
    if (!t) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `%s`: null tensor", name);
    if (t->ndim < 0 || t->ndim > LUCEM_MAX_DIMS)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "%s expects 0..%d-D array, got %d-D", name,
                    LUCEM_MAX_DIMS, t->ndim);
    if (dtype_size(t->dtype) == 0)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "%s: unsupported element type %d", name, t->dtype);
    // crates/lucem-core/src/compute/limits.rs:16-22 (overflow refused too).
    int64_t n = 1;
    for (int i = 0; i < t->ndim; ++i) {
        if (t->dims[i] < 0)
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `%s`: negative dimension", name);
        if (i < skip_leading) continue;
        if (t->dims[i] != 0 && n > kMaxDeviceElements / t->dims[i])
            return fail(LUCEM_ERR_TOO_MANY_ELEMENTS,
                        "%s %s needs more than %lld elements in one device buffer (kernels use "
                        "32-bit indices): use smaller tiles or batches",
                        name, dims_str(t).c_str(), (long long)kMaxDeviceElements);
        n *= t->dims[i];
    }
    if (n > 0 && !t->data)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `%s`: null data pointer", name);
    return ok();
}

// crates/lucem-ops/src/core/check.rs:10-26.
lucem_status same_shape(const char *a_name, const lucem_tensor *a, const char *b_name,
                        const lucem_tensor *b) {
    bool same = a->ndim == b->ndim;
    for (int i = 0; same && i < a->ndim; ++i) same = a->dims[i] == b->dims[i];
    if (same) return ok();
    return fail(LUCEM_ERR_SHAPE_MISMATCH, "%s shape %s does not match %s shape %s", a_name,
                dims_str(a).c_str(), b_name, dims_str(b).c_str());
}

// crates/lucem-ops/src/core/check.rs:47-57: byte ranges that overlap.
lucem_status not_aliased(const lucem_tensor *a, const lucem_tensor *b) {
    uintptr_t a0 = reinterpret_cast<uintptr_t>(a->data), b0 = reinterpret_cast<uintptr_t>(b->data);
    uintptr_t a1 = a0 + (uintptr_t)(numel(a) * (int64_t)dtype_size(a->dtype));
    uintptr_t b1 = b0 + (uintptr_t)(numel(b) * (int64_t)dtype_size(b->dtype));
    if (numel(a) > 0 && numel(b) > 0 && a0 < b1 && b0 < a1)
        return fail(LUCEM_ERR_ALIASED_BUFFERS,
                    "input and output arrays must not share the same device buffer");
    return ok();
}

lucem_status require_f32_out(const lucem_tensor *out) {
    if (out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "output must be f32, got element type %d", out->dtype);
    return ok();
}

lucem_status check_mode(int32_t mode) {
    if (mode < 0 || mode > 4) return fail(LUCEM_ERR_UNKNOWN_PAD_MODE, "boundary pad mode '%d' is not supported (expected reflect, constant, nearest, mirror, or wrap)", mode);
    return ok();
}

// numpy axis normalisation (crates/lucem-core/src/shape.rs:48-58).
lucem_status norm_axis(int64_t axis, int ndim, int *out) {
    int64_t a = axis < 0 ? axis + ndim : axis;
    if (a < 0 || a >= ndim)
        return fail(LUCEM_ERR_AXIS_OUT_OF_BOUNDS, "axis %lld is out of bounds for array of dimension %d",
                    (long long)axis, ndim);
    *out = (int)a;
    return ok();
}

// crates/lucem-ops/src/core/check.rs:95-109.
template <typename T>
lucem_status broadcast(const char *name, const T *vals, int n_vals, int num_axes, std::vector<T> *out) {
    out->clear();
    if (num_axes == 0) return ok();
    if (n_vals == 1) {
        out->assign(num_axes, vals[0]);
        return ok();
    }
    if (n_vals == num_axes) {
        out->assign(vals, vals + n_vals);
        return ok();
    }
    return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `%s`: expected 1 or %d values, got %d",
                name, num_axes, n_vals);
}

double radius_of(double truncate, double sigma) {
    double r = std::floor(truncate * sigma + 0.5);
    return r > 0.0 ? r : 0.0;
}

// crates/lucem-ops/src/filter/gaussian.rs:22-63.
void gaussian_taps(double sigma, uint32_t order, int64_t radius, double *out) {
    if (radius == 0) {
        out[0] = order == 0 ? 1.0 : 0.0;
        return;
    }
    const double s2 = sigma * sigma;
    const int64_t n = 2 * radius + 1;
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double x = (double)(i - radius);
        out[i] = std::exp(-0.5 * (x * x) / s2);
    }
    for (int64_t i = 0; i < n; ++i) sum += out[i];
    for (int64_t i = 0; i < n; ++i) out[i] /= sum;
    if (order == 0) return;
    for (int64_t i = 0; i < n; ++i) {
        double x = (double)(i - radius), q;
        if (order == 1) q = -x / s2;
        else if (order == 2) q = (x * x - s2) / (s2 * s2);
        else if (order == 3) q = -(x * x * x - 3.0 * x * s2) / (s2 * s2 * s2);
        else {
            double hp = 1.0, hc = -x / s2;
            for (uint32_t k = 1; k < order; ++k) {
                double hn = (-x / s2) * hc - ((double)k / s2) * hp;
                hp = hc;
                hc = hn;
            }
            q = hc;
        }
        out[i] = ((order % 2 == 1) ? -1.0 : 1.0) * q * out[i];
    }
}

}  // namespace

namespace lucem {
const char *pass_name(int kind) {
    static const char *names[kPassCount] = {"rl_row_pass", "rl_col_forward", "rl_col_full", "rl_col_inverse",
                                            "rl_transfer_function", "gaussian_family", "correlate_1d",
                                            "elementwise", "rl_col_y", "rl_col_z", "fft"};
    return kind >= 0 && kind < kPassCount ? names[kind] : "?";
}
}  // namespace lucem

// ---------------------------------------------------------------------------
// Context and workspace.

struct lucem_ctx {
    int device = 0;
    int sms = 148;
    std::mutex mu;
    // Constant cache: key -> device buffer (crates/lucem-core/src/memory/cache.rs:19-44).
    std::map<std::string, void *> cache;
    // Autotuned FFT pass costs: (kind 0 column / 1 row, length) -> ns per element.
    std::map<std::pair<int, int64_t>, double> tune;
    // Autotuned launch settings of the family kernels: key -> FamParams::plan.
    std::map<std::string, int> plans;
    bool tune_on = false;
    void *get_or_upload(const std::string &key, const void *host, size_t bytes, int *err) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
        void *d = nullptr;
        int e = (int)cudaMalloc(&d, bytes > 0 ? bytes : 16);
        if (e) { *err = e; return nullptr; }
        e = (int)cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice);
        if (e) { cudaFree(d); *err = e; return nullptr; }
        cache[key] = d;
        return d;
    }
};

namespace {

// CUDA events around each launch while a workspace's timing is on.
struct EventTimer : PassTimer {
    struct Rec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double total_ms[kPassCount] = {};
    int64_t count[kPassCount] = {};
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int kind, void *stream) override {
        Rec r{kind, take(), nullptr};
        cudaEventRecord(r.a, static_cast<cudaStream_t>(stream));
        recs.push_back(r);
    }
    void end(int kind, void *stream) override {
        if (recs.empty() || recs.back().kind != kind || recs.back().b) return;
        recs.back().b = take();
        cudaEventRecord(recs.back().b, static_cast<cudaStream_t>(stream));
    }
    int collect() {
        int err = 0;
        for (auto &r : recs) {
            if (!r.b) continue;
            int e = (int)cudaEventSynchronize(r.b);
            float ms = 0.f;
            if (!e) e = (int)cudaEventElapsedTime(&ms, r.a, r.b);
            if (e && !err) err = e;
            if (!e) {
                total_ms[r.kind] += ms;
                count[r.kind] += 1;
            }
        }
        for (auto &r : recs) {
            pool.push_back(r.a);
            if (r.b) pool.push_back(r.b);
        }
        recs.clear();
        return err;
    }
    void reset() {
        collect();
        for (int k = 0; k < kPassCount; ++k) {
            total_ms[k] = 0.0;
            count[k] = 0;
        }
    }
    ~EventTimer() override {
        for (auto &r : recs) {
            pool.push_back(r.a);
            if (r.b) pool.push_back(r.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct Slot {
    void *ptr = nullptr;
    size_t cap = 0;
    std::string key;  // what the slot's content was computed from (for caches)
};
}  // namespace

namespace {
// The timer of the workspace the current entry point runs with (if timing).
thread_local PassTimer *g_timer = nullptr;
template <typename F>
int timed(int kind, void *stream, F &&f) {
    if (g_timer) g_timer->begin(kind, stream);
    int e = f();
    if (g_timer) g_timer->end(kind, stream);
    return e;
}
}  // namespace

struct lucem_workspace {
    lucem_ctx *ctx = nullptr;
    std::map<std::string, Slot> slots;
    std::unique_ptr<EventTimer> timer;  // set while timing is enabled
    PassTimer *t() { return timer.get(); }
    int64_t wait_limit_ns = -1;         // bounded device waits: -1 the default (one second)
    // crates/lucem-core/src/memory/workspace.rs:28-37: grow-only, budget checked.
    lucem_status get(const char *name, size_t bytes, void **out, Slot **slot_out = nullptr) {
        Slot &s = slots[name];
        if (s.cap < bytes) {
            if (s.ptr) {
                cudaFree(s.ptr);
                s.ptr = nullptr;
                s.cap = 0;
                s.key.clear();
            }
            size_t free_b = 0, total_b = 0;
            cudaMemGetInfo(&free_b, &total_b);
            void *p = nullptr;
            cudaError_t e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(LUCEM_ERR_OUT_OF_DEVICE_MEMORY,
                            "%s needs %zu bytes of device memory; the budget leaves %zu (limit %zu)",
                            name, bytes, free_b, total_b);
            }
            s.ptr = p;
            s.cap = bytes;
        }
        *out = s.ptr;
        if (slot_out) *slot_out = &s;
        return ok();
    }
    ~lucem_workspace() {
        for (auto &kv : slots)
            if (kv.second.ptr) cudaFree(kv.second.ptr);
    }
};

namespace {
struct TimerScope {
    PassTimer *prev;
    explicit TimerScope(lucem_workspace *ws) : prev(g_timer) { g_timer = ws ? ws->t() : nullptr; }
    ~TimerScope() { g_timer = prev; }
};
}  // namespace

extern "C" {

int32_t lucem_abi_version(void) { return LUCEM_B200_ABI_VERSION; }

const char *lucem_last_error_message(void) { return g_last_error.c_str(); }

lucem_status lucem_ctx_create(int32_t device, lucem_ctx **out) {
    if (!out) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `out`: null");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(LUCEM_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= count)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `device`: %d of %d", device, count);
    CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    auto *c = new lucem_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return ok();
}

void lucem_ctx_destroy(lucem_ctx *ctx) {
    if (!ctx) return;
    for (auto &kv : ctx->cache) cudaFree(kv.second);
    delete ctx;
}

lucem_status lucem_workspace_create(lucem_ctx *ctx, lucem_workspace **out) {
    if (!ctx || !out) return fail(LUCEM_ERR_INVALID_HANDLE, "null context or output pointer");
    auto *w = new lucem_workspace();
    w->ctx = ctx;
    *out = w;
    return ok();
}

void lucem_workspace_destroy(lucem_workspace *ws) { delete ws; }

lucem_status lucem_workspace_set_timing(lucem_workspace *ws, int32_t enable) {
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "null workspace");
    if (enable) {
        if (!ws->timer) ws->timer.reset(new EventTimer());
        ws->timer->reset();
    } else {
        ws->timer.reset();
    }
    return ok();
}

lucem_status lucem_workspace_set_wait_limit(lucem_workspace *ws, int64_t ns) {
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "null workspace");
    if (ns < 0) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `ns`: a wait limit cannot be negative");
    ws->wait_limit_ns = ns;
    return ok();
}

lucem_status lucem_workspace_wait_status(lucem_workspace *ws, void *stream, int64_t *gave_up) {
    if (!ws || !gave_up) return fail(LUCEM_ERR_INVALID_HANDLE, "null workspace or output");
    *gave_up = 0;
    auto it = ws->slots.find("device_status");
    if (it == ws->slots.end() || !it->second.ptr) return ok();
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    int32_t n = 0;
    CUDA_TRY(cudaMemcpyAsync(&n, it->second.ptr, sizeof n, cudaMemcpyDeviceToHost, cs), "status read");
    CUDA_TRY(cudaStreamSynchronize(cs), "status read");
    if (n == 0) return ok();
    CUDA_TRY(cudaMemsetAsync(it->second.ptr, 0, sizeof n, cs), "status reset");
    CUDA_TRY(cudaStreamSynchronize(cs), "status reset");
    *gave_up = n;
    return fail(LUCEM_ERR_DEVICE_TIMEOUT,
                "%d bounded device wait(s) gave up (tensor copies of the staged blur; those tiles were loaded "
                "directly, results are unaffected)", (int)n);
}

lucem_status lucem_workspace_timings(lucem_workspace *ws, char *names, double *ms, int64_t *launches,
                                     int32_t cap, int32_t *n_out) {
    if (!ws || !n_out) return fail(LUCEM_ERR_INVALID_HANDLE, "null workspace or output");
    *n_out = 0;
    if (!ws->timer) return ok();
    int e = ws->timer->collect();
    if (e) return cuda_fail(e, "timing events");
    int n = 0;
    for (int k = 0; k < kPassCount; ++k) {
        if (ws->timer->count[k] == 0) continue;
        if (n < cap) {
            if (names) {
                std::strncpy(names + 32 * n, pass_name(k), 31);
                names[32 * n + 31] = 0;
            }
            if (ms) ms[n] = ws->timer->total_ms[k];
            if (launches) launches[n] = ws->timer->count[k];
        }
        ++n;
    }
    *n_out = n;
    return ok();
}

size_t lucem_workspace_capacity_bytes(const lucem_workspace *ws) {
    if (!ws) return 0;
    size_t n = 0;
    for (auto &kv : ws->slots) n += kv.second.cap;
    return n;
}

lucem_status lucem_pad_mode_parse(const char *name, int32_t *mode_out) {
    if (!name || !mode_out) return fail(LUCEM_ERR_INVALID_PARAMETER, "null argument");
    std::string s(name);
    size_t b = s.find_first_not_of(" \t\n\r"), e = s.find_last_not_of(" \t\n\r");
    s = b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
    for (auto &ch : s) ch = (char)std::tolower((unsigned char)ch);
    if (s == "reflect" || s == "symmetric" || s == "grid-mirror") *mode_out = LUCEM_PAD_REFLECT;
    else if (s == "constant" || s == "grid-constant" || s == "zeros") *mode_out = LUCEM_PAD_CONSTANT;
    else if (s == "nearest" || s == "edge" || s == "replicate") *mode_out = LUCEM_PAD_NEAREST;
    else if (s == "mirror") *mode_out = LUCEM_PAD_MIRROR;
    else if (s == "wrap" || s == "grid-wrap" || s == "periodic") *mode_out = LUCEM_PAD_WRAP;
    else
        return fail(LUCEM_ERR_UNKNOWN_PAD_MODE,
                    "boundary pad mode '%s' is not supported (expected reflect, constant, nearest, "
                    "mirror, or wrap)", s.c_str());
    return ok();
}

lucem_status lucem_gaussian_kernel_1d(double sigma, uint32_t order, int64_t radius, double *out) {
    if (!out || radius < 0) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `radius`");
    gaussian_taps(sigma, order, radius, out);
    return ok();
}

int64_t lucem_gaussian_radius(double truncate, double sigma) {
    return (int64_t)radius_of(truncate, sigma);
}

int64_t lucem_pad_index(int64_t p, int64_t len, int32_t mode) {
    if (p >= 0 && p < len) return p;
    switch (mode) {
    case LUCEM_PAD_CONSTANT: return -1;
    case LUCEM_PAD_NEAREST: return p < 0 ? 0 : len - 1;
    case LUCEM_PAD_WRAP: return ((p % len) + len) % len;
    case LUCEM_PAD_REFLECT: {
        int64_t period = 2 * len, r = ((p % period) + period) % period;
        return r < len ? r : period - 1 - r;
    }
    default: {
        int64_t period = std::max<int64_t>(2 * len - 2, 1), r = ((p % period) + period) % period;
        return r < len ? r : period - r;
    }
    }
}

void lucem_gaussian_settings_default(lucem_gaussian_settings *s) {
    std::memset(s, 0, sizeof *s);
    s->mode = LUCEM_PAD_REFLECT;
    s->cval = 0.0;
    s->truncate = 4.0;
    s->input_scale = 1.0;
}

void lucem_gaussian_1d_settings_default(lucem_gaussian_1d_settings *s) {
    std::memset(s, 0, sizeof *s);
    s->axis = -1;
    s->order = 0;
    s->mode = LUCEM_PAD_REFLECT;
    s->cval = 0.0;
    s->truncate = 4.0;
    s->radius = -1;
}

void lucem_rl_settings_default(lucem_rl_settings *s) {
    std::memset(s, 0, sizeof *s);
    s->num_iter = 30;
    s->clip = 1;
    s->has_filter_epsilon = 0;
    s->filter_epsilon = 0.0;
    s->mode = LUCEM_PAD_REFLECT;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Separable passes.

namespace {

using Pass = lucem::GaussPass;

// crates/lucem-ops/src/filter/gaussian.rs:184-219.
lucem_status plan_passes(int ndim, const double *sigmas, int n_sigmas, const lucem_gaussian_settings *s,
                         std::vector<Pass> *passes) {
    std::vector<int> axes;
    if (s->axes == nullptr) {
        for (int d = 0; d < ndim; ++d) axes.push_back(d);
    } else {
        for (int i = 0; i < s->n_axes; ++i) {
            int a;
            lucem_status st = norm_axis(s->axes[i], ndim, &a);
            if (st) return st;
            if (std::find(axes.begin(), axes.end(), a) != axes.end())
                return fail(LUCEM_ERR_REPEATED_AXIS, "repeated axis %lld", (long long)s->axes[i]);
            axes.push_back(a);
        }
    }
    if (s->has_channel_axis) {
        int ch;
        lucem_status st = norm_axis(s->channel_axis, ndim, &ch);
        if (st) return st;
        axes.erase(std::remove(axes.begin(), axes.end(), ch), axes.end());
    }
    const int na = (int)axes.size();
    std::vector<double> sig;
    lucem_status st = broadcast("sigmas", sigmas, n_sigmas, na, &sig);
    if (st) return st;
    for (double v : sig)
        if (!std::isfinite(v) || v < 0.0)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "invalid parameter `sigmas`: sigma must be non-negative and finite, got %g", v);
    static const uint32_t zero_order = 0;
    std::vector<uint32_t> ords;
    st = s->n_orders > 0 ? broadcast("orders", s->orders, s->n_orders, na, &ords)
                         : broadcast("orders", &zero_order, 1, na, &ords);
    if (st) return st;
    std::vector<int64_t> rad;
    bool has_r = s->n_radii > 0 && s->radii;
    if (has_r) {
        st = broadcast("radii", s->radii, s->n_radii, na, &rad);
        if (st) return st;
    }
    passes->clear();
    for (int i = 0; i < na; ++i) {
        if (!(sig[i] > 0.0)) continue;
        int64_t r = has_r ? rad[i] : (int64_t)radius_of(s->truncate, sig[i]);
        if (r < 0) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `radii`: negative radius");
        passes->push_back(Pass{axes[i], sig[i], ords[i], r});
    }
    return ok();
}

// Device copy of f32 weights, cached per context under `key`.
lucem_status cached_weights(lucem_ctx *ctx, const std::string &key, const std::vector<float> &w,
                            const float **out) {
    int err = 0;
    void *d = ctx->get_or_upload(key, w.data(), w.size() * sizeof(float), &err);
    if (!d) return cuda_fail(err, "uploading filter taps");
    *out = static_cast<const float *>(d);
    return ok();
}

std::string tap_key(double sigma, uint32_t order, int64_t radius) {
    char buf[128];
    // Same identity as GAUSSIAN_TAPS' key (crates/lucem-ops/src/filter/gaussian.rs:107).
    snprintf(buf, sizeof buf, "f32-gauss1d-%.12f-o%u-r%lld", sigma, order, (long long)radius);
    return buf;
}

std::vector<float> taps_f32(double sigma, uint32_t order, int64_t radius) {
    std::vector<double> d((size_t)(2 * radius + 1));
    gaussian_taps(sigma, order, radius, d.data());
    return std::vector<float>(d.begin(), d.end());
}

void split_axis(const lucem_tensor *t, int axis, int64_t *outer, int64_t *len, int64_t *inner) {
    *outer = 1;
    *inner = 1;
    for (int d = 0; d < axis; ++d) *outer *= t->dims[d];
    for (int d = axis + 1; d < t->ndim; ++d) *inner *= t->dims[d];
    *len = t->dims[axis];
}

// One generic pass: src (dtype, scale) -> dst f32 along `axis`.
lucem_status generic_pass(lucem_ctx *ctx, const lucem_tensor *shape, const void *src, int src_dtype,
                          float scale, float *dst, const Pass &p, int mode, double cval, void *stream) {
    const float *w = nullptr;
    lucem_status st = cached_weights(ctx, tap_key(p.sigma, p.order, p.radius),
                                     taps_f32(p.sigma, p.order, p.radius), &w);
    if (st) return st;
    int64_t outer, len, inner;
    split_axis(shape, p.axis, &outer, &len, &inner);
    int size = (int)(2 * p.radius + 1);
    int e = timed(kPassCorrelate, stream, [&] { return launch_correlate_1d(src, src_dtype, scale, dst, outer, len, inner, w, size, size / 2,
                                mode, (float)cval, stream); });
    if (e) return cuda_fail(e, "correlate_1d launch");
    return ok();
}

void fill_filter_taps(FamParams *fp, int f, const Pass *p0, const Pass *p1) {
    // p0: axis 0 (rows) pass or null (identity), p1: axis 1 (columns).  Taps
    // are stored as (w, w) pairs at the kernel radius, centred.
    std::memset(fp->taps0[f], 0, sizeof fp->taps0[f]);
    std::memset(fp->taps1[f], 0, sizeof fp->taps1[f]);
    auto put = [](float2_ *dst, const Pass *p) -> int {
        if (!p) {
            dst[0] = float2_{1.0f, 1.0f};
            return 0;
        }
        std::vector<float> t = taps_f32(p->sigma, p->order, p->radius);
        const int r = (int)p->radius, rk = fam_kernel_radius(r);
        for (size_t i = 0; i < t.size(); ++i) dst[i + (rk - r)] = float2_{t[i], t[i]};
        return rk;
    };
    fp->r0[f] = put(fp->taps0[f], p0);
    fp->r1[f] = put(fp->taps1[f], p1);
}

void init_fam(FamParams *fp, const lucem_tensor *in, int mode, double cval, double scale) {
    std::memset(fp, 0, sizeof *fp);
    fp->in = in->data;
    const int nd = in->ndim;
    fp->H = (int32_t)in->dims[nd - 2];
    fp->W = (int32_t)in->dims[nd - 1];
    int64_t B = 1;
    for (int d = 0; d < nd - 2; ++d) B *= in->dims[d];
    fp->B = (int32_t)B;
    fp->in_plane_stride = (int64_t)fp->H * fp->W;
    fp->in_row_pitch = fp->W;
    fp->mode = mode;
    fp->cval = (float)cval;
    fp->in_scale = (float)scale;
}

// The workspace's bounded-wait settings and give-up counter for a family
// launch (a 64-byte "device_status" slot, zeroed when first allocated).
lucem_status fam_waits(lucem_workspace *ws, FamParams *fp, void *stream) {
    if (!ws) return ok();
    void *p = nullptr;
    Slot *sl = nullptr;
    lucem_status st = ws->get("device_status", 64, &p, &sl);
    if (st) return st;
    if (sl->key.empty()) {
        CUDA_TRY(cudaMemsetAsync(p, 0, 64, static_cast<cudaStream_t>(stream)), "status reset");
        sl->key = "zeroed";
    }
    fp->wait_status = static_cast<int32_t *>(p);
    fp->wait_ns = ws->wait_limit_ns < 0 ? 0 : (ws->wait_limit_ns == 0 ? -1 : ws->wait_limit_ns);
    return ok();
}

// Launch-settings key of a family launch: kernel kind, SM count, element
// type, filter count, largest radius and the power-of-two class of its tile
// count (the reference keys CubeCL's tuning by device id and size class,
// crates/lucem-core/src/compute/tune.rs:12-27).
std::string plan_key(const lucem_ctx *ctx, const char *kind, int dtype, const FamParams &fp, int64_t tiles) {
    int64_t cls = 1;
    while (cls < tiles) cls <<= 1;
    char b[96];
    snprintf(b, sizeof b, "%s-sm%d-t%d-f%d-r%d-n%lld", kind, ctx->sms, dtype, fp.n_filters,
             std::max(fp.rmax0, fp.rmax1), (long long)cls);
    return b;
}

int64_t plane_tiles(const FamParams &fp) {
    return (int64_t)((fp.H + kFamTile - 1) / kFamTile) * ((fp.W + kFamTile - 1) / kFamTile) * fp.B;
}

// Runs launch() with the key's cached plan; while tuning is on and the key
// is new (and the stream is not being captured), first times every
// candidate plan on this call's data (one warm-up and two timed runs each;
// every candidate computes the same result), caches the fastest and runs it
// last.
template <class F>
int tuned_launch(lucem_ctx *ctx, const std::string &key, const std::vector<int> &cands, FamParams *fp,
                 void *stream, F &&launch) {
    bool tune = false;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->plans.find(key);
        if (it != ctx->plans.end()) fp->plan = it->second;
        else tune = ctx->tune_on && cands.size() > 1;
    }
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (tune && cudaStreamIsCapturing(cs, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone) {
        cudaEvent_t a = nullptr, b = nullptr;
        int e = (int)cudaEventCreate(&a);
        if (!e) e = (int)cudaEventCreate(&b);
        int best_plan = 0;
        float best = 0.f;
        for (size_t i = 0; i < cands.size() && !e; ++i) {
            fp->plan = cands[i];
            float tmin = -1.f;
            for (int rep = 0; rep < 3 && !e; ++rep) {
                e = (int)cudaEventRecord(a, cs);
                if (!e) e = launch();
                if (!e) e = (int)cudaEventRecord(b, cs);
                if (!e) e = (int)cudaEventSynchronize(b);
                float ms = 0.f;
                if (!e) e = (int)cudaEventElapsedTime(&ms, a, b);
                if (!e && rep > 0 && (tmin < 0.f || ms < tmin)) tmin = ms;
            }
            if (!e && (best_plan == 0 || tmin < best)) {
                best = tmin;
                best_plan = cands[i];
            }
        }
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        if (e) return e;
        fp->plan = best_plan;
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->plans[key] = best_plan;
    }
    return launch();
}

// Candidate plans: the plain 2-D blur (loads or tensor copies ahead), the
// persistent walk (copies ahead or not, one or as many CTAs per SM as fit).
std::vector<int> blur_candidates(const FamParams &fp) {
    const int r = fp.r0[0];
    const bool rf = fp.n_filters == 1 && fp.r1[0] == r && fp.rmax0 == r && fp.rmax1 == r && r >= 2 && r <= 16 &&
                    (r <= 12 || r == 16);
    if (!rf) return {};
    return {1, 1 + kPlanAhead};
}
std::vector<int> walk_candidates() {
    return {1, 1 + kPlanAhead, 1 + kPlanOneCta, 1 + kPlanAhead + kPlanOneCta};
}

// Executes a pass list from `in` into `out` (f32): the reference's
// separable::run (crates/lucem-ops/src/core/separable.rs:20-61), with the
// last two passes fused into one launch when they are the two innermost axes
// in ascending order.
lucem_status run_passes(lucem_ctx *ctx, const lucem_tensor *in, const std::vector<Pass> &passes,
                        int mode, double cval, double scale, float *out, lucem_workspace *ws,
                        void *stream) {
    const int64_t n = numel(in);
    if (n == 0) return ok();
    if (passes.empty()) {
        int e = timed(kPassElementwise, stream, [&] { return launch_cast(in->data, in->dtype, (float)scale, out, n, stream); });
        return e ? cuda_fail(e, "copy launch") : ok();
    }
    const int nd = in->ndim;
    size_t np = passes.size();
    bool fuse = np >= 2 && passes[np - 2].axis == nd - 2 && passes[np - 1].axis == nd - 1 &&
                passes[np - 2].radius <= kFamMaxRadius && passes[np - 1].radius <= kFamMaxRadius &&
                in->dims[nd - 2] < (1 << 30) && in->dims[nd - 1] < (1 << 30);
    size_t n_generic = fuse ? np - 2 : np;
    // Ping/pong slots as the reference's "sep_ping"/"sep_pong".
    float *bufs[2] = {nullptr, nullptr};
    size_t needed = n_generic + (fuse ? 1 : 0) > 1 ? std::min<size_t>(2, n_generic) : 0;
    if (n_generic >= 1 && (fuse || n_generic >= 2)) needed = n_generic >= 2 ? 2 : 1;
    for (size_t i = 0; i < needed; ++i) {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required for multi-pass filters");
        void *p = nullptr;
        lucem_status st = ws->get(i == 0 ? "sep_ping" : "sep_pong", (size_t)n * sizeof(float), &p);
        if (st) return st;
        bufs[i] = static_cast<float *>(p);
    }
    const void *src = in->data;
    int src_dtype = in->dtype;
    float src_scale = (float)scale;
    int ping = 0;
    for (size_t i = 0; i < n_generic; ++i) {
        bool last = !fuse && i + 1 == n_generic;
        float *dst = last ? out : bufs[ping];
        lucem_status st = generic_pass(ctx, in, src, src_dtype, src_scale, dst, passes[i], mode, cval, stream);
        if (st) return st;
        src = dst;
        src_dtype = LUCEM_F32;
        src_scale = 1.0f;
        ping ^= 1;
    }
    if (fuse) {
        FamParams fp;
        lucem_tensor view = *in;
        view.data = const_cast<void *>(src);
        view.dtype = src_dtype;
        init_fam(&fp, &view, mode, cval, src_scale);
        fp.n_filters = 1;
        fill_filter_taps(&fp, 0, &passes[np - 2], &passes[np - 1]);
        fp.rmax0 = fp.r0[0];
        fp.rmax1 = fp.r1[0];
        fp.n_outputs = 1;
        FamOutput &o = fp.outs[0];
        o.out = out;
        o.plane_stride = (int64_t)fp.H * fp.W;
        o.row_pitch = fp.W;
        o.combine = (int)Combine::kLinear;
        o.fa = 0;
        o.fb = -1;
        o.alpha = 1.0f;
        o.beta = 0.0f;
        o.bias = 0.0f;
        if (lucem_status ws_st = fam_waits(ws, &fp, stream)) return ws_st;
        int e = tuned_launch(ctx, plan_key(ctx, "blur", src_dtype, fp, plane_tiles(fp)), blur_candidates(fp), &fp,
                             stream, [&] {
                                 return timed(kPassFamily, stream,
                                              [&] { return launch_family_planes(fp, src_dtype, stream); });
                             });
        if (e) return cuda_fail(e, "gaussian family launch");
    }
    return ok();
}

// The adjoint of run_passes' linear map x -> out (f32 in and out): the
// adjoint of each pass in reverse order.  One pass's adjoint is the
// zero-padded correlation with the reversed taps plus the fold of the halo
// reads back onto the positions the pad mode mapped them to
// (launch_adjoint_fold).  `scale` is the forward's input_scale; cval does not
// enter (it belongs to the map's constant term).
lucem_status adjoint_passes(lucem_ctx *ctx, const lucem_tensor *shape, const float *g,
                            const std::vector<Pass> &passes, int mode, double scale, float *out,
                            lucem_workspace *ws, void *stream) {
    const int64_t n = numel(shape);
    if (n == 0) return ok();
    const size_t np = passes.size();
    if (np == 0) {
        int e = timed(kPassElementwise, stream, [&] { return launch_cast(g, LUCEM_F32, (float)scale, out, n, stream); });
        return e ? cuda_fail(e, "copy launch") : ok();
    }
    float *bufs[2] = {nullptr, nullptr};
    const size_t needed = np >= 3 ? 2 : np - 1;
    for (size_t i = 0; i < needed; ++i) {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required for multi-pass filters");
        void *p = nullptr;
        lucem_status st = ws->get(i == 0 ? "sep_ping" : "sep_pong", (size_t)n * sizeof(float), &p);
        if (st) return st;
        bufs[i] = static_cast<float *>(p);
    }
    const float *src = g;
    float src_scale = (float)scale;
    int ping = 0;
    for (size_t k = 0; k < np; ++k) {
        const Pass &p = passes[np - 1 - k];
        float *dst = k + 1 == np ? out : bufs[ping];
        const std::vector<float> w = taps_f32(p.sigma, p.order, p.radius);
        const std::vector<float> wr(w.rbegin(), w.rend());
        const float *w_dev = nullptr, *wr_dev = nullptr;
        lucem_status st;
        const std::string key = tap_key(p.sigma, p.order, p.radius);
        if ((st = cached_weights(ctx, key, w, &w_dev)) || (st = cached_weights(ctx, "rev-" + key, wr, &wr_dev)))
            return st;
        int64_t outer, len, inner;
        split_axis(shape, p.axis, &outer, &len, &inner);
        const int size = (int)(2 * p.radius + 1), left = size / 2;
        int e = timed(kPassCorrelate, stream, [&] {
            return launch_correlate_1d(src, LUCEM_F32, src_scale, dst, outer, len, inner, wr_dev, size,
                                       size - 1 - left, LUCEM_PAD_CONSTANT, 0.0f, stream);
        });
        if (!e)
            e = timed(kPassCorrelate, stream, [&] {
                return launch_adjoint_fold(src, src_scale, dst, outer, len, inner, w_dev, size, left, mode, stream);
            });
        if (e) return cuda_fail(e, "adjoint pass launch");
        src = dst;
        src_scale = 1.0f;
        ping ^= 1;
    }
    return ok();
}

lucem_status check_in_out(const lucem_tensor *in, const lucem_tensor *out) {
    lucem_status st;
    if ((st = check_tensor("input", in))) return st;
    if ((st = check_tensor("output", out))) return st;
    if ((st = same_shape("input", in, "output", out))) return st;
    if ((st = not_aliased(in, out))) return st;
    return require_f32_out(out);
}

}  // namespace

// ---------------------------------------------------------------------------
// Gaussian family entry points.

extern "C" {

lucem_status lucem_gaussian_blur(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                 int32_t n_sigmas, const lucem_gaussian_settings *settings,
                                 lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    const lucem_gaussian_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_in_out(in, out))) return st;
    if ((st = check_mode(s->mode))) return st;
    std::vector<Pass> passes;
    if ((st = plan_passes(in->ndim, sigmas, n_sigmas, s, &passes))) return st;
    return run_passes(ctx, in, passes, s->mode, s->cval, s->input_scale, static_cast<float *>(out->data),
                      ws, stream);
}

lucem_status lucem_gaussian_blur_adjoint(lucem_ctx *ctx, const lucem_tensor *grad_out, const double *sigmas,
                                         int32_t n_sigmas, const lucem_gaussian_settings *settings,
                                         lucem_tensor *grad_in, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    const lucem_gaussian_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_in_out(grad_out, grad_in))) return st;
    if (grad_out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "gaussian_blur_adjoint takes an f32 gradient");
    if ((st = check_mode(s->mode))) return st;
    std::vector<Pass> passes;
    if ((st = plan_passes(grad_out->ndim, sigmas, n_sigmas, s, &passes))) return st;
    return adjoint_passes(ctx, grad_out, static_cast<const float *>(grad_out->data), passes, s->mode,
                          s->input_scale, static_cast<float *>(grad_in->data), ws, stream);
}

lucem_status lucem_gaussian_1d(lucem_ctx *ctx, const lucem_tensor *in, double sigma,
                               const lucem_gaussian_1d_settings *settings, lucem_tensor *out,
                               void *stream) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_gaussian_1d_settings def;
    lucem_gaussian_1d_settings_default(&def);
    const lucem_gaussian_1d_settings *s = settings ? settings : &def;
    lucem_status st;
    // crates/lucem-ops/src/filter/gaussian.rs:96-104 (sigma checked first).
    if (!std::isfinite(sigma) || sigma < 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `sigma`: sigma must be non-negative and finite, got %g", sigma);
    if ((st = check_in_out(in, out))) return st;
    if ((st = check_mode(s->mode))) return st;
    int axis;
    if ((st = norm_axis(s->axis, in->ndim, &axis))) return st;
    std::vector<Pass> passes;
    if (sigma > 0.0) {
        int64_t r = s->radius >= 0 ? s->radius : (int64_t)radius_of(s->truncate, sigma);
        passes.push_back(Pass{axis, sigma, s->order, r});
    }
    return run_passes(ctx, in, passes, s->mode, s->cval, 1.0, static_cast<float *>(out->data), nullptr,
                      stream);
}

lucem_status lucem_correlate_1d(lucem_ctx *ctx, const lucem_tensor *in, const double *weights,
                                int64_t n_weights, const lucem_correlate_1d_settings *settings,
                                lucem_tensor *out, void *stream) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!settings) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `settings`: null");
    lucem_status st;
    // crates/lucem-ops/src/core/check.rs:74-82.
    if (!weights || n_weights <= 0)
        return fail(LUCEM_ERR_INVALID_WEIGHTS, "weights: filter weights cannot be empty");
    for (int64_t i = 0; i < n_weights; ++i)
        if (!std::isfinite(weights[i]))
            return fail(LUCEM_ERR_INVALID_WEIGHTS, "weights: filter weights must be finite");
    if ((st = check_in_out(in, out))) return st;
    if ((st = check_mode(settings->mode))) return st;
    // crates/lucem-ops/src/core/check.rs:60-71.
    int32_t mn = -(int32_t)(n_weights / 2), mx = (int32_t)((n_weights - 1) / 2);
    if (settings->origin < mn || settings->origin > mx)
        return fail(LUCEM_ERR_INVALID_ORIGIN,
                    "origin %d is out of bounds for window of size %lld (must be in %d..=%d)",
                    settings->origin, (long long)n_weights, mn, mx);
    int axis;
    if ((st = norm_axis(settings->axis, in->ndim, &axis))) return st;
    if (numel(in) == 0) return ok();
    std::vector<float> w(weights, weights + n_weights);
    std::string key = "f32-corr1d-";
    key.append(reinterpret_cast<const char *>(weights), (size_t)n_weights * sizeof(double));
    const float *wd = nullptr;
    if ((st = cached_weights(ctx, key, w, &wd))) return st;
    int64_t outer, len, inner;
    split_axis(in, axis, &outer, &len, &inner);
    int left = (int)(n_weights / 2) + settings->origin;
    int e = timed(kPassCorrelate, stream, [&] { return launch_correlate_1d(in->data, in->dtype, 1.0f, static_cast<float *>(out->data), outer, len,
                                inner, wd, (int)n_weights, left, settings->mode,
                                (float)settings->cval, stream); });
    return e ? cuda_fail(e, "correlate_1d launch") : ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Multi-response family (fused) and the composite ops.

namespace {

struct FilterKey {
    double s0, s1;
    uint32_t o0, o1;
    bool operator==(const FilterKey &o) const { return s0 == o.s0 && s1 == o.s1 && o0 == o.o0 && o1 == o.o1; }
};

struct FamilyPlan {
    std::vector<FilterKey> filters;
    struct Out { int kind; int fa, fb; float alpha, beta, bias; };
    std::vector<Out> outs;
};

int add_filter(FamilyPlan *pl, FilterKey k) {
    for (size_t i = 0; i < pl->filters.size(); ++i)
        if (pl->filters[i] == k) return (int)i;
    pl->filters.push_back(k);
    return (int)pl->filters.size() - 1;
}

lucem_status check_sigma(double s, const char *name) {
    if (!std::isfinite(s) || s < 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `%s`: sigma must be non-negative and finite, got %g", name, s);
    return ok();
}

lucem_status plan_family(const lucem_response *r, int n, FamilyPlan *pl) {
    lucem_status st;
    for (int i = 0; i < n; ++i) {
        const lucem_response &x = r[i];
        if ((st = check_sigma(x.sigma, "sigma"))) return st;
        FamilyPlan::Out o{};
        o.kind = x.kind;
        o.alpha = 1.0f;
        o.beta = 0.0f;
        o.bias = 0.0f;
        o.fb = -1;
        switch (x.kind) {
        case LUCEM_RESP_GAUSSIAN:
            o.fa = add_filter(pl, {x.sigma, x.sigma, 0, 0});
            break;
        case LUCEM_RESP_DOG:
            if ((st = check_sigma(x.sigma2, "sigma2"))) return st;
            o.fa = add_filter(pl, {x.sigma, x.sigma, 0, 0});
            o.fb = add_filter(pl, {x.sigma2, x.sigma2, 0, 0});
            o.beta = -1.0f;
            break;
        case LUCEM_RESP_LAPLACE:
            o.fa = add_filter(pl, {x.sigma, x.sigma, 2, 0});
            o.fb = add_filter(pl, {x.sigma, x.sigma, 0, 2});
            o.beta = 1.0f;
            break;
        case LUCEM_RESP_GRAD_MAG:
            o.fa = add_filter(pl, {x.sigma, x.sigma, 1, 0});
            o.fb = add_filter(pl, {x.sigma, x.sigma, 0, 1});
            break;
        case LUCEM_RESP_UNSHARP:
            o.fa = -2;
            o.fb = add_filter(pl, {x.sigma, x.sigma, 0, 0});
            o.alpha = (float)(1.0 + x.amount);
            o.beta = (float)(-x.amount);
            break;
        default:
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `kind`: %d", x.kind);
        }
        pl->outs.push_back(o);
    }
    return ok();
}

bool family_fusable(const FamilyPlan &pl, double truncate) {
    if ((int)pl.filters.size() > kFamMaxFilters || (int)pl.outs.size() > kFamMaxOutputs) return false;
    for (auto &f : pl.filters)
        if (radius_of(truncate, f.s0) > kFamMaxRadius || radius_of(truncate, f.s1) > kFamMaxRadius)
            return false;
    return true;
}

void build_fam(FamParams *fp, const FamilyPlan &pl, double truncate) {
    fp->n_filters = (int)pl.filters.size();
    fp->rmax0 = fp->rmax1 = 0;
    for (int f = 0; f < fp->n_filters; ++f) {
        const FilterKey &k = pl.filters[f];
        Pass p0{0, k.s0, k.o0, (int64_t)radius_of(truncate, k.s0)};
        Pass p1{1, k.s1, k.o1, (int64_t)radius_of(truncate, k.s1)};
        // sigma == 0 skips the axis (gaussian.rs:217): identity taps.
        fill_filter_taps(fp, f, k.s0 > 0.0 ? &p0 : nullptr, k.s1 > 0.0 ? &p1 : nullptr);
        fp->rmax0 = std::max(fp->rmax0, fp->r0[f]);
        fp->rmax1 = std::max(fp->rmax1, fp->r1[f]);
    }
    fp->n_outputs = (int)pl.outs.size();
    for (int k = 0; k < fp->n_outputs; ++k) {
        const auto &o = pl.outs[k];
        FamOutput &fo = fp->outs[k];
        fo.combine = o.kind == LUCEM_RESP_GRAD_MAG ? (int)Combine::kHypot : (int)Combine::kLinear;
        fo.fa = o.fa;
        fo.fb = o.fb;
        fo.alpha = o.alpha;
        fo.beta = o.beta;
        fo.bias = o.bias;
    }
}

// Composite responses through per-axis passes (any ndim), mirroring the
// reference's sequence of gaussian_blur_into + elementwise kernels.
lucem_status composite_generic(lucem_ctx *ctx, const lucem_tensor *in, const lucem_response &r,
                               const std::vector<int> &axes, int mode, double cval, double truncate,
                               double scale, lucem_workspace *ws, void *stream) {
    const int64_t n = numel(in);
    float *out = static_cast<float *>(r.out.data);
    auto blur = [&](double sigma, int order_axis, uint32_t order, float *dst) -> lucem_status {
        std::vector<Pass> passes;
        for (int a : axes) {
            if (!(sigma > 0.0)) continue;
            uint32_t o = (a == order_axis) ? order : 0;
            passes.push_back(Pass{a, sigma, o, (int64_t)radius_of(truncate, sigma)});
        }
        return run_passes(ctx, in, passes, mode, cval, scale, dst, ws, stream);
    };
    auto slot = [&](const char *name, float **p) -> lucem_status {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
        void *v = nullptr;
        lucem_status st = ws->get(name, (size_t)n * sizeof(float), &v);
        *p = static_cast<float *>(v);
        return st;
    };
    lucem_status st;
    int e = 0;
    switch (r.kind) {
    case LUCEM_RESP_GAUSSIAN: return blur(r.sigma, -1, 0, out);
    case LUCEM_RESP_DOG: {  // gaussian.rs:374-390
        float *lo, *hi;
        if ((st = slot("dog_low", &lo)) || (st = slot("dog_high", &hi))) return st;
        if ((st = blur(r.sigma, -1, 0, lo)) || (st = blur(r.sigma2, -1, 0, hi))) return st;
        e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(lo, hi, out, n, 1.0f, -1.0f, 0.0f, stream); });
        break;
    }
    case LUCEM_RESP_LAPLACE: {  // gaussian.rs:255-288
        float *term;
        if ((st = slot("log_term", &term))) return st;
        for (size_t i = 0; i < axes.size(); ++i) {
            if (i == 0) {
                if ((st = blur(r.sigma, axes[i], 2, out))) return st;
            } else {
                if ((st = blur(r.sigma, axes[i], 2, term))) return st;
                if ((e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(out, term, out, n, 1.0f, 1.0f, 0.0f, stream); }))) break;
            }
        }
        break;
    }
    case LUCEM_RESP_GRAD_MAG: {  // gaussian.rs:307-356
        float *acc, *deriv;
        if ((st = slot("ggm_accum", &acc)) || (st = slot("ggm_deriv", &deriv))) return st;
        if ((e = timed(kPassElementwise, stream, [&] { return launch_fill(acc, n, 0.0f, stream); }))) break;
        for (int a : axes) {
            if ((st = blur(r.sigma, a, 1, deriv))) return st;
            if ((e = timed(kPassElementwise, stream, [&] { return launch_add_sq(deriv, acc, n, stream); }))) break;
        }
        if (!e) e = timed(kPassElementwise, stream, [&] { return launch_sqrt_scale(acc, out, n, 1.0f, stream); });
        break;
    }
    case LUCEM_RESP_UNSHARP: {  // gaussian.rs:407-421
        float *bl, *x = nullptr;
        if ((st = slot("unsharp_blur", &bl))) return st;
        if ((st = blur(r.sigma, -1, 0, bl))) return st;
        const float *xin = static_cast<const float *>(in->data);
        if (in->dtype != LUCEM_F32 || scale != 1.0) {
            if ((st = slot("unsharp_input", &x))) return st;
            if ((e = timed(kPassElementwise, stream, [&] { return launch_cast(in->data, in->dtype, (float)scale, x, n, stream); }))) break;
            xin = x;
        }
        e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(xin, bl, out, n, (float)(1.0 + r.amount), (float)(-r.amount), 0.0f, stream); });
        break;
    }
    default: return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `kind`: %d", r.kind);
    }
    return e ? cuda_fail(e, "elementwise launch") : ok();
}

lucem_status family_impl(lucem_ctx *ctx, const lucem_tensor *in, const lucem_response *responses,
                         int32_t n_responses, const std::vector<int> &axes, int32_t mode, double cval,
                         double truncate, double input_scale, lucem_workspace *ws, void *stream) {
    lucem_status st;
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if ((st = check_tensor("input", in))) return st;
    if ((st = check_mode(mode))) return st;
    if (n_responses < 0 || (n_responses > 0 && !responses))
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `responses`");
    for (int i = 0; i < n_responses; ++i) {
        if ((st = check_tensor("output", &responses[i].out))) return st;
        if ((st = same_shape("input", in, "output", &responses[i].out))) return st;
        if ((st = not_aliased(in, &responses[i].out))) return st;
        if ((st = require_f32_out(&responses[i].out))) return st;
    }
    FamilyPlan pl;
    if ((st = plan_family(responses, n_responses, &pl))) return st;
    if (numel(in) == 0 || n_responses == 0) return ok();
    const int nd = in->ndim;
    bool two_inner = nd >= 2 && axes.size() == 2 && axes[0] == nd - 2 && axes[1] == nd - 1;
    if (two_inner && family_fusable(pl, truncate)) {
        FamParams fp;
        init_fam(&fp, in, mode, cval, input_scale);
        build_fam(&fp, pl, truncate);
        for (int k = 0; k < n_responses; ++k) {
            fp.outs[k].out = static_cast<float *>(responses[k].out.data);
            fp.outs[k].plane_stride = (int64_t)fp.H * fp.W;
            fp.outs[k].row_pitch = fp.W;
        }
        if ((st = fam_waits(ws, &fp, stream))) return st;
        int e = timed(kPassFamily, stream, [&] { return launch_family_planes(fp, in->dtype, stream); });
        return e ? cuda_fail(e, "gaussian family launch") : ok();
    }
    for (int k = 0; k < n_responses; ++k)
        if ((st = composite_generic(ctx, in, responses[k], axes, mode, cval, truncate, input_scale, ws,
                                    stream)))
            return st;
    return ok();
}

std::vector<int> all_axes(int nd) {
    std::vector<int> a;
    for (int d = 0; d < nd; ++d) a.push_back(d);
    return a;
}

// Isotropic sigma list check: the family path takes one sigma for all axes.
bool isotropic(const double *s, int n, double *out) {
    if (n < 1) return false;
    for (int i = 1; i < n; ++i)
        if (s[i] != s[0]) return false;
    *out = s[0];
    return true;
}

lucem_status check_sigma_list(const char *name, const double *s, int n, int num_axes) {
    std::vector<double> v;
    lucem_status st = broadcast(name, s, n, num_axes, &v);
    if (st) return st;
    for (double x : v)
        if (!std::isfinite(x) || x < 0.0)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "invalid parameter `%s`: sigma must be non-negative and finite, got %g", name, x);
    return ok();
}

// Per-axis sigmas that differ: compose with generic blurs (run_passes).
lucem_status composite_axes(lucem_ctx *ctx, const lucem_tensor *in, int kind, const double *s1, int n1,
                            const double *s2, int n2, double amount, const lucem_gaussian_settings *gs,
                            lucem_tensor *out, lucem_workspace *ws, void *stream) {
    const int64_t n = numel(in);
    float *o = static_cast<float *>(out->data);
    auto blur = [&](const double *s, int ns, std::vector<uint32_t> orders, float *dst) -> lucem_status {
        lucem_gaussian_settings x = *gs;
        x.orders = orders.empty() ? gs->orders : orders.data();
        x.n_orders = orders.empty() ? gs->n_orders : (int32_t)orders.size();
        std::vector<Pass> passes;
        lucem_status st = plan_passes(in->ndim, s, ns, &x, &passes);
        if (st) return st;
        return run_passes(ctx, in, passes, gs->mode, gs->cval, gs->input_scale, dst, ws, stream);
    };
    auto slot = [&](const char *name, float **p) -> lucem_status {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
        void *v = nullptr;
        lucem_status st = ws->get(name, (size_t)n * sizeof(float), &v);
        *p = static_cast<float *>(v);
        return st;
    };
    lucem_status st;
    int e = 0;
    const int nd = in->ndim;
    if (kind == LUCEM_RESP_DOG) {
        float *lo, *hi;
        if ((st = slot("dog_low", &lo)) || (st = slot("dog_high", &hi))) return st;
        if ((st = blur(s1, n1, {}, lo)) || (st = blur(s2, n2, {}, hi))) return st;
        e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(lo, hi, o, n, 1.0f, -1.0f, 0.0f, stream); });
    } else if (kind == LUCEM_RESP_UNSHARP) {
        float *bl, *x = nullptr;
        if ((st = slot("unsharp_blur", &bl))) return st;
        if ((st = blur(s1, n1, {}, bl))) return st;
        const float *xin = static_cast<const float *>(in->data);
        if (in->dtype != LUCEM_F32 || gs->input_scale != 1.0) {
            if ((st = slot("unsharp_input", &x))) return st;
            if ((e = timed(kPassElementwise, stream, [&] { return launch_cast(in->data, in->dtype, (float)gs->input_scale, x, n, stream); })))
                return cuda_fail(e, "cast");
            xin = x;
        }
        e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(xin, bl, o, n, (float)(1.0 + amount), (float)(-amount), 0.0f, stream); });
    } else if (kind == LUCEM_RESP_LAPLACE) {
        float *term;
        if ((st = slot("log_term", &term))) return st;
        for (int ax = 0; ax < nd && !e; ++ax) {
            std::vector<uint32_t> ord(nd, 0);
            ord[ax] = 2;
            if (ax == 0) {
                if ((st = blur(s1, n1, ord, o))) return st;
            } else {
                if ((st = blur(s1, n1, ord, term))) return st;
                e = timed(kPassElementwise, stream, [&] { return launch_linear_comb(o, term, o, n, 1.0f, 1.0f, 0.0f, stream); });
            }
        }
    } else {  // gradient magnitude
        float *acc, *deriv;
        if ((st = slot("ggm_accum", &acc)) || (st = slot("ggm_deriv", &deriv))) return st;
        e = timed(kPassElementwise, stream, [&] { return launch_fill(acc, n, 0.0f, stream); });
        for (int ax = 0; ax < nd && !e; ++ax) {
            std::vector<uint32_t> ord(nd, 0);
            ord[ax] = 1;
            if ((st = blur(s1, n1, ord, deriv))) return st;
            e = timed(kPassElementwise, stream, [&] { return launch_add_sq(deriv, acc, n, stream); });
        }
        if (!e) e = timed(kPassElementwise, stream, [&] { return launch_sqrt_scale(acc, o, n, 1.0f, stream); });
    }
    return e ? cuda_fail(e, "elementwise launch") : ok();
}

// Shared front end of DoG / LoG / |grad| / unsharp.
lucem_status composite_entry(lucem_ctx *ctx, const lucem_tensor *in, int kind, const double *s1, int n1,
                             const double *s2, int n2, double amount,
                             const lucem_gaussian_settings *gs, lucem_tensor *out, lucem_workspace *ws,
                             void *stream) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_in_out(in, out))) return st;
    if ((st = check_mode(gs->mode))) return st;
    // Axes the composite filters (LoG / |grad| use all axes).
    std::vector<int> axes;
    if (kind == LUCEM_RESP_LAPLACE || kind == LUCEM_RESP_GRAD_MAG) {
        axes = all_axes(in->ndim);
    } else {
        std::vector<Pass> probe;
        lucem_gaussian_settings x = *gs;
        x.n_orders = 0;
        static const double one = 1.0;
        if ((st = plan_passes(in->ndim, &one, 1, &x, &probe))) return st;
        for (auto &p : probe) axes.push_back(p.axis);
    }
    if ((st = check_sigma_list("sigmas", s1, n1, (int)axes.size()))) return st;
    if (kind == LUCEM_RESP_DOG && (st = check_sigma_list("high_sigmas", s2, n2, (int)axes.size()))) return st;
    bool custom_orders = gs->n_orders > 0;
    for (int i = 0; i < gs->n_orders; ++i) custom_orders = custom_orders && gs->orders[i] != 0;
    double a = 0, b = 0;
    bool iso = isotropic(s1, n1, &a) && (kind != LUCEM_RESP_DOG || isotropic(s2, n2, &b)) &&
               gs->n_radii == 0 && !custom_orders;
    if (iso) {
        lucem_response r{};
        r.kind = kind;
        r.sigma = a;
        r.sigma2 = b;
        r.amount = amount;
        r.out = *out;
        return family_impl(ctx, in, &r, 1, axes, gs->mode, gs->cval, gs->truncate, gs->input_scale, ws,
                           stream);
    }
    return composite_axes(ctx, in, kind, s1, n1, s2, n2, amount, gs, out, ws, stream);
}

}  // namespace

extern "C" {

lucem_status lucem_difference_of_gaussians(lucem_ctx *ctx, const lucem_tensor *in,
                                           const double *low_sigmas, int32_t n_low,
                                           const double *high_sigmas, int32_t n_high,
                                           const lucem_gaussian_settings *settings,
                                           lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    return composite_entry(ctx, in, LUCEM_RESP_DOG, low_sigmas, n_low, high_sigmas, n_high, 0.0,
                           settings ? settings : &def, out, ws, stream);
}

lucem_status lucem_gaussian_laplace(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                    int32_t n_sigmas, int32_t mode, double cval, double truncate,
                                    lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_gaussian_settings s;
    lucem_gaussian_settings_default(&s);
    s.mode = mode;
    s.cval = cval;
    s.truncate = truncate;
    return composite_entry(ctx, in, LUCEM_RESP_LAPLACE, sigmas, n_sigmas, nullptr, 0, 0.0, &s, out, ws,
                           stream);
}

lucem_status lucem_gaussian_grad_mag(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                     int32_t n_sigmas, int32_t mode, double cval, double truncate,
                                     lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_gaussian_settings s;
    lucem_gaussian_settings_default(&s);
    s.mode = mode;
    s.cval = cval;
    s.truncate = truncate;
    return composite_entry(ctx, in, LUCEM_RESP_GRAD_MAG, sigmas, n_sigmas, nullptr, 0, 0.0, &s, out, ws,
                           stream);
}

lucem_status lucem_unsharp_mask(lucem_ctx *ctx, const lucem_tensor *in, const double *sigmas,
                                int32_t n_sigmas, double amount,
                                const lucem_gaussian_settings *settings, lucem_tensor *out,
                                lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    return composite_entry(ctx, in, LUCEM_RESP_UNSHARP, sigmas, n_sigmas, nullptr, 0, amount,
                           settings ? settings : &def, out, ws, stream);
}

lucem_status lucem_gaussian_family(lucem_ctx *ctx, const lucem_tensor *in,
                                   const lucem_response *responses, int32_t n_responses,
                                   int32_t mode, double cval, double truncate, double input_scale,
                                   lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_status st;
    if ((st = check_tensor("input", in))) return st;
    if (in->ndim < 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "gaussian_family expects >=2-D array, got %d-D shape %s",
                    in->ndim, dims_str(in).c_str());
    std::vector<int> axes = {in->ndim - 2, in->ndim - 1};
    return family_impl(ctx, in, responses, n_responses, axes, mode, cval, truncate, input_scale, ws,
                       stream);
}

// crates/lucem-core/src/tiling.rs:54-78.
lucem_status lucem_schedule(const int64_t dims[3], const int64_t block[3], const int64_t halo[3],
                            lucem_block *out, int64_t cap, int64_t *n_out) {
    if (!dims || !block || !halo || !n_out) return fail(LUCEM_ERR_INVALID_PARAMETER, "null argument");
    for (int a = 0; a < 3; ++a)
        if (dims[a] < 0 || block[a] < 0 || halo[a] < 0)
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `dims`: negative value");
    *n_out = 0;
    if (dims[0] == 0 || dims[1] == 0 || dims[2] == 0) return ok();
    int64_t step[3];
    for (int a = 0; a < 3; ++a) step[a] = block[a] == 0 ? dims[a] : std::min(block[a], dims[a]);
    int64_t count = 0;
    for (int64_t z = 0; z < dims[0]; z += step[0])
        for (int64_t y = 0; y < dims[1]; y += step[1])
            for (int64_t x = 0; x < dims[2]; x += step[2]) {
                if (out && count < cap) {
                    lucem_block &b = out[count];
                    int64_t o[3] = {z, y, x};
                    b.index = count;
                    for (int a = 0; a < 3; ++a) {
                        b.origin[a] = o[a];
                        b.size[a] = std::min(step[a], dims[a] - o[a]);
                        int64_t start = o[a] > halo[a] ? o[a] - halo[a] : 0;
                        int64_t end = std::min(o[a] + b.size[a] + halo[a], dims[a]);
                        b.read_origin[a] = start;
                        b.read_size[a] = end - start;
                    }
                }
                ++count;
            }
    *n_out = count;
    return ok();
}

lucem_status lucem_gaussian_family_tiles(lucem_ctx *ctx, const lucem_tensor *slide,
                                         const lucem_block *blocks, int64_t n_blocks,
                                         const lucem_response *responses, int32_t n_responses,
                                         int32_t mode, double cval, double truncate,
                                         double input_scale, int32_t persistent,
                                         lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    lucem_status st;
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    // The element cap applies per channel plane (crates/lucem-core/src/compute/limits.rs:12
    // bounds one buffer; the walk reads one block of one channel at a time).
    if ((st = check_tensor_cap("slide", slide, slide && slide->ndim == 3 ? 1 : 0))) return st;
    if (slide->ndim != 2 && slide->ndim != 3)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "gaussian_family_tiles expects 2-D or 3-D array, got %d-D shape %s",
                    slide->ndim, dims_str(slide).c_str());
    if ((st = check_mode(mode))) return st;
    const int nd = slide->ndim;
    const int64_t C = nd == 3 ? slide->dims[0] : 1, H = slide->dims[nd - 2], W = slide->dims[nd - 1];
    if (H >= (1 << 30) || W >= (1 << 30))
        return fail(LUCEM_ERR_TOO_MANY_ELEMENTS, "slide side exceeds 2^30");
    for (int i = 0; i < n_responses; ++i) {
        if ((st = check_tensor_cap("output", &responses[i].out, responses[i].out.ndim == 3 ? 1 : 0))) return st;
        if ((st = same_shape("slide", slide, "output", &responses[i].out))) return st;
        if ((st = not_aliased(slide, &responses[i].out))) return st;
        if ((st = require_f32_out(&responses[i].out))) return st;
    }
    if (n_blocks < 0 || (n_blocks > 0 && !blocks)) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `blocks`");
    FamilyPlan pl;
    if ((st = plan_family(responses, n_responses, &pl))) return st;
    if (!family_fusable(pl, truncate))
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `responses`: at most %d filters / %d outputs of radius <= %d per tiled walk",
                    kFamMaxFilters, kFamMaxOutputs, kFamMaxRadius);
    if (numel(slide) == 0 || n_blocks == 0 || n_responses == 0) return ok();
    int th, tw;
    family_tile_dims(&th, &tw);
    // Work list: every channel x every block (tiling.rs Block -> read / owned boxes).
    std::vector<FamWork> work;
    work.reserve((size_t)(C * n_blocks));
    int64_t tiles = 0;
    for (int64_t c = 0; c < C; ++c)
        for (int64_t i = 0; i < n_blocks; ++i) {
            const lucem_block &b = blocks[i];
            bool valid = b.read_origin[1] >= 0 && b.read_origin[2] >= 0 && b.read_size[1] > 0 &&
                         b.read_size[2] > 0 && b.read_origin[1] + b.read_size[1] <= H &&
                         b.read_origin[2] + b.read_size[2] <= W && b.origin[1] >= b.read_origin[1] &&
                         b.origin[2] >= b.read_origin[2] &&
                         b.origin[1] + b.size[1] <= b.read_origin[1] + b.read_size[1] &&
                         b.origin[2] + b.size[2] <= b.read_origin[2] + b.read_size[2] && b.size[1] > 0 &&
                         b.size[2] > 0;
            if (!valid)
                return fail(LUCEM_ERR_INVALID_PARAMETER,
                            "invalid parameter `blocks`: block %lld is outside the slide or its read box",
                            (long long)i);
            FamWork w;
            w.channel = (int32_t)c;
            w.read_y = (int32_t)b.read_origin[1];
            w.read_x = (int32_t)b.read_origin[2];
            w.read_h = (int32_t)b.read_size[1];
            w.read_w = (int32_t)b.read_size[2];
            w.own_y = (int32_t)b.origin[1];
            w.own_x = (int32_t)b.origin[2];
            w.own_h = (int32_t)b.size[1];
            w.own_w = (int32_t)b.size[2];
            w.tile_begin = (int32_t)tiles;
            tiles += ((b.size[1] + th - 1) / th) * ((b.size[2] + tw - 1) / tw);
            work.push_back(w);
        }
    if (tiles >= (int64_t)1 << 31) return fail(LUCEM_ERR_TOO_MANY_ELEMENTS, "too many tiles in one walk");
    // Upload the work list once per distinct list (it is then reused, which
    // also lets a CUDA graph capture later calls).
    void *wdev = nullptr;
    Slot *wslot = nullptr;
    size_t wbytes = work.size() * sizeof(FamWork);
    if ((st = ws->get("tile_work", wbytes + sizeof(int32_t) * 4, &wdev, &wslot))) return st;
    std::string key(reinterpret_cast<const char *>(work.data()), wbytes);
    if (wslot->key != key) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs);
        if (cs != cudaStreamCaptureStatusNone)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "a new tile list cannot be uploaded during stream capture: call once before capturing");
        CUDA_TRY(cudaMemcpyAsync(wdev, work.data(), wbytes, cudaMemcpyHostToDevice,
                                 static_cast<cudaStream_t>(stream)),
                 "uploading the tile list");
        CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "tile list upload");
        wslot->key = key;
    }
    void *cnt = nullptr;
    if ((st = ws->get("tile_counter", 64, &cnt))) return st;

    FamParams fp;
    std::memset(&fp, 0, sizeof fp);
    fp.in = slide->data;
    fp.H = (int32_t)H;
    fp.W = (int32_t)W;
    fp.B = (int32_t)C;
    fp.in_plane_stride = H * W;
    fp.in_row_pitch = W;
    fp.mode = mode;
    fp.cval = (float)cval;
    fp.in_scale = (float)input_scale;
    build_fam(&fp, pl, truncate);
    for (int k = 0; k < n_responses; ++k) {
        fp.outs[k].out = static_cast<float *>(responses[k].out.data);
        fp.outs[k].plane_stride = H * W;
        fp.outs[k].row_pitch = W;
    }
    const FamWork *wd = static_cast<const FamWork *>(wdev);
    int e = 0;
    if (persistent) {
        // The launcher caps the grid at the CTAs that are resident at once.
        e = tuned_launch(ctx, plan_key(ctx, "walk", slide->dtype, fp, (int64_t)tiles), walk_candidates(), &fp, stream,
                         [&] {
                             int r = (int)cudaMemsetAsync(cnt, 0, sizeof(int32_t), static_cast<cudaStream_t>(stream));
                             if (r) return r;
                             return timed(kPassFamily, stream, [&] {
                                 return launch_family_work(fp, slide->dtype, wd, (int32_t)work.size(), (int32_t)tiles,
                                                           0, static_cast<int32_t *>(cnt), ctx->sms * 4, stream);
                             });
                         });
    } else {
        for (size_t i = 0; i < work.size() && !e; ++i) {
            int32_t t0 = work[i].tile_begin;
            int32_t t1 = i + 1 < work.size() ? work[i + 1].tile_begin : (int32_t)tiles;
            // One launch per block and channel: the plain per-tile drop-in.
            e = timed(kPassFamily, stream, [&] { return launch_family_work(fp, slide->dtype, wd + i, 1, t1 - t0, t0, nullptr, 0, stream); });
        }
    }
    return e ? cuda_fail(e, "tiled family launch") : ok();
}

lucem_status lucem_gaussian_batch(lucem_ctx *ctx, int32_t n, const lucem_tensor *ins, lucem_tensor *outs,
                                  const int32_t *set_ids, int32_t n_sets, const double *set_sigmas, int32_t mode,
                                  double cval, double truncate, double input_scale, lucem_workspace *ws,
                                  void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (n < 1 || !ins || !outs || !set_ids)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `n`: a batch needs at least one image");
    if (n_sets < 1 || !set_sigmas)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `n_sets`: at least one sigma set");
    lucem_status st;
    if ((st = check_mode(mode))) return st;
    for (int s2 = 0; s2 < n_sets; ++s2) {
        const double sg = set_sigmas[s2];
        if (!std::isfinite(sg) || sg < 0.0)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "invalid parameter `sigmas`: sigma must be non-negative and finite, got %g", sg);
        if (sg > 0.0 && radius_of(truncate, sg) > kFamMaxRadius)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "invalid parameter `sigmas`: radius %d of sigma %g exceeds the batched kernel's %d",
                        (int)radius_of(truncate, sg), sg, kFamMaxRadius);
    }
    for (int i = 0; i < n; ++i) {
        if ((st = check_in_out(&ins[i], &outs[i]))) return st;
        if (ins[i].ndim != 2)
            return fail(LUCEM_ERR_INVALID_DIMENSION, "gaussian_batch takes 2-D images, image %d is %d-D", i, ins[i].ndim);
        if (ins[i].dtype != ins[0].dtype)
            return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "gaussian_batch: every image has the first image's dtype");
        if (set_ids[i] < 0 || set_ids[i] >= n_sets)
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `set_ids`: image %d has set %d of %d", i,
                        set_ids[i], n_sets);
    }
    int th = kFamTile, tw = kFamTile;
    family_tile_dims(&th, &tw);
    // Work list: images grouped by sigma set, each set's tiles numbered from 0.
    std::vector<FamImage> items;
    std::vector<int32_t> set_begin((size_t)n_sets + 1, 0), set_tiles((size_t)n_sets, 0);
    for (int s2 = 0; s2 < n_sets; ++s2) {
        set_begin[(size_t)s2] = (int32_t)items.size();
        int64_t t = 0;
        for (int i = 0; i < n; ++i) {
            if (set_ids[i] != s2 || numel(&ins[i]) == 0) continue;
            FamImage it{};
            it.in = ins[i].data;
            it.out = static_cast<float *>(outs[i].data);
            it.H = (int32_t)ins[i].dims[0];
            it.W = (int32_t)ins[i].dims[1];
            it.in_pitch = it.W;
            it.out_pitch = it.W;
            it.tile_begin = (int32_t)t;
            t += ((int64_t)(it.H + th - 1) / th) * ((it.W + tw - 1) / tw);
            if (t > INT32_MAX) return fail(LUCEM_ERR_TOO_MANY_ELEMENTS, "gaussian_batch: too many tiles in one set");
            items.push_back(it);
        }
        set_tiles[(size_t)s2] = (int32_t)t;
    }
    set_begin[(size_t)n_sets] = (int32_t)items.size();
    if (items.empty()) return ok();
    // Upload the work list once per distinct list (then calls only launch).
    void *wdev = nullptr;
    Slot *wslot = nullptr;
    const size_t wbytes = items.size() * sizeof(FamImage);
    if ((st = ws->get("gauss_batch_items", wbytes, &wdev, &wslot))) return st;
    std::string key(reinterpret_cast<const char *>(items.data()), wbytes);
    if (wslot->key != key) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs);
        if (cs != cudaStreamCaptureStatusNone)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "a new image list cannot be uploaded during stream capture: call once before capturing");
        CUDA_TRY(cudaMemcpyAsync(wdev, items.data(), wbytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)),
                 "uploading the image list");
        CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)), "image list upload");
        wslot->key = key;
    }
    const FamImage *idev = static_cast<const FamImage *>(wdev);
    for (int s2 = 0; s2 < n_sets; ++s2) {
        const int32_t b = set_begin[(size_t)s2], cnt = set_begin[(size_t)s2 + 1] - b;
        if (cnt == 0) continue;
        const double sg = set_sigmas[s2];
        int e = 0;
        if (!(sg > 0.0)) {
            // sigma 0: the reference copies the input (gaussian.rs:102-104).
            for (int32_t k = 0; k < cnt && !e; ++k) {
                const FamImage &it = items[(size_t)(b + k)];
                e = timed(kPassElementwise, stream, [&] {
                    return launch_cast(it.in, ins[0].dtype, (float)input_scale, it.out, (int64_t)it.H * it.W, stream);
                });
            }
        } else {
            const int64_t r = (int64_t)radius_of(truncate, sg);
            const GaussPass rows{0, sg, 0, r}, cols{1, sg, 0, r};
            FamParams fp;
            lucem_tensor view = ins[0];
            gaussian_fused_params(&fp, &view, mode, cval, (float)input_scale, rows, cols, nullptr);
            e = tuned_launch(ctx, plan_key(ctx, "batch", ins[0].dtype, fp, set_tiles[(size_t)s2]), {1, 1 + kPlanAhead},
                             &fp, stream, [&] {
                                 return timed(kPassFamily, stream, [&] {
                                     return launch_family_batch(fp, ins[0].dtype, idev + b, cnt,
                                                                set_tiles[(size_t)s2], stream);
                                 });
                             });
        }
        if (e) return cuda_fail(e, "gaussian_batch launch");
    }
    return ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Richardson-Lucy.

namespace {

// Extension halo along one axis: zero padding needs none; the other modes
// extend by k/2 on each side (the reference's correlation reads at most k/2
// samples past either border of the image).
int64_t rl_halo(int64_t k, int mode) { return mode == LUCEM_PAD_CONSTANT ? 0 : k / 2; }

// Smallest grid length that keeps the circular correlation equal to the
// padded linear one: n + k/2 for zero padding (the correlation reaches
// k - 1 - k/2 <= k/2 samples past one side), n + 2*(k/2) with an extension.
int64_t rl_min_length(int64_t n, int64_t k, int mode) {
    return mode == LUCEM_PAD_CONSTANT ? n + k / 2 : n + 2 * (k / 2);
}

bool good_factors(int64_t n) {
    if (n < 1) return false;
    for (int f : {2, 3, 5, 7})
        while (n % f == 0) n /= f;
    return n == 1;
}

// ---- batched 2-D Richardson-Lucy, FFT-length autotuning -------------------

// Relative cost per transformed element of one pass at length n (kind 0:
// column pass, 1: row pass): the autotuned figure when one was measured for
// this context (ctx may be null), else 1 for the register-resident
// power-of-two kernels and, for the shared-memory Stockham kernels (other
// 2/3/5/7-smooth lengths), the ratio measured on B200: 5 (columns), 2.7 (rows).
double length_cost(lucem_ctx *ctx, int kind, int64_t n) {
    auto fast = [kind](int64_t m) {
        const bool pow2 = (m & (m - 1)) == 0;
        return kind == 0 ? (pow2 && m >= 64 && m <= 2048) : (pow2 && m >= 128 && m <= 2048);
    };
    const double slow = kind == 0 ? 5.0 : 2.7;
    if (!ctx) return fast(n) ? 1.0 : slow;
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->tune.find({kind, n});
    if (it != ctx->tune.end()) return it->second;
    // Untuned length: the default ratio, in the units of the tuned entries of
    // this kind when there are any (their mean over the fast lengths).
    double base = 0.0;
    int cnt = 0;
    for (auto &kv : ctx->tune)
        if (kv.first.first == kind && fast(kv.first.second)) {
            base += kv.second;
            ++cnt;
        }
    base = cnt ? base / cnt : 1.0;
    return base * (fast(n) ? 1.0 : slow);
}

// The grid length chosen for a need: the cheapest of m * 2^k >= need (m in a
// short list, so that uneven problems of a batch fall into few length groups,
// one launch each) by length * cost.
int64_t batch_length(lucem_ctx *ctx, int kind, int64_t need) {
    static const int ms[] = {1, 3, 5, 7, 9, 15, 21, 25, 27};
    int64_t best = 0;
    double best_cost = 0.0;
    for (int m : ms) {
        int64_t n = m;
        while (n < need || (kind == 1 && (n & 1))) n *= 2;
        if (n > 2 * need + 64) continue;
        if (kind == 1 && (n / 2) < 2) continue;
        const double c = (double)n * length_cost(ctx, kind, n);
        if (best == 0 || c < best_cost || (c == best_cost && n < best)) {
            best = n;
            best_cost = c;
        }
    }
    return best > 0 ? best : fft_good_length(need, kind == 1);
}

lucem_status rl_grid_impl(const int64_t *dims, const int64_t *kdims, int ndim, int mode,
                          const int64_t *requested, int64_t *grid, lucem_ctx *ctx = nullptr) {
    for (int d = 0; d < ndim; ++d) {
        bool x_axis = d == ndim - 1;
        int64_t need = rl_min_length(dims[d], kdims[d], mode);
        int64_t r = requested ? requested[d] : 0;
        if (r > 0) {
            if (r < need)
                return fail(LUCEM_ERR_INVALID_PARAMETER,
                            "invalid parameter `grid`: axis %d length %lld is below the %lld the padding needs",
                            d, (long long)r, (long long)need);
            if (!good_factors(r) || (x_axis && (r & 1)))
                return fail(LUCEM_ERR_INVALID_PARAMETER,
                            "invalid parameter `grid`: axis %d length %lld must factor into 2, 3, 5, 7%s",
                            d, (long long)r, x_axis ? " and be even" : "");
            grid[d] = r;
        } else {
            grid[d] = batch_length(ctx, x_axis ? 1 : 0, need);
        }
        if (grid[d] > 16384)
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `grid`: axis %d length %lld exceeds 16384",
                        d, (long long)grid[d]);
    }
    return ok();
}

// Twiddle tables e^{-2 pi i m / n}, m < n, from double-precision cos/sin;
// f32 copies are rounded once from the f64 values.
lucem_status twiddles(lucem_ctx *ctx, int64_t n, const float2_ **f32, const double **f64) {
    std::vector<double> d((size_t)(2 * n));
    for (int64_t m = 0; m < n; ++m) {
        // Reduce the angle to the first octant's accuracy by exact symmetry.
        double a = 2.0 * M_PI * (double)m / (double)n;
        d[2 * m] = std::cos(a);
        d[2 * m + 1] = -std::sin(a);
    }
    // Exact values at the quarter points.
    for (int64_t m = 0; m < n; ++m) {
        if ((4 * m) % n == 0) {
            int64_t q = (4 * m) / n;
            const double re[4] = {1, 0, -1, 0}, im[4] = {0, -1, 0, 1};
            d[2 * m] = re[q];
            d[2 * m + 1] = im[q];
        }
    }
    std::vector<float> f((size_t)(2 * n));
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)d[i];
    int err = 0;
    std::string k = "tw-f32-" + std::to_string(n);
    void *pf = ctx->get_or_upload(k, f.data(), f.size() * sizeof(float), &err);
    if (!pf) return cuda_fail(err, "twiddle upload");
    k = "tw-f64-" + std::to_string(n);
    void *pd = ctx->get_or_upload(k, d.data(), d.size() * sizeof(double), &err);
    if (!pd) return cuda_fail(err, "twiddle upload");
    *f32 = static_cast<const float2_ *>(pf);
    *f64 = static_cast<const double *>(pd);
    return ok();
}

// Argument checks of the RL-family entry points
// (crates/lucem-ops/src/restore/deconvolve.rs:53-71, same order).
lucem_status rl_check(const lucem_tensor *in, const lucem_tensor *psf, const lucem_tensor *out, int32_t num_iter,
                      int32_t mode, const char *what) {
    lucem_status st;
    if ((st = check_tensor("input", in)) || (st = check_tensor("output", out)) || (st = check_tensor("psf", psf)))
        return st;
    if ((st = same_shape("input", in, "output", out))) return st;
    if ((st = not_aliased(in, out))) return st;
    // A leading batch axis on the input (one more axis than the PSF): the
    // images or volumes share the PSF.
    const bool batched = in->ndim == psf->ndim + 1 && (psf->ndim == 2 || psf->ndim == 3);
    const int nd = batched ? psf->ndim : in->ndim;
    if (nd != 2 && nd != 3)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "%s input expects 2 or 3-D array, got %d-D shape %s", what,
                    in->ndim, dims_str(in).c_str());
    if (!batched && psf->ndim != in->ndim)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "%s psf expects %d-D array, got %d-D shape %s", what, in->ndim,
                    psf->ndim, dims_str(psf).c_str());
    if (numel(psf) == 0) return fail(LUCEM_ERR_INVALID_WEIGHTS, "psf: PSF cannot be empty");
    if (num_iter < 1) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `num_iter`: num_iter must be >= 1");
    if (in->dtype != LUCEM_F32 || psf->dtype != LUCEM_F32 || out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "%s takes f32 input, psf and output", what);
    return check_mode(mode);
}

// deconvolve.rs:104.
float rl_eps(const lucem_rl_settings *s) {
    const double eps = s->has_filter_epsilon ? s->filter_epsilon : 1e-12;
    return (float)std::max(eps, 1e-15);
}

// One problem's geometry, transfer functions and spectrum buffers.
struct RlSetup {
    RlGeom g{};
    RlBuffers b{};
    int64_t kd[3] = {1, 1, 1}, grid[3] = {1, 1, 1};
    int64_t kn = 0;
    int32_t c_conv[3] = {0, 0, 0}, c_corr[3] = {0, 0, 0};
    bool same_centre = true;
    bool norm_active = false;  // the PSF was scaled by norm = 1 / sum(psf)
    double norm = 1.0;
    std::vector<double> pn;    // the PSF the transfer functions were built from (f64)
};

// Geometry, PSF (normalised on the host in f64 when `normalise`, as
// deconvolve.rs:77-88 does), transfer functions (cached per workspace by
// content) and the two spectrum buffers.  Synchronises the stream once (the
// PSF download) and once more when the transfer functions are rebuilt.
lucem_status rl_prepare(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf, int32_t mode,
                        const int64_t *grid_req, bool normalise, lucem_workspace *ws, void *stream, RlSetup *su) {
    lucem_status st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    // in: [nb,] + the PSF's rank (rl_check); the nb volumes share the PSF.
    const int nd = psf->ndim, boff = in->ndim - nd;
    int64_t dims[3] = {1, 1, 1};
    for (int d = 0; d < nd; ++d) {
        dims[3 - nd + d] = in->dims[boff + d];
        su->kd[3 - nd + d] = psf->dims[d];
    }
    const int64_t nb = boff ? in->dims[0] : 1;
    int64_t req[3] = {0, 0, 0};
    for (int d = 0; d < nd; ++d) req[3 - nd + d] = grid_req ? grid_req[d] : 0;
    if ((st = rl_grid_impl(dims + (3 - nd), su->kd + (3 - nd), nd, mode, req + (3 - nd), su->grid + (3 - nd),
                           ctx)))
        return st;
    const int64_t *kd = su->kd, *grid = su->grid;
    RlGeom &g = su->g;
    g.ndim = nd;
    g.Z = (int32_t)dims[0]; g.Y = (int32_t)dims[1]; g.X = (int32_t)dims[2];
    g.Pz = (int32_t)grid[0]; g.Py = (int32_t)grid[1]; g.Px = (int32_t)grid[2];
    g.hz = nd == 3 ? (int32_t)rl_halo(kd[0], mode) : 0;
    g.hy = (int32_t)rl_halo(kd[1], mode);
    g.hx = (int32_t)rl_halo(kd[2], mode);
    g.Hx = g.Px / 2 + 1;
    g.Hp = (g.Hx + 15) & ~15;
    g.mode = mode;
    g.nb = (int32_t)nb;

    const int64_t kn = numel(psf);
    su->kn = kn;
    std::vector<float> hp((size_t)kn);
    CUDA_TRY(cudaMemcpyAsync(hp.data(), psf->data, (size_t)kn * sizeof(float), cudaMemcpyDeviceToHost, cs),
             "psf download");
    CUDA_TRY(cudaStreamSynchronize(cs), "psf download");
    double sum = 0.0;
    for (float v : hp) sum += (double)v;
    su->norm_active = normalise && std::fabs(sum) > 1e-12;
    su->norm = su->norm_active ? 1.0 / sum : 1.0;
    su->pn.resize((size_t)kn);
    for (int64_t i = 0; i < kn; ++i) su->pn[(size_t)i] = (double)hp[(size_t)i] * su->norm;
    const std::vector<double> &pn = su->pn;

    const float2_ *tw32[3];
    const double *tw64[3];
    for (int d = 0; d < 3; ++d)
        if ((st = twiddles(ctx, grid[d], &tw32[d], &tw64[d]))) return st;

    // Transfer functions: convolution with the PSF centred at k-1-k/2 and
    // correlation with it centred at k/2 (convolve.rs:144-145 with the flip at
    // deconvolve.rs:82-88); equal for odd sizes.
    int32_t kdi[3] = {(int32_t)kd[0], (int32_t)kd[1], (int32_t)kd[2]};
    su->same_centre = true;
    for (int d = 0; d < 3; ++d) {
        su->c_conv[d] = (int32_t)(kd[d] - 1 - kd[d] / 2);
        su->c_corr[d] = (int32_t)(kd[d] / 2);
        su->same_centre = su->same_centre && su->c_conv[d] == su->c_corr[d];
    }
    const bool same_centre = su->same_centre;
    // A separable PSF (p = mz (x) my (x) mx / S^2 with the axis marginals, S =
    // sum p, to 1e-6 of max |p|: the Gaussian PSFs) gets a factored transfer
    // function built on the host: the z (3-D) or y (2-D) factor stays a
    // vector and the pass multiplies it in, so no dense [Pz][Py][Hp] array is
    // streamed through the passes.
    std::vector<double> marg[3];
    bool separable = false;
    {
        double S = 0.0, pmax = 0.0;
        for (int d = 0; d < 3; ++d) marg[d].assign((size_t)kd[d], 0.0);
        for (int64_t z = 0; z < kd[0]; ++z)
            for (int64_t y = 0; y < kd[1]; ++y)
                for (int64_t x = 0; x < kd[2]; ++x) {
                    const double v = pn[(size_t)((z * kd[1] + y) * kd[2] + x)];
                    marg[0][(size_t)z] += v;
                    marg[1][(size_t)y] += v;
                    marg[2][(size_t)x] += v;
                    S += v;
                    pmax = std::max(pmax, std::fabs(v));
                }
        if (std::fabs(S) > 1e-12 && pmax > 0.0) {
            double err = 0.0;
            for (int64_t z = 0; z < kd[0]; ++z)
                for (int64_t y = 0; y < kd[1]; ++y)
                    for (int64_t x = 0; x < kd[2]; ++x) {
                        const double prod = marg[0][(size_t)z] * marg[1][(size_t)y] * marg[2][(size_t)x] / (S * S);
                        err = std::max(err, std::fabs(pn[(size_t)((z * kd[1] + y) * kd[2] + x)] - prod));
                    }
            separable = err <= 1e-6 * pmax && kn > 1;
            for (double &v : marg[2]) v /= S * S;
        }
    }
    const size_t hbytes = separable ? (size_t)(nd == 3 ? g.Py : 1) * g.Hp * sizeof(float2_)
                                    : (size_t)g.Pz * g.Py * g.Hp * sizeof(float2_);
    const int64_t nrow = nd == 3 ? g.Pz : g.Py;
    std::string key(reinterpret_cast<const char *>(pn.data()), pn.size() * sizeof(double));
    key.append(reinterpret_cast<const char *>(kdi), sizeof kdi);
    key.append(reinterpret_cast<const char *>(grid), 3 * sizeof(int64_t));
    key.append(reinterpret_cast<const char *>(&g.Hp), sizeof g.Hp);
    key.push_back(separable ? 's' : 'd');
    key.push_back((char)('0' + nd));
    void *h_conv = nullptr, *h_corr = nullptr, *r_conv = nullptr, *r_corr = nullptr;
    Slot *sl_conv = nullptr, *sl_corr = nullptr;
    if ((st = ws->get("rl_otf_conv", hbytes, &h_conv, &sl_conv))) return st;
    if (!same_centre && (st = ws->get("rl_otf_corr", hbytes, &h_corr, &sl_corr))) return st;
    void *y_conv = nullptr, *y_corr = nullptr, *x_conv = nullptr, *x_corr = nullptr;
    if (separable) {
        if ((st = ws->get("rl_otf_conv_row", (size_t)nrow * sizeof(float2_), &r_conv))) return st;
        if (!same_centre && (st = ws->get("rl_otf_corr_row", (size_t)nrow * sizeof(float2_), &r_corr))) return st;
        if (nd == 3) {
            if ((st = ws->get("rl_otf_conv_y", (size_t)g.Py * sizeof(float2_), &y_conv))) return st;
            if ((st = ws->get("rl_otf_conv_x", (size_t)g.Hp * sizeof(float2_), &x_conv))) return st;
            if (!same_centre) {
                if ((st = ws->get("rl_otf_corr_y", (size_t)g.Py * sizeof(float2_), &y_corr))) return st;
                if ((st = ws->get("rl_otf_corr_x", (size_t)g.Hp * sizeof(float2_), &x_corr))) return st;
            }
        }
    }
    if (same_centre) {
        h_corr = h_conv;
        r_corr = r_conv;
        y_corr = y_conv;
        x_corr = x_conv;
    }
    const bool fresh = sl_conv->key != key || (!same_centre && sl_corr->key != key);
    if (fresh && separable) {
        // 1-D DFTs of the marginals at each centre, f64 (exact integer angle
        // reduction), scale 1/(Pz Py Px) folded into the table.
        auto dft = [](const std::vector<double> &m, int64_t c, int64_t P, int64_t nbins) {
            std::vector<double> out((size_t)(2 * nbins), 0.0);
            for (int64_t k = 0; k < nbins; ++k) {
                double re = 0.0, im = 0.0;
                for (int64_t s2 = 0; s2 < (int64_t)m.size(); ++s2) {
                    const int64_t q = (((k * (s2 - c)) % P) + P) % P;
                    const double a = 2.0 * M_PI * (double)q / (double)P;
                    re += m[(size_t)s2] * std::cos(a);
                    im -= m[(size_t)s2] * std::sin(a);
                }
                out[(size_t)(2 * k)] = re;
                out[(size_t)(2 * k + 1)] = im;
            }
            return out;
        };
        const double scale = 1.0 / ((double)g.Pz * (double)g.Py * (double)g.Px);
        cudaStream_t cs2 = static_cast<cudaStream_t>(stream);
        std::vector<float> tab, rowv, yv, xv;
        auto build = [&](const int32_t *cen, void *hdst, void *rdst, void *ydst, void *xdst) -> lucem_status {
            const std::vector<double> fz = dft(marg[0], cen[0], g.Pz, g.Pz);
            const std::vector<double> fy = dft(marg[1], cen[1], g.Py, g.Py);
            const std::vector<double> fx = dft(marg[2], cen[2], g.Px, g.Hx);
            const int64_t ny = nd == 3 ? g.Py : 1;
            tab.assign((size_t)(2 * ny * g.Hp), 0.0f);
            for (int64_t y = 0; y < ny; ++y)
                for (int64_t x = 0; x < g.Hx; ++x) {
                    // 3-D: Fy(y) Fx(x); 2-D: Fz(0) Fx(x) (Fz(0) = the z marginal's sum).
                    const double ar = nd == 3 ? fy[(size_t)(2 * y)] : fz[0];
                    const double ai = nd == 3 ? fy[(size_t)(2 * y + 1)] : fz[1];
                    const double br = fx[(size_t)(2 * x)], bi = fx[(size_t)(2 * x + 1)];
                    tab[(size_t)(2 * (y * g.Hp + x))] = (float)((ar * br - ai * bi) * scale);
                    tab[(size_t)(2 * (y * g.Hp + x) + 1)] = (float)((ar * bi + ai * br) * scale);
                }
            const std::vector<double> &fr = nd == 3 ? fz : fy;
            rowv.assign(fr.begin(), fr.end());
            CUDA_TRY(cudaMemcpyAsync(hdst, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice, cs2),
                     "transfer function upload");
            CUDA_TRY(cudaMemcpyAsync(rdst, rowv.data(), rowv.size() * sizeof(float), cudaMemcpyHostToDevice, cs2),
                     "transfer function upload");
            if (ydst) {
                // Per-axis factors of the 3-D table: Fy alone, Fx with the scale.
                yv.assign(fy.begin(), fy.end());
                xv.assign((size_t)(2 * g.Hp), 0.0f);
                for (int64_t x = 0; x < g.Hx; ++x) {
                    xv[(size_t)(2 * x)] = (float)(fx[(size_t)(2 * x)] * scale);
                    xv[(size_t)(2 * x + 1)] = (float)(fx[(size_t)(2 * x + 1)] * scale);
                }
                CUDA_TRY(cudaMemcpyAsync(ydst, yv.data(), yv.size() * sizeof(float), cudaMemcpyHostToDevice, cs2),
                         "transfer function upload");
                CUDA_TRY(cudaMemcpyAsync(xdst, xv.data(), xv.size() * sizeof(float), cudaMemcpyHostToDevice, cs2),
                         "transfer function upload");
            }
            // The host tables are reused for the second centre.
            CUDA_TRY(cudaStreamSynchronize(cs2), "transfer function upload");
            return ok();
        };
        if ((st = build(su->c_conv, h_conv, r_conv, y_conv, x_conv))) return st;
        if (!same_centre && (st = build(su->c_corr, h_corr, r_corr, y_corr, x_corr))) return st;
        sl_conv->key = key;
        if (sl_corr) sl_corr->key = key;
    } else if (fresh) {
        void *psf64 = nullptr, *wa = nullptr, *wb = nullptr;
        if ((st = ws->get("rl_psf64", (size_t)kn * sizeof(double), &psf64))) return st;
        if ((st = ws->get("rl_otf_a", (size_t)kd[0] * kd[1] * g.Hp * 16, &wa))) return st;
        if ((st = ws->get("rl_otf_b", (size_t)kd[0] * g.Py * g.Hp * 16, &wb))) return st;
        CUDA_TRY(cudaMemcpyAsync(psf64, pn.data(), (size_t)kn * sizeof(double), cudaMemcpyHostToDevice, cs),
                 "psf upload");
        if (ws->t()) ws->t()->begin(kPassRlOtf, stream);
        int e = rl_launch_otf(g, static_cast<const double *>(psf64), kdi, su->c_conv, static_cast<double *>(wa),
                              static_cast<double *>(wb), h_conv, tw64[2], tw64[1], tw64[0], stream);
        if (ws->t()) ws->t()->end(kPassRlOtf, stream);
        if (e) return cuda_fail(e, "transfer function launch");
        if (!same_centre) {
            e = rl_launch_otf(g, static_cast<const double *>(psf64), kdi, su->c_corr, static_cast<double *>(wa),
                              static_cast<double *>(wb), h_corr, tw64[2], tw64[1], tw64[0], stream);
            if (e) return cuda_fail(e, "transfer function launch");
        }
        // The host PSF copy must outlive the upload.
        CUDA_TRY(cudaStreamSynchronize(cs), "transfer function");
        sl_conv->key = key;
        if (sl_corr) sl_corr->key = key;
    }

    void *s1 = nullptr, *s2 = nullptr;
    if ((st = ws->get("rl_s1", (size_t)nb * g.Z * g.Y * g.Hp * sizeof(float2_), &s1))) return st;
    if (nd == 3 && (st = ws->get("rl_s2", (size_t)nb * g.Z * g.Py * g.Hp * sizeof(float2_), &s2))) return st;
    RlBuffers &b = su->b;
    b.s1 = s1;
    b.s2 = s2;
    b.h_conv = h_conv;
    b.h_corr = h_corr;
    b.hrow_conv = separable ? r_conv : nullptr;
    b.hrow_corr = separable ? r_corr : nullptr;
    b.hy_conv = y_conv;
    b.hy_corr = y_corr;
    b.hx_conv = x_conv;
    b.hx_corr = x_corr;
    b.tw_x = tw32[2];
    b.tw_y = tw32[1];
    b.tw_z = tw32[0];
    return ok();
}

// Workspace buffers of the reverse passes: the full set for the unrolled
// iterations (full_rl), or the few the convolution's gradient needs.
lucem_status rl_bwd_buffers(const RlSetup &su, int T, int K, bool full_rl, lucem_workspace *ws, RlBwdBuffers *w) {
    lucem_status st;
    const RlGeom &g = su.g;
    // Volumes and per-volume spectra hold every volume of a batch; the
    // accumulated cross-spectra (pbar) and the full-grid buffers one.
    const size_t nb = g.nb > 1 ? (size_t)g.nb : 1;
    const size_t vb = nb * g.Z * g.Y * g.X * sizeof(float);
    const size_t sb = (size_t)g.Pz * g.Py * g.Hp * sizeof(float2_);
    std::memset(w, 0, sizeof *w);
    void *p = nullptr;
    auto vol = [&](const char *name, size_t count, float **dst) -> lucem_status {
        lucem_status s2 = ws->get(name, vb * count, &p);
        if (!s2) *dst = static_cast<float *>(p);
        return s2;
    };
    auto spec = [&](const char *name, float2_ **dst, size_t count = 1) -> lucem_status {
        lucem_status s2 = ws->get(name, sb * count, &p);
        if (!s2) *dst = static_cast<float2_ *>(p);
        return s2;
    };
    if (full_rl) {
        const int nseg = (T + K - 1) / K;
        if ((st = vol("rlb_ckpt", (size_t)nseg, &w->ckpt)) || (st = vol("rlb_seg", (size_t)K, &w->seg))) return st;
        const char *names[8] = {"rlb_c", "rlb_r", "rlb_a", "rlb_abar", "rlb_rbar", "rlb_cbar", "rlb_t", "rlb_ebar"};
        float **dst[8] = {&w->c, &w->r, &w->a, &w->abar, &w->rbar, &w->cbar, &w->t, &w->ebar};
        for (int i = 0; i < 8; ++i)
            if ((st = vol(names[i], 1, dst[i]))) return st;
        if ((st = spec("rlb_spec_r", &w->spec_r, nb)) || (st = spec("rlb_spec_abar", &w->spec_abar, nb))) return st;
        if (!su.same_centre && (st = spec("rlb_pbar2", &w->pbar2))) return st;
    } else {
        if ((st = vol("rlb_c", 1, &w->c)) || (st = vol("rlb_t", 1, &w->t))) return st;
    }
    if ((st = spec("rlb_spec_e", &w->spec_e, nb)) || (st = spec("rlb_spec_cbar", &w->spec_cbar, nb)) ||
        (st = spec("rlb_pbar1", &w->pbar1)))
        return st;
    const size_t fz = g.ndim == 3 ? (size_t)g.Pz : 1;
    if ((st = ws->get("rlb_full_s1", fz * g.Py * g.Hp * sizeof(float2_), &w->full_s1))) return st;
    if (g.ndim == 3 && (st = ws->get("rlb_full_s2", fz * g.Py * g.Hp * sizeof(float2_), &w->full_s2))) return st;
    if ((st = ws->get("rlb_full_real", fz * g.Py * g.Px * sizeof(float), &p))) return st;
    w->full_real = static_cast<float *>(p);
    for (int d = 0; d < 3; ++d) {
        w->kdims[d] = (int32_t)su.kd[d];
        w->c_conv[d] = su.c_conv[d];
        w->c_corr[d] = su.c_corr[d];
    }
    return ok();
}

// d loss / d psf from d loss / d (the PSF the transfer functions were built
// from).  Through the host normalisation p_n = p * norm, norm = 1 / sum(p):
// g_p = norm * (g_n - sum(g_n * p_n)).  gcorr (even sides) adds the
// correlation's lags.  Synchronises the stream.
lucem_status psf_grad_finish(const RlSetup &su, const float *gconv, const float *gcorr, bool normalised,
                             lucem_tensor *grad_psf, void *stream) {
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    const int64_t kn = su.kn;
    std::vector<float> a((size_t)kn), b(gcorr ? (size_t)kn : 0);
    CUDA_TRY(cudaMemcpyAsync(a.data(), gconv, (size_t)kn * sizeof(float), cudaMemcpyDeviceToHost, cs), "psf grad");
    if (gcorr)
        CUDA_TRY(cudaMemcpyAsync(b.data(), gcorr, (size_t)kn * sizeof(float), cudaMemcpyDeviceToHost, cs), "psf grad");
    CUDA_TRY(cudaStreamSynchronize(cs), "psf grad");
    std::vector<double> gn((size_t)kn);
    for (int64_t i = 0; i < kn; ++i) gn[(size_t)i] = (double)a[(size_t)i] + (gcorr ? (double)b[(size_t)i] : 0.0);
    std::vector<float> out((size_t)kn);
    if (normalised && su.norm_active) {
        double dot = 0.0;
        for (int64_t i = 0; i < kn; ++i) dot += gn[(size_t)i] * su.pn[(size_t)i];
        for (int64_t i = 0; i < kn; ++i) out[(size_t)i] = (float)(su.norm * (gn[(size_t)i] - dot));
    } else {
        for (int64_t i = 0; i < kn; ++i) out[(size_t)i] = (float)gn[(size_t)i];
    }
    CUDA_TRY(cudaMemcpyAsync(grad_psf->data, out.data(), (size_t)kn * sizeof(float), cudaMemcpyHostToDevice, cs),
             "psf grad upload");
    CUDA_TRY(cudaStreamSynchronize(cs), "psf grad upload");
    return ok();
}

}  // namespace

// An instantiated capture.
struct lucem_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// A planned batch: geometry, transfer functions, spectra and the launch
// groups, all owned by the plan (allocated once at creation).
struct lucem_rl_batch {
    int device = 0;
    std::vector<void *> mem;
    std::vector<RlBatchGroup> rows, cols;      // problems grouped by length
    std::vector<RlBatchGroup> rows1, cols1;    // one group per problem
    std::vector<int64_t> grids;                // (Py, Px) per problem
    int32_t num_iter = 0, clip = 0, mode = 0;
    float eps = 0.f;
    ~lucem_rl_batch() {
        for (void *p : mem) cudaFree(p);
    }
    void *alloc(size_t bytes, int *err) {
        void *p = nullptr;
        *err = (int)cudaMalloc(&p, bytes > 0 ? bytes : 16);
        if (*err) return nullptr;
        mem.push_back(p);
        return p;
    }
};

namespace {

// Uploads one group's items and records the group.
template <class Item>
lucem_status upload_group(lucem_rl_batch *b, int32_t n, std::vector<Item> &items, int tile_unit,
                          const float2_ *tw, std::vector<RlBatchGroup> *out) {
    int32_t t = 0;
    for (auto &it : items) {
        it.tile_begin = t;
        int32_t units = 0;
        if constexpr (std::is_same<Item, RlColItem>::value) units = it.ncols;
        else units = it.nrows;
        t += (units + tile_unit - 1) / tile_unit;
    }
    int err = 0;
    void *d = b->alloc(items.size() * sizeof(Item), &err);
    if (!d) return cuda_fail(err, "batch plan allocation");
    CUDA_TRY(cudaMemcpy(d, items.data(), items.size() * sizeof(Item), cudaMemcpyHostToDevice), "batch plan upload");
    out->push_back(RlBatchGroup{n, d, (int32_t)items.size(), t, tw});
    return ok();
}

}  // namespace

extern "C" {

lucem_status lucem_rl_grid(const int64_t *dims, const int64_t *kdims, int32_t ndim, int32_t mode,
                           const int64_t *requested, int64_t *grid_out) {
    if (!dims || !kdims || !grid_out) return fail(LUCEM_ERR_INVALID_PARAMETER, "null argument");
    if (ndim < 1 || ndim > 3) return fail(LUCEM_ERR_INVALID_DIMENSION, "richardson_lucy expects 2-D or 3-D");
    lucem_status st = check_mode(mode);
    if (st) return st;
    return rl_grid_impl(dims, kdims, ndim, mode, requested, grid_out);
}

int64_t lucem_fft_good_length(int64_t n, int32_t even) { return fft_good_length(n, even != 0); }

lucem_status lucem_richardson_lucy(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                   const lucem_rl_settings *settings, lucem_tensor *out,
                                   lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_rl_settings def;
    lucem_rl_settings_default(&def);
    const lucem_rl_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = rl_check(in, psf, out, s->num_iter, s->mode, "richardson_lucy"))) return st;
    if (numel(in) == 0) return ok();
    RlSetup su;
    if ((st = rl_prepare(ctx, in, psf, s->mode, s->grid, true, ws, stream, &su))) return st;
    int e = rl_launch_iterations(su.g, su.b, static_cast<const float *>(in->data), static_cast<float *>(out->data),
                                 s->num_iter, s->clip, rl_eps(s), stream, ws->t());
    return e ? cuda_fail(e, "richardson_lucy launch") : ok();
}

lucem_status lucem_richardson_lucy_backward(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                            const lucem_rl_settings *settings, const lucem_tensor *grad_out,
                                            int32_t checkpoint_every, lucem_tensor *grad_psf,
                                            lucem_tensor *grad_in, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_rl_settings def;
    lucem_rl_settings_default(&def);
    const lucem_rl_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = rl_check(in, psf, grad_out, s->num_iter, s->mode, "richardson_lucy_backward"))) return st;
    if (s->mode != LUCEM_PAD_CONSTANT || s->clip)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `settings`: the backward pass takes zero padding (mode constant) and clip off");
    if (checkpoint_every < 1)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `checkpoint_every`: must be >= 1");
    if (grad_psf) {
        if ((st = check_tensor("grad_psf", grad_psf)) || (st = same_shape("psf", psf, "grad_psf", grad_psf)) ||
            (st = require_f32_out(grad_psf)))
            return st;
    }
    if (grad_in) {
        if ((st = check_tensor("grad_in", grad_in)) || (st = same_shape("input", in, "grad_in", grad_in)) ||
            (st = require_f32_out(grad_in)) || (st = not_aliased(grad_out, grad_in)))
            return st;
    }
    if (numel(in) == 0) return ok();
    RlSetup su;
    if ((st = rl_prepare(ctx, in, psf, s->mode, s->grid, true, ws, stream, &su))) return st;
    RlBwdBuffers w;
    const int T = s->num_iter, K = checkpoint_every < T ? checkpoint_every : T;
    if ((st = rl_bwd_buffers(su, T, K, true, ws, &w))) return st;
    void *gp = nullptr;
    if ((st = ws->get("rlb_gpsf", (size_t)su.kn * 2 * sizeof(float), &gp))) return st;
    float *gconv = static_cast<float *>(gp), *gcorr = gconv + su.kn;
    int e = rl_backward(su.g, su.b, w, static_cast<const float *>(in->data), T, K, rl_eps(s),
                        static_cast<const float *>(grad_out->data), gconv, w.pbar2 ? gcorr : nullptr,
                        grad_in ? static_cast<float *>(grad_in->data) : nullptr, stream, ws->t());
    if (e) return cuda_fail(e, "richardson_lucy_backward launch");
    if (grad_psf) return psf_grad_finish(su, gconv, w.pbar2 ? gcorr : nullptr, true, grad_psf, stream);
    return ok();
}

lucem_status lucem_fft_convolve(lucem_ctx *ctx, const lucem_tensor *x, const lucem_tensor *psf, int32_t mode,
                                const int64_t *grid, lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_status st;
    if ((st = rl_check(x, psf, out, 1, mode, "fft_convolve"))) return st;
    if (mode != LUCEM_PAD_CONSTANT)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `mode`: fft_convolve takes zero padding");
    if (numel(x) == 0) return ok();
    int64_t req[3] = {0, 0, 0};
    if (grid)
        for (int d = 0; d < psf->ndim && d < 3; ++d) req[d] = grid[d];
    RlSetup su;
    if ((st = rl_prepare(ctx, x, psf, mode, req, false, ws, stream, &su))) return st;
    int e = rl_apply(su.g, su.b, su.b.h_conv, 0, static_cast<const float *>(x->data), static_cast<float *>(out->data),
                     stream, ws->t());
    return e ? cuda_fail(e, "fft_convolve launch") : ok();
}

lucem_status lucem_fft_convolve_backward(lucem_ctx *ctx, const lucem_tensor *x, const lucem_tensor *psf,
                                         int32_t mode, const int64_t *grid, const lucem_tensor *grad_out,
                                         lucem_tensor *grad_x, lucem_tensor *grad_psf, lucem_workspace *ws,
                                         void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_status st;
    if ((st = rl_check(x, psf, grad_out, 1, mode, "fft_convolve_backward"))) return st;
    if (mode != LUCEM_PAD_CONSTANT)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `mode`: fft_convolve takes zero padding");
    if (grad_x) {
        if ((st = check_tensor("grad_x", grad_x)) || (st = same_shape("input", x, "grad_x", grad_x)) ||
            (st = require_f32_out(grad_x)) || (st = not_aliased(grad_out, grad_x)))
            return st;
    }
    if (grad_psf) {
        if ((st = check_tensor("grad_psf", grad_psf)) || (st = same_shape("psf", psf, "grad_psf", grad_psf)) ||
            (st = require_f32_out(grad_psf)))
            return st;
    }
    if (numel(x) == 0) return ok();
    int64_t req[3] = {0, 0, 0};
    if (grid)
        for (int d = 0; d < psf->ndim && d < 3; ++d) req[d] = grid[d];
    RlSetup su;
    if ((st = rl_prepare(ctx, x, psf, mode, req, false, ws, stream, &su))) return st;
    RlBwdBuffers w;
    if ((st = rl_bwd_buffers(su, 1, 1, false, ws, &w))) return st;
    void *gp = nullptr;
    if (grad_psf && (st = ws->get("rlb_gpsf", (size_t)su.kn * 2 * sizeof(float), &gp))) return st;
    int e = rl_convolve_backward(su.g, su.b, w, static_cast<const float *>(x->data),
                                 static_cast<const float *>(grad_out->data),
                                 grad_x ? static_cast<float *>(grad_x->data) : nullptr,
                                 grad_psf ? static_cast<float *>(gp) : nullptr, stream, ws->t());
    if (e) return cuda_fail(e, "fft_convolve_backward launch");
    if (grad_psf) return psf_grad_finish(su, static_cast<float *>(gp), nullptr, false, grad_psf, stream);
    return ok();
}

lucem_status lucem_rl_batch_create(lucem_ctx *ctx, int32_t n, const lucem_tensor *obs, const lucem_tensor *psfs,
                                   const lucem_rl_settings *settings, lucem_tensor *outs, lucem_workspace *ws,
                                   void *stream, lucem_rl_batch **out) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (!out) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `out`: null");
    *out = nullptr;
    if (n < 1 || !obs || !psfs || !outs)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `n`: a batch needs at least one problem");
    lucem_rl_settings def;
    lucem_rl_settings_default(&def);
    const lucem_rl_settings *s = settings ? settings : &def;
    lucem_status st;
    for (int i = 0; i < n; ++i) {
        if ((st = rl_check(&obs[i], &psfs[i], &outs[i], s->num_iter, s->mode, "richardson_lucy_batch"))) return st;
        if (obs[i].ndim != 2)
            return fail(LUCEM_ERR_INVALID_DIMENSION, "richardson_lucy_batch takes 2-D problems, problem %d is %d-D",
                        i, obs[i].ndim);
        if (numel(&obs[i]) == 0)
            return fail(LUCEM_ERR_EMPTY_INPUT, "richardson_lucy_batch: problem %d is empty", i);
    }
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    std::unique_ptr<lucem_rl_batch> b(new lucem_rl_batch());
    b->device = ctx->device;
    b->num_iter = s->num_iter;
    b->clip = s->clip;
    b->mode = s->mode;
    b->eps = rl_eps(s);
    const int mode = s->mode;

    // PSFs to the host (one synchronisation for the batch), normalised in f64.
    std::vector<std::vector<float>> hp((size_t)n);
    for (int i = 0; i < n; ++i) {
        hp[(size_t)i].resize((size_t)numel(&psfs[i]));
        CUDA_TRY(cudaMemcpyAsync(hp[(size_t)i].data(), psfs[i].data, hp[(size_t)i].size() * sizeof(float),
                                 cudaMemcpyDeviceToHost, cs), "psf download");
    }
    CUDA_TRY(cudaStreamSynchronize(cs), "psf download");

    std::map<int64_t, std::vector<RlRowItem>> row_groups;
    std::map<int64_t, std::vector<RlColItem>> col_groups;
    std::map<int64_t, const float2_ *> tw32;
    std::vector<RlRowItem> rows_one;
    std::vector<RlColItem> cols_one;
    std::vector<int64_t> px_one, py_one;
    int err = 0;
    for (int i = 0; i < n; ++i) {
        const int64_t Y = obs[i].dims[0], X = obs[i].dims[1], ky = psfs[i].dims[0], kx = psfs[i].dims[1];
        const int64_t Py = batch_length(ctx, 0, rl_min_length(Y, ky, mode));
        const int64_t Px = batch_length(ctx, 1, rl_min_length(X, kx, mode));
        b->grids.push_back(Py);
        b->grids.push_back(Px);
        RlGeom g{};
        g.ndim = 2;
        g.Z = 1; g.Y = (int32_t)Y; g.X = (int32_t)X;
        g.Pz = 1; g.Py = (int32_t)Py; g.Px = (int32_t)Px;
        g.hz = 0; g.hy = (int32_t)rl_halo(ky, mode); g.hx = (int32_t)rl_halo(kx, mode);
        g.Hx = g.Px / 2 + 1;
        g.Hp = (g.Hx + 15) & ~15;
        g.mode = mode;
        const float2_ *t32[3];
        const double *t64[3];
        if ((st = twiddles(ctx, 1, &t32[0], &t64[0])) || (st = twiddles(ctx, Py, &t32[1], &t64[1])) ||
            (st = twiddles(ctx, Px, &t32[2], &t64[2])))
            return st;
        tw32[Py] = t32[1];
        tw32[Px] = t32[2];
        // Transfer functions (deconvolve.rs:77-88 normalisation; centres as
        // lucem_richardson_lucy).
        const std::vector<float> &h = hp[(size_t)i];
        double sum = 0.0;
        for (float v : h) sum += (double)v;
        const double norm = std::fabs(sum) > 1e-12 ? 1.0 / sum : 1.0;
        std::vector<double> pn(h.size());
        for (size_t j = 0; j < h.size(); ++j) pn[j] = (double)h[j] * norm;
        const int32_t kdi[3] = {1, (int32_t)ky, (int32_t)kx};
        const int32_t c_conv[3] = {0, (int32_t)(ky - 1 - ky / 2), (int32_t)(kx - 1 - kx / 2)};
        const int32_t c_corr[3] = {0, (int32_t)(ky / 2), (int32_t)(kx / 2)};
        const bool same = c_conv[1] == c_corr[1] && c_conv[2] == c_corr[2];
        const size_t hbytes = (size_t)Py * g.Hp * sizeof(float2_);
        void *h_conv = b->alloc(hbytes, &err);
        void *h_corr = same ? h_conv : b->alloc(hbytes, &err);
        void *s1 = b->alloc((size_t)Y * g.Hp * sizeof(float2_), &err);
        if (!h_conv || !h_corr || !s1) return cuda_fail(err, "batch plan allocation");
        void *psf64 = nullptr, *wa = nullptr, *wb = nullptr;
        if ((st = ws->get("rl_psf64", pn.size() * sizeof(double), &psf64)) ||
            (st = ws->get("rl_otf_a", (size_t)ky * g.Hp * 16, &wa)) ||
            (st = ws->get("rl_otf_b", (size_t)Py * g.Hp * 16, &wb)))
            return st;
        CUDA_TRY(cudaMemcpyAsync(psf64, pn.data(), pn.size() * sizeof(double), cudaMemcpyHostToDevice, cs),
                 "psf upload");
        int e = rl_launch_otf(g, static_cast<const double *>(psf64), kdi, c_conv, static_cast<double *>(wa),
                              static_cast<double *>(wb), h_conv, t64[2], t64[1], t64[0], stream);
        if (!e && !same)
            e = rl_launch_otf(g, static_cast<const double *>(psf64), kdi, c_corr, static_cast<double *>(wa),
                              static_cast<double *>(wb), h_corr, t64[2], t64[1], t64[0], stream);
        if (e) return cuda_fail(e, "transfer function launch");
        // The scratch and the host copy are reused by the next problem.
        CUDA_TRY(cudaStreamSynchronize(cs), "transfer function");

        RlRowItem r{};
        r.s1 = static_cast<float2_ *>(s1);
        r.obs = static_cast<const float *>(obs[i].data);
        r.est = static_cast<float *>(outs[i].data);
        r.nrows = (int32_t)Y;
        r.X = (int32_t)X;
        r.hx = g.hx;
        RlColItem c{};
        c.src = static_cast<const float2_ *>(s1);
        c.dst = static_cast<float2_ *>(s1);
        c.H = static_cast<const float2_ *>(h_conv);
        c.H2 = static_cast<const float2_ *>(h_corr);
        c.src_row = c.dst_row = c.h_row = g.Hp;
        c.ncols = g.Hx;
        c.Hx = g.Hx;
        c.n_img = (int32_t)Y;
        c.halo = g.hy;
        c.store_begin = g.hy;
        c.store_count = (int32_t)Y;
        row_groups[Px].push_back(r);
        col_groups[Py].push_back(c);
        rows_one.push_back(r);
        cols_one.push_back(c);
        px_one.push_back(Px);
        py_one.push_back(Py);
    }
    for (auto &kv : row_groups)
        if ((st = upload_group(b.get(), (int32_t)kv.first, kv.second, row_tile_rows((int)kv.first / 2),
                               tw32[kv.first], &b->rows)))
            return st;
    for (auto &kv : col_groups)
        if ((st = upload_group(b.get(), (int32_t)kv.first, kv.second, col_tile_width((int)kv.first),
                               tw32[kv.first], &b->cols)))
            return st;
    for (int i = 0; i < n; ++i) {
        std::vector<RlRowItem> r1{rows_one[(size_t)i]};
        std::vector<RlColItem> c1{cols_one[(size_t)i]};
        if ((st = upload_group(b.get(), (int32_t)px_one[(size_t)i], r1, row_tile_rows((int)px_one[(size_t)i] / 2),
                               tw32[px_one[(size_t)i]], &b->rows1)) ||
            (st = upload_group(b.get(), (int32_t)py_one[(size_t)i], c1, col_tile_width((int)py_one[(size_t)i]),
                               tw32[py_one[(size_t)i]], &b->cols1)))
            return st;
    }
    *out = b.release();
    return ok();
}

lucem_status lucem_rl_batch_run(lucem_rl_batch *b, int32_t per_problem, lucem_workspace *ws, void *stream) {
    if (!b) return fail(LUCEM_ERR_INVALID_HANDLE, "null batch plan");
    TimerScope timer_scope(ws);
    PassTimer *t = ws ? ws->t() : nullptr;
    if (!per_problem) {
        RlBatchLaunch L{b->mode, b->rows.data(), (int32_t)b->rows.size(), b->cols.data(), (int32_t)b->cols.size()};
        int e = rl_batch_iterations(L, b->num_iter, b->clip, b->eps, stream, t);
        return e ? cuda_fail(e, "richardson_lucy_batch launch") : ok();
    }
    for (size_t i = 0; i < b->rows1.size(); ++i) {
        RlBatchLaunch L{b->mode, &b->rows1[i], 1, &b->cols1[i], 1};
        int e = rl_batch_iterations(L, b->num_iter, b->clip, b->eps, stream, t);
        if (e) return cuda_fail(e, "richardson_lucy_batch launch");
    }
    return ok();
}

lucem_status lucem_rl_batch_info(const lucem_rl_batch *b, int64_t *grids, int32_t *n_row_launches,
                                 int32_t *n_col_launches) {
    if (!b) return fail(LUCEM_ERR_INVALID_HANDLE, "null batch plan");
    if (grids) std::copy(b->grids.begin(), b->grids.end(), grids);
    if (n_row_launches) *n_row_launches = (int32_t)b->rows.size();
    if (n_col_launches) *n_col_launches = (int32_t)b->cols.size();
    return ok();
}

void lucem_rl_batch_destroy(lucem_rl_batch *b) { delete b; }

lucem_status lucem_autotune_fft(lucem_ctx *ctx, const int64_t *lengths, int32_t n, lucem_workspace *ws,
                                void *stream) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (n < 0 || (n > 0 && !lengths)) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `lengths`");
    lucem_status st;
    const int64_t elems = (int64_t)1 << 24;
    for (int i = 0; i < n; ++i) {
        const int64_t L = lengths[i];
        if (L < 32 || L > 16384 || !good_factors(L))
            return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `lengths`: %lld does not factor into 2, 3, 5, 7",
                        (long long)L);
        const float2_ *t32;
        const double *t64;
        if ((st = twiddles(ctx, L, &t32, &t64))) return st;
        for (int kind = 0; kind < 2; ++kind) {
            if (kind == 1 && (L & 1)) continue;
            const int lines = (int)std::max<int64_t>(64, (elems / L) & ~(int64_t)15);
            void *a = nullptr, *bb = nullptr;
            const size_t abytes = (size_t)lines * (size_t)L * sizeof(float2_);
            if ((st = ws->get("tune_a", abytes, &a)) || (st = ws->get("tune_b", (size_t)lines * L * sizeof(float), &bb)))
                return st;
            CUDA_TRY(cudaMemsetAsync(a, 0, abytes, static_cast<cudaStream_t>(stream)), "tune buffers");
            CUDA_TRY(cudaMemsetAsync(bb, 0, (size_t)lines * L * sizeof(float), static_cast<cudaStream_t>(stream)),
                     "tune buffers");
            float ms = 0.f;
            int e = rl_tune_pass(kind, (int)L, lines, a, bb, t32, 3, stream, &ms);
            if (e) return cuda_fail(e, "autotune launch");
            // ns per transformed element, relative to nothing: the cost model
            // only compares lengths of one kind.
            const double per = (double)ms * 1e6 / ((double)lines * (double)L);
            std::lock_guard<std::mutex> lk(ctx->mu);
            ctx->tune[{kind, L}] = per;
        }
    }
    return ok();
}

lucem_status lucem_autotune_query(lucem_ctx *ctx, int32_t kind, int64_t length, double *ns_per_element) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ns_per_element) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `ns_per_element`: null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->tune.find({kind, length});
    if (it == ctx->tune.end()) {
        *ns_per_element = 0.0;
        return fail(LUCEM_ERR_INVALID_PARAMETER, "no autotune entry for kind %d length %lld", kind, (long long)length);
    }
    *ns_per_element = it->second;
    return ok();
}

lucem_status lucem_autotune_save(lucem_ctx *ctx, const char *path) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!path) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `path`: null");
    FILE *f = std::fopen(path, "w");
    if (!f) return fail(LUCEM_ERR_INVALID_PARAMETER, "cannot write %s", path);
    std::lock_guard<std::mutex> lk(ctx->mu);
    std::fprintf(f, "# lucem_b200 FFT pass costs: kind (0 column, 1 row) length ns_per_element\n");
    for (auto &kv : ctx->tune) std::fprintf(f, "%d %lld %.9g\n", kv.first.first, (long long)kv.first.second, kv.second);
    std::fprintf(f, "# family launch settings: plan key code\n");
    for (auto &kv : ctx->plans) std::fprintf(f, "plan %s %d\n", kv.first.c_str(), kv.second);
    std::fclose(f);
    return ok();
}

lucem_status lucem_autotune_load(lucem_ctx *ctx, const char *path) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!path) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `path`: null");
    FILE *f = std::fopen(path, "r");
    if (!f) return fail(LUCEM_ERR_INVALID_PARAMETER, "cannot read %s", path);
    char line[256];
    std::map<std::pair<int, int64_t>, double> got;
    std::map<std::string, int> plans;
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        if (std::strncmp(line, "plan ", 5) == 0) {
            char key[96];
            int code = 0;
            if (std::sscanf(line + 5, "%95s %d", key, &code) != 2 || code < 1 || code > 4) {
                std::fclose(f);
                return fail(LUCEM_ERR_INVALID_PARAMETER, "malformed autotune line in %s: %s", path, line);
            }
            plans[key] = code;
            continue;
        }
        int kind;
        long long len;
        double v;
        if (std::sscanf(line, "%d %lld %lf", &kind, &len, &v) != 3 || (kind != 0 && kind != 1) || len < 1 ||
            !(v > 0.0)) {
            std::fclose(f);
            return fail(LUCEM_ERR_INVALID_PARAMETER, "malformed autotune line in %s: %s", path, line);
        }
        got[{kind, (int64_t)len}] = v;
    }
    std::fclose(f);
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (auto &kv : got) ctx->tune[kv.first] = kv.second;
    for (auto &kv : plans) ctx->plans[kv.first] = kv.second;
    return ok();
}

lucem_status lucem_autotune_enable(lucem_ctx *ctx, int32_t enable) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->tune_on = enable != 0;
    return ok();
}

lucem_status lucem_autotune_plans(lucem_ctx *ctx, char *keys, int32_t *plans, int32_t cap, int32_t *n_out) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!n_out || cap < 0 || (cap > 0 && (!keys || !plans)))
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `keys`");
    std::lock_guard<std::mutex> lk(ctx->mu);
    int32_t i = 0;
    for (auto &kv : ctx->plans) {
        if (i < cap) {
            std::snprintf(keys + 64 * (size_t)i, 64, "%s", kv.first.c_str());
            plans[i] = kv.second;
        }
        ++i;
    }
    *n_out = i;
    return ok();
}

lucem_status lucem_graph_begin(void *stream) {
    if (!stream) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `stream`: the legacy default stream cannot be captured");
    CUDA_TRY(cudaStreamBeginCapture(static_cast<cudaStream_t>(stream), cudaStreamCaptureModeThreadLocal),
             "stream capture");
    return ok();
}

lucem_status lucem_graph_end(void *stream, lucem_graph **out) {
    if (!out) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `out`: null");
    *out = nullptr;
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamEndCapture(static_cast<cudaStream_t>(stream), &g), "stream capture");
    cudaGraphExec_t x = nullptr;
    cudaError_t e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail((int)e, "graph instantiation");
    }
    auto *h = new lucem_graph();
    h->graph = g;
    h->exec = x;
    *out = h;
    return ok();
}

lucem_status lucem_graph_launch(lucem_graph *graph, void *stream) {
    if (!graph) return fail(LUCEM_ERR_INVALID_HANDLE, "null graph");
    CUDA_TRY(cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream)), "graph launch");
    return ok();
}

void lucem_graph_destroy(lucem_graph *graph) {
    if (!graph) return;
    cudaGraphExecDestroy(graph->exec);
    cudaGraphDestroy(graph->graph);
    delete graph;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The general complex FFT (crates/lucem-ops/src/core/fft.rs:14-100) and the
// spectral operators on it.

namespace {

using cd = std::complex<double>;

// Forward DFT of a 2,3,5,7-smooth length in FP64 (recursive decimation in
// time on the smallest factor; host tables only).
void host_fft64(std::vector<cd> &a) {
    const size_t n = a.size();
    if (n <= 1) return;
    size_t p = 0;
    for (size_t f : {2, 3, 5, 7})
        if (n % f == 0) {
            p = f;
            break;
        }
    const size_t m = n / p;
    std::vector<std::vector<cd>> sub(p, std::vector<cd>(m));
    for (size_t r = 0; r < p; ++r)
        for (size_t j = 0; j < m; ++j) sub[r][j] = a[j * p + r];
    for (auto &v : sub) host_fft64(v);
    for (size_t k = 0; k < n; ++k) {
        cd acc = 0.0;
        for (size_t r = 0; r < p; ++r) {
            const size_t q = (r * k) % n;
            const double ang = -2.0 * M_PI * (double)q / (double)n;
            acc += sub[r][k % m] * cd(std::cos(ang), std::sin(ang));
        }
        a[k] = acc;
    }
}

// Bluestein tables of length len on a smooth M >= 2 len - 1 (device, cached
// in the context): the chirp c[k] = e^{-i pi k^2 / len} (exact phase
// k^2 mod 2 len) and the spectrum of the conjugate chirp filter divided by M.
lucem_status bluestein_tables(lucem_ctx *ctx, int64_t len, int64_t M, const float2_ **chirp, const float2_ **filt) {
    std::string kc = "bluestein-chirp-" + std::to_string(len);
    std::string kf = "bluestein-filter-" + std::to_string(len) + "-" + std::to_string(M);
    std::vector<float> c((size_t)(2 * len));
    std::vector<cd> b((size_t)M, cd(0.0, 0.0));
    for (int64_t k = 0; k < len; ++k) {
        const int64_t q = (k * k) % (2 * len);
        const double ang = M_PI * (double)q / (double)len;
        c[(size_t)(2 * k)] = (float)std::cos(ang);
        c[(size_t)(2 * k + 1)] = (float)-std::sin(ang);
        const cd conjc(std::cos(ang), std::sin(ang));
        b[(size_t)k] = conjc;
        if (k > 0) b[(size_t)(M - k)] = conjc;
    }
    int err = 0;
    void *pc = ctx->get_or_upload(kc, c.data(), c.size() * sizeof(float), &err);
    if (!pc) return cuda_fail(err, "chirp upload");
    void *pf = nullptr;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->cache.find(kf);
        if (it != ctx->cache.end()) pf = it->second;
    }
    if (!pf) {
        host_fft64(b);
        std::vector<float> f((size_t)(2 * M));
        for (int64_t k = 0; k < M; ++k) {
            f[(size_t)(2 * k)] = (float)(b[(size_t)k].real() / (double)M);
            f[(size_t)(2 * k + 1)] = (float)(b[(size_t)k].imag() / (double)M);
        }
        pf = ctx->get_or_upload(kf, f.data(), f.size() * sizeof(float), &err);
        if (!pf) return cuda_fail(err, "chirp filter upload");
    }
    *chirp = static_cast<const float2_ *>(pc);
    *filt = static_cast<const float2_ *>(pf);
    return ok();
}

// One side of an axis pass: split (re, im) or interleaved (c).
struct FftSide {
    const float *re = nullptr;
    const float *im = nullptr;
    float2_ *c = nullptr;
    float *wre = nullptr, *wim = nullptr;  // destination split
};

// Largest smooth divisor n1 <= kFftLinesMax of n with n / n1 <= kFftLinesMax.
int64_t four_step_split(int64_t n) {
    int64_t best = 0;
    for (int64_t d = 1; d * d <= n; ++d) {
        if (n % d) continue;
        for (int64_t n1 : {d, n / d}) {
            const int64_t n2 = n / n1;
            FftPlan a, b;
            if (n1 <= kFftLinesMax && n2 <= kFftLinesMax && fft_make_plan(n1, &a) && fft_make_plan(n2, &b))
                if (best == 0 || std::llabs(n1 - n2) < std::llabs(best - n / best)) best = n1;
        }
    }
    return best;
}

// The transform along one axis of an [outer, len, inner] array: src -> dst,
// inverse scaled by 1 / len as the reference's dft_axis_kernel
// (crates/lucem-ops/src/core/kernels/fft.rs:41-43).  `scratch` (outer * len *
// inner complex) is needed for smooth lengths above kFftLinesMax.
lucem_status fft_axis(lucem_ctx *ctx, const FftSide &src, const FftSide &dst, int64_t outer, int64_t len,
                      int64_t inner, bool inverse, int clip, float2_ *scratch, void *stream) {
    FftLines p{};
    p.sre = src.re;
    p.sim = src.im;
    p.sc = src.c;
    p.dre = dst.wre;
    p.dim = dst.wim;
    p.dc = dst.c;
    p.n_outer = outer;
    p.inner = inner;
    p.s_os_hi = p.d_os_hi = len * inner;
    p.s_rs = p.d_rs = inner;
    p.scale = inverse ? (float)(1.0 / (double)len) : 1.0f;
    p.clip = clip;
    lucem_status st;
    const float2_ *tw32 = nullptr;
    const double *tw64 = nullptr;
    FftPlan plan;
    const bool smooth = fft_make_plan(len, &plan);
    if (smooth && len <= kFftLinesMax) {
        if ((st = twiddles(ctx, len, &tw32, &tw64))) return st;
        p.n = (int32_t)len;
        p.src_rows = p.dst_rows = (int32_t)len;
        p.inverse = inverse;
        p.plan = plan;
        p.tw = tw32;
        int e = timed(kPassFft, stream, [&] { return launch_fft_lines(p, stream); });
        return e ? cuda_fail(e, "fft launch") : ok();
    }
    if (smooth) {
        // Four-step: n = n1 n2, element m1 n2 + m2 -> X[k1 + n1 k2].
        const int64_t n1 = four_step_split(len), n2 = n1 ? len / n1 : 0;
        if (!n1 || !scratch) return fail(LUCEM_ERR_INVALID_PARAMETER, "fft: no four-step split for length %lld",
                                        (long long)len);
        const float2_ *tw_n = nullptr, *tw_1 = nullptr, *tw_2 = nullptr;
        if ((st = twiddles(ctx, len, &tw_n, &tw64)) || (st = twiddles(ctx, n1, &tw_1, &tw64)) ||
            (st = twiddles(ctx, n2, &tw_2, &tw64)))
            return st;
        FftLines a = p;
        a.dre = a.dim = nullptr;
        a.dc = scratch;
        a.inner = n2 * inner;
        a.s_rs = a.d_rs = n2 * inner;
        a.n = (int32_t)n1;
        a.src_rows = a.dst_rows = (int32_t)n1;
        a.inverse = inverse;
        fft_make_plan(n1, &a.plan);
        a.tw = tw_1;
        a.twiddle_n = (int32_t)len;
        a.tw_big = tw_n;
        a.tw_div = inner;
        a.scale = 1.0f;
        a.clip = 0;
        int e = timed(kPassFft, stream, [&] { return launch_fft_lines(a, stream); });
        if (e) return cuda_fail(e, "fft launch");
        FftLines b = p;
        b.sre = b.sim = nullptr;
        b.sc = scratch;
        b.n_outer = outer * n1;
        b.inner = inner;
        b.s_os_hi = n2 * inner;
        b.s_rs = inner;
        b.d_odiv = (int32_t)n1;
        b.d_os_hi = len * inner;
        b.d_os_lo = inner;
        b.d_rs = n1 * inner;
        b.n = (int32_t)n2;
        b.src_rows = b.dst_rows = (int32_t)n2;
        b.inverse = inverse;
        fft_make_plan(n2, &b.plan);
        b.tw = tw_2;
        e = timed(kPassFft, stream, [&] { return launch_fft_lines(b, stream); });
        return e ? cuda_fail(e, "fft launch") : ok();
    }
    const int64_t M = fft_good_length(2 * len - 1, false);
    if (M <= kFftLinesMax) {
        // Bluestein: X = c (.) ((x c) (*) conj(c)), the circular convolution on
        // M points; the inverse transform through conjugation.
        const float2_ *chirp = nullptr, *filt = nullptr;
        if ((st = bluestein_tables(ctx, len, M, &chirp, &filt))) return st;
        if ((st = twiddles(ctx, M, &tw32, &tw64))) return st;
        p.n = (int32_t)M;
        p.src_rows = p.dst_rows = (int32_t)len;
        p.inverse = 0;
        fft_make_plan(M, &p.plan);
        p.tw = tw32;
        p.pre = chirp;
        p.mid = filt;
        p.post = chirp;
        p.conj_in = p.conj_out = inverse;
        int e = timed(kPassFft, stream, [&] { return launch_fft_lines(p, stream); });
        return e ? cuda_fail(e, "fft launch") : ok();
    }
    // Longer lengths without a smooth factorisation: the direct DFT.
    if ((st = twiddles(ctx, len, &tw32, &tw64))) return st;
    p.n = (int32_t)len;
    p.src_rows = p.dst_rows = (int32_t)len;
    p.inverse = inverse;
    p.tw = tw32;
    int e = timed(kPassFft, stream, [&] { return launch_dft_direct(p, stream); });
    return e ? cuda_fail(e, "dft launch") : ok();
}

// N-D transform across all axes in order (fft_nd_into, core/fft.rs:55-100):
// axis 0 src -> ping, the middle axes between ping and pong, the last one
// into dst.  dims: the array's shape.
lucem_status fft_nd(lucem_ctx *ctx, const int64_t *dims, int nd, const FftSide &src, const FftSide &dst,
                    bool inverse, int clip, lucem_workspace *ws, void *stream) {
    int64_t n = 1;
    for (int d = 0; d < nd; ++d) n *= dims[d];
    bool four = false;
    for (int d = 0; d < nd; ++d) {
        FftPlan pl;
        four = four || (dims[d] > kFftLinesMax && fft_make_plan(dims[d], &pl));
    }
    lucem_status st;
    void *scr = nullptr, *ping = nullptr, *pong = nullptr;
    if (four && (st = ws->get("fft_four_step", (size_t)n * sizeof(float2_), &scr))) return st;
    if (nd >= 2 && (st = ws->get("fft_ping", (size_t)n * sizeof(float2_), &ping))) return st;
    if (nd >= 3 && (st = ws->get("fft_pong", (size_t)n * sizeof(float2_), &pong))) return st;
    float2_ *scratch = static_cast<float2_ *>(scr);
    FftSide cur = src;
    float2_ *bufs[2] = {static_cast<float2_ *>(ping), static_cast<float2_ *>(pong)};
    int which = 0;
    for (int d = 0; d < nd; ++d) {
        int64_t outer = 1, inner = 1;
        for (int i = 0; i < d; ++i) outer *= dims[i];
        for (int i = d + 1; i < nd; ++i) inner *= dims[i];
        FftSide out;
        const bool last = d + 1 == nd;
        if (last) {
            out = dst;
        } else {
            out.c = bufs[which];
        }
        if ((st = fft_axis(ctx, cur, out, outer, dims[d], inner, inverse, last ? clip : 0, scratch, stream)))
            return st;
        if (!last) {
            cur = FftSide{};
            cur.c = bufs[which];
            which ^= 1;
        }
    }
    return ok();
}

lucem_status fft_check(const lucem_tensor *re_in, const lucem_tensor *im_in, const lucem_tensor *re_out,
                       const lucem_tensor *im_out) {
    lucem_status st;
    if ((st = check_tensor("re_in", re_in)) || (st = check_tensor("im_in", im_in)) ||
        (st = check_tensor("re_out", re_out)) || (st = check_tensor("im_out", im_out)))
        return st;
    if ((st = same_shape("re_in", re_in, "im_in", im_in)) || (st = same_shape("re_in", re_in, "re_out", re_out)) ||
        (st = same_shape("re_in", re_in, "im_out", im_out)))
        return st;
    if ((st = not_aliased(re_in, re_out)) || (st = not_aliased(im_in, im_out))) return st;
    for (const lucem_tensor *t : {re_in, im_in, re_out, im_out})
        if (t->dtype != LUCEM_F32) return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "fft takes f32 arrays");
    return ok();
}

}  // namespace

extern "C" {

lucem_status lucem_fft_nd(lucem_ctx *ctx, const lucem_tensor *re_in, const lucem_tensor *im_in,
                          lucem_tensor *re_out, lucem_tensor *im_out, int32_t inverse, lucem_workspace *ws,
                          void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_status st;
    if ((st = fft_check(re_in, im_in, re_out, im_out))) return st;
    const int64_t n = numel(re_in);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if (re_in->ndim == 0 || n == 0) {
        // fft.rs:69-72: copies.
        if (n > 0) {
            CUDA_TRY(cudaMemcpyAsync(re_out->data, re_in->data, (size_t)n * 4, cudaMemcpyDeviceToDevice, cs), "copy");
            CUDA_TRY(cudaMemcpyAsync(im_out->data, im_in->data, (size_t)n * 4, cudaMemcpyDeviceToDevice, cs), "copy");
        }
        return ok();
    }
    FftSide src, dst;
    src.re = static_cast<const float *>(re_in->data);
    src.im = static_cast<const float *>(im_in->data);
    dst.wre = static_cast<float *>(re_out->data);
    dst.wim = static_cast<float *>(im_out->data);
    return fft_nd(ctx, re_in->dims, re_in->ndim, src, dst, inverse != 0, 0, ws, stream);
}

lucem_status lucem_fft_1d(lucem_ctx *ctx, const lucem_tensor *re_in, const lucem_tensor *im_in,
                          lucem_tensor *re_out, lucem_tensor *im_out, int32_t axis, int32_t inverse,
                          lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = fft_check(re_in, im_in, re_out, im_out))) return st;
    const int nd = re_in->ndim;
    const int ax = axis < 0 ? axis + nd : axis;
    if (nd == 0 || ax < 0 || ax >= nd)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "axis %d is out of range for a %d-D array", (int)axis, nd);
    if (numel(re_in) == 0) return ok();
    int64_t outer = 1, inner = 1;
    for (int i = 0; i < ax; ++i) outer *= re_in->dims[i];
    for (int i = ax + 1; i < nd; ++i) inner *= re_in->dims[i];
    const int64_t len = re_in->dims[ax];
    void *scr = nullptr;
    FftPlan pl;
    if (len > kFftLinesMax && fft_make_plan(len, &pl)) {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required for lengths above %d", kFftLinesMax);
        if ((st = ws->get("fft_four_step", (size_t)numel(re_in) * sizeof(float2_), &scr))) return st;
    }
    FftSide src, dst;
    src.re = static_cast<const float *>(re_in->data);
    src.im = static_cast<const float *>(im_in->data);
    dst.wre = static_cast<float *>(re_out->data);
    dst.wim = static_cast<float *>(im_out->data);
    return fft_axis(ctx, src, dst, outer, len, inner, inverse != 0, 0, static_cast<float2_ *>(scr), stream);
}

lucem_status lucem_complex_mul(const lucem_tensor *a_re, const lucem_tensor *a_im, const lucem_tensor *b_re,
                               const lucem_tensor *b_im, lucem_tensor *out_re, lucem_tensor *out_im, int32_t conj_b,
                               void *stream) {
    lucem_status st;
    if ((st = check_tensor("a_re", a_re)) || (st = check_tensor("a_im", a_im)) || (st = check_tensor("b_re", b_re)) ||
        (st = check_tensor("b_im", b_im)) || (st = check_tensor("out_re", out_re)) ||
        (st = check_tensor("out_im", out_im)))
        return st;
    if ((st = same_shape("a_re", a_re, "b_re", b_re)) || (st = same_shape("a_re", a_re, "out_re", out_re)) ||
        (st = same_shape("a_re", a_re, "a_im", a_im)) || (st = same_shape("a_re", a_re, "b_im", b_im)) ||
        (st = same_shape("a_re", a_re, "out_im", out_im)))
        return st;
    for (const lucem_tensor *t : {a_re, a_im, b_re, b_im, (const lucem_tensor *)out_re, (const lucem_tensor *)out_im})
        if (t->dtype != LUCEM_F32) return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "complex_mul takes f32 arrays");
    const int64_t n = numel(a_re);
    if (n == 0) return ok();
    int e = launch_complex_mul(static_cast<const float *>(a_re->data), static_cast<const float *>(a_im->data),
                               static_cast<const float *>(b_re->data), static_cast<const float *>(b_im->data),
                               static_cast<float *>(out_re->data), static_cast<float *>(out_im->data), n, conj_b,
                               stream);
    return e ? cuda_fail(e, "complex_mul launch") : ok();
}

void lucem_wiener_settings_default(lucem_wiener_settings *s) {
    s->balance = 0.1;
    s->clip = 1;
}

lucem_status lucem_wiener_deconvolve(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                     const lucem_wiener_settings *settings, lucem_tensor *out, lucem_workspace *ws,
                                     void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_wiener_settings def;
    lucem_wiener_settings_default(&def);
    const lucem_wiener_settings *s = settings ? settings : &def;
    lucem_status st;
    // restore/deconvolve.rs:218-244, same order.
    if ((st = check_tensor("input", in)) || (st = check_tensor("output", out)) || (st = check_tensor("psf", psf)))
        return st;
    if ((st = same_shape("input", in, "output", out)) || (st = not_aliased(in, out))) return st;
    if (in->ndim != 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "wiener_deconvolve input expects 2-D array, got %d-D shape %s",
                    in->ndim, dims_str(in).c_str());
    if (psf->ndim != 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "wiener_deconvolve psf expects 2-D array, got %d-D shape %s",
                    psf->ndim, dims_str(psf).c_str());
    if (numel(psf) == 0) return fail(LUCEM_ERR_INVALID_WEIGHTS, "psf: PSF cannot be empty");
    if (!std::isfinite(s->balance) || s->balance < 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `balance`: balance must be non-negative and finite, got %g", s->balance);
    if (in->dtype != LUCEM_F32 || psf->dtype != LUCEM_F32 || out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "wiener_deconvolve takes f32 input, psf and output");
    if (numel(in) == 0) return ok();
    const int64_t H = in->dims[0], W = in->dims[1];
    if (psf->dims[0] > H || psf->dims[1] > W)
        return fail(LUCEM_ERR_INVALID_WEIGHTS, "psf: PSF dimensions must not exceed image dimensions");
    const int64_t n = H * W;
    void *bufs[4] = {};
    const char *names[4] = {"wiener_y", "wiener_h", "wiener_l", "wiener_x"};
    for (int i = 0; i < 4; ++i)
        if ((st = ws->get(names[i], (size_t)n * sizeof(float2_), &bufs[i]))) return st;
    float2_ *Y = static_cast<float2_ *>(bufs[0]), *Hk = static_cast<float2_ *>(bufs[1]);
    float2_ *Lk = static_cast<float2_ *>(bufs[2]), *X = static_cast<float2_ *>(bufs[3]);
    // Y = FFT(input).
    FftSide src, dst;
    src.re = static_cast<const float *>(in->data);
    dst.c = Y;
    if ((st = fft_nd(ctx, in->dims, 2, src, dst, false, 0, ws, stream))) return st;
    // H = FFT of the PSF centred at (kh/2, kw/2); X stages it.
    auto centred_fft = [&](const float *k, int kh, int kw, float2_ *dst_c) -> lucem_status {
        int e = launch_centre_kernel(k, kh, kw, X, (int)H, (int)W, stream);
        if (e) return cuda_fail(e, "kernel centring");
        FftSide a, b;
        a.c = X;
        b.c = dst_c;
        return fft_nd(ctx, in->dims, 2, a, b, false, 0, ws, stream);
    };
    if ((st = centred_fft(static_cast<const float *>(psf->data), (int)psf->dims[0], (int)psf->dims[1], Hk))) return st;
    // The discrete Laplacian [0 -1 0; -1 4 -1; 0 -1 0] (a 1 x 1 one below
    // 3 x 3 images), as deconvolve.rs:250-262.
    const bool lap3 = H >= 3 && W >= 3;
    const float lap[9] = {0, -1, 0, -1, 4, -1, 0, -1, 0}, one = 1.0f;
    int err = 0;
    void *lapd = ctx->get_or_upload(lap3 ? "wiener-laplacian-3x3" : "wiener-laplacian-1x1", lap3 ? lap : &one,
                                    lap3 ? sizeof lap : sizeof one, &err);
    if (!lapd) return cuda_fail(err, "laplacian upload");
    if ((st = centred_fft(static_cast<const float *>(lapd), lap3 ? 3 : 1, lap3 ? 3 : 1, Lk))) return st;
    int e = timed(kPassElementwise, stream, [&] {
        return launch_wiener_filter(Y, Hk, Lk, X, n, (float)s->balance, 1.0e-12f, stream);
    });
    if (e) return cuda_fail(e, "wiener filter launch");
    // out = Re(IFFT(X)), clipped to [-1, 1] when asked (deconvolve.rs:285-292).
    FftSide xs, os;
    xs.c = X;
    os.wre = static_cast<float *>(out->data);
    return fft_nd(ctx, in->dims, 2, xs, os, true, s->clip ? 1 : 0, ws, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Spectral filters, Butterworth, phase correlation and unsupervised Wiener
// (kernels in spectral_ops.cu).

namespace {

// Bins of a C-contiguous array (< 2^32 elements, checked by the caller).
SpecAxes spec_axes(const lucem_tensor *t) {
    SpecAxes a{};
    a.ndim = t->ndim;
    uint32_t inner = 1;
    for (int d = t->ndim - 1; d >= 0; --d) {
        a.len[d] = (uint32_t)t->dims[d];
        a.inner[d] = inner;
        inner *= (uint32_t)t->dims[d];
    }
    return a;
}

// The signed normalised frequency of bin k on an n-point axis, as the
// reference's host tables (filter/spectral.rs:38-41).
double bin_freq(int64_t k, int64_t n) {
    return k <= n / 2 ? (double)k / (double)n : (double)(k - n) / (double)n;
}

enum class SpecKind { kGaussian, kBox, kShift };

// fourier_{gaussian,box,shift}_into (filter/spectral.rs:21-164): per axis a
// table of the transfer function (FP64 on the host, cast to f32 as
// cast_all), all axes applied in one pass (spectral_axes_kernel).
lucem_status spectral_filter(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *vals, int32_t n_vals,
                             SpecKind kind, const char *name, void *stream) {
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_tensor("re", re)) || (st = check_tensor("im", im))) return st;
    if ((st = same_shape("re", re, "im", im))) return st;
    if (re->dtype != LUCEM_F32 || im->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "spectral filters take f32 arrays");
    if ((st = not_aliased(re, im))) return st;
    const int nd = re->ndim;
    if (n_vals > 0 && !vals) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `%s`: null values", name);
    std::vector<double> per;
    if ((st = broadcast(name, vals, n_vals, nd, &per))) return st;
    const int64_t n = numel(re);
    if (n == 0 || nd == 0) return ok();
    SpecAxes a = spec_axes(re);
    a.phase = kind == SpecKind::kShift ? 1 : 0;
    std::vector<float> tab;
    char buf[64];
    std::string key = kind == SpecKind::kGaussian ? "fgauss" : kind == SpecKind::kBox ? "fbox" : "fshift";
    for (int d = 0; d < nd; ++d) {
        const int64_t len = re->dims[d];
        const double v = per[(size_t)d];
        snprintf(buf, sizeof buf, "-%lld:%.17g", (long long)len, v);
        key += buf;
        a.off[d] = (uint32_t)tab.size();
        std::vector<float> c((size_t)len), sn;
        if (kind == SpecKind::kShift) sn.resize((size_t)len);
        for (int64_t k = 0; k < len; ++k) {
            const double f = bin_freq(k, len);
            if (kind == SpecKind::kGaussian) {
                c[(size_t)k] = (float)std::exp(-2.0 * M_PI * M_PI * v * v * f * f);
            } else if (kind == SpecKind::kBox) {
                const double x = M_PI * v * f;
                c[(size_t)k] = (float)(std::fabs(x) < 1e-12 ? 1.0 : std::sin(x) / x);
            } else {
                c[(size_t)k] = (float)std::cos(-2.0 * M_PI * v * f);
                sn[(size_t)k] = (float)std::sin(-2.0 * M_PI * v * f);
            }
        }
        tab.insert(tab.end(), c.begin(), c.end());
        tab.insert(tab.end(), sn.begin(), sn.end());
    }
    int err = 0;
    void *dtab = ctx->get_or_upload(key, tab.data(), tab.size() * sizeof(float), &err);
    if (!dtab) return cuda_fail(err, "spectral table upload");
    int e = launch_spectral_axes(static_cast<float *>(re->data), static_cast<float *>(im->data), n,
                                 static_cast<const float *>(dtab), a, stream);
    return e ? cuda_fail(e, "spectral filter launch") : ok();
}

}  // namespace

extern "C" {

lucem_status lucem_fourier_gaussian(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *sigmas,
                                    int32_t n_sigmas, void *stream) {
    return spectral_filter(ctx, re, im, sigmas, n_sigmas, SpecKind::kGaussian, "sigmas", stream);
}

lucem_status lucem_fourier_box(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *sizes,
                               int32_t n_sizes, void *stream) {
    return spectral_filter(ctx, re, im, sizes, n_sizes, SpecKind::kBox, "sizes", stream);
}

lucem_status lucem_fourier_shift(lucem_ctx *ctx, lucem_tensor *re, lucem_tensor *im, const double *shifts,
                                 int32_t n_shifts, void *stream) {
    return spectral_filter(ctx, re, im, shifts, n_shifts, SpecKind::kShift, "shifts", stream);
}

// filter/spectral.rs:168-213.
lucem_status lucem_butterworth(lucem_ctx *ctx, const lucem_tensor *in, double cutoff_ratio, int32_t high_pass,
                               double order, lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (!(cutoff_ratio > 0.0 && cutoff_ratio <= 0.5))
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `cutoff_ratio`: cutoff_ratio must be in (0.0, 0.5], got %g", cutoff_ratio);
    lucem_status st;
    if ((st = check_tensor("input", in)) || (st = check_tensor("output", out))) return st;
    if ((st = same_shape("input", in, "output", out)) || (st = not_aliased(in, out))) return st;
    if (in->dtype != LUCEM_F32 || out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "butterworth takes f32 input and output");
    const int64_t n = numel(in);
    if (n == 0) return ok();
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    if (in->ndim == 0) {
        // fft_nd of a 0-D array copies; w = 1 / (1 + 0) (low pass) or 0.
        if (high_pass) CUDA_TRY(cudaMemsetAsync(out->data, 0, 4, cs), "fill");
        else CUDA_TRY(cudaMemcpyAsync(out->data, in->data, 4, cudaMemcpyDeviceToDevice, cs), "copy");
        return ok();
    }
    void *xb = nullptr;
    if ((st = ws->get("bw_spectrum", (size_t)n * sizeof(float2_), &xb))) return st;
    float2_ *X = static_cast<float2_ *>(xb);
    FftSide src, dst;
    src.re = static_cast<const float *>(in->data);
    dst.c = X;
    if ((st = fft_nd(ctx, in->dims, in->ndim, src, dst, false, 0, ws, stream))) return st;
    int e = timed(kPassElementwise, stream,
                  [&] { return launch_butterworth(X, n, spec_axes(in), cutoff_ratio, order, high_pass ? 1 : 0, stream); });
    if (e) return cuda_fail(e, "butterworth launch");
    FftSide xs, os;
    xs.c = X;
    os.wre = static_cast<float *>(out->data);
    return fft_nd(ctx, in->dims, in->ndim, xs, os, true, 0, ws, stream);
}

void lucem_phase_correlation_settings_default(lucem_phase_correlation_settings *s) {
    s->upsample_factor = 1;
    s->normalize_phase = 1;
}

// register/phase.rs:51-255.
lucem_status lucem_phase_correlation(lucem_ctx *ctx, const lucem_tensor *reference, const lucem_tensor *moving,
                                     const lucem_phase_correlation_settings *settings,
                                     lucem_phase_correlation_result *result, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (!result) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `result`: null");
    lucem_phase_correlation_settings def;
    lucem_phase_correlation_settings_default(&def);
    const lucem_phase_correlation_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_tensor("reference", reference)) || (st = check_tensor("moving", moving))) return st;
    if ((st = same_shape("reference", reference, "moving", moving))) return st;
    if (reference->dtype != LUCEM_F32 || moving->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "phase_correlation takes f32 images");
    const int64_t n = numel(reference);
    if (n == 0) return fail(LUCEM_ERR_EMPTY_INPUT, "phase_correlation: empty input");
    if (s->upsample_factor < 1)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `upsample_factor`: upsample_factor must be >= 1");
    // A 0-D array is one sample: the same as a 1-D array of length 1.
    lucem_tensor view = *reference;
    if (view.ndim == 0) {
        view.ndim = 1;
        view.dims[0] = 1;
    }
    const int nd = view.ndim;
    const double u = (double)s->upsample_factor;
    const int half_span = (int)std::ceil(1.5 * u);
    const int max_cand = 2 * (half_span > 2 ? half_span : 2) + 1;
    int64_t max_len = 1;
    for (int d = 0; d < nd; ++d) max_len = std::max(max_len, view.dims[d]);
    const size_t cbytes = (size_t)n * sizeof(float2_);
    void *pa = nullptr, *pb = nullptr, *pr = nullptr, *pc = nullptr, *po = nullptr, *pt = nullptr, *pp = nullptr,
         *pv = nullptr, *pi = nullptr, *ps = nullptr;
    const size_t part_bytes = std::max((size_t)max_cand * kCandBlocks * sizeof(double2), (size_t)4 * kRedBlocks * sizeof(double));
    if ((st = ws->get("pc_a", cbytes, &pa)) || (st = ws->get("pc_b", cbytes, &pb)) ||
        (st = ws->get("pc_r", cbytes, &pr)) || (st = ws->get("pc_cc", cbytes, &pc)) ||
        (st = ws->get("pc_part", part_bytes, &pp)) || (st = ws->get("pc_pv", kRedBlocks * sizeof(float), &pv)) ||
        (st = ws->get("pc_pi", kRedBlocks * sizeof(uint32_t), &pi)) ||
        (st = ws->get("pc_state", sizeof(PcState) + 4 * sizeof(double), &ps)))
        return st;
    if (s->upsample_factor > 1 &&
        ((st = ws->get("pc_other", (size_t)n * sizeof(double2), &po)) ||
         (st = ws->get("pc_axis", (size_t)max_cand * (size_t)max_len * sizeof(double2), &pt))))
        return st;
    float2_ *A = static_cast<float2_ *>(pa), *B = static_cast<float2_ *>(pb);
    float2_ *R = static_cast<float2_ *>(pr), *CC = static_cast<float2_ *>(pc);
    PcState *dst_state = static_cast<PcState *>(ps);
    double *dsums = reinterpret_cast<double *>(static_cast<char *>(ps) + sizeof(PcState));
    const SpecAxes axes = spec_axes(&view);
    // F_ref, F_mov (phase.rs:81-82), R (:85-102), cc = IFFT(R) (:104-106).
    FftSide src, dst;
    src.re = static_cast<const float *>(reference->data);
    dst.c = A;
    if ((st = fft_nd(ctx, view.dims, nd, src, dst, false, 0, ws, stream))) return st;
    src.re = static_cast<const float *>(moving->data);
    dst.c = B;
    if ((st = fft_nd(ctx, view.dims, nd, src, dst, false, 0, ws, stream))) return st;
    int e = timed(kPassElementwise, stream,
                  [&] { return launch_phase_cross_power(A, B, R, n, s->normalize_phase ? 1 : 0, stream); });
    if (e) return cuda_fail(e, "cross-power spectrum launch");
    FftSide rs, cs;
    rs.c = R;
    cs.c = CC;
    if ((st = fft_nd(ctx, view.dims, nd, rs, cs, true, 0, ws, stream))) return st;
    // Integer peak (:108-131).
    e = timed(kPassElementwise, stream, [&] {
        return launch_phase_argmax(CC, n, axes, static_cast<float *>(pv), static_cast<uint32_t *>(pi), dst_state,
                                   stream);
    });
    if (e) return cuda_fail(e, "argmax launch");
    // Subpixel refinement (:134-227): two passes, coordinate-wise.
    if (s->upsample_factor > 1) {
        for (int pass = 0; pass < 2; ++pass) {
            const int radius = pass == 0 ? half_span : 2;
            const double step = pass == 0 ? 1.0 / u : 0.25 / u;
            for (int ax = 0; ax < nd; ++ax) {
                e = timed(kPassElementwise, stream, [&] {
                    return launch_phase_refine_axis(R, n, axes, ax, radius, step, static_cast<double2 *>(po),
                                                    static_cast<double2 *>(pt), static_cast<double2 *>(pp),
                                                    dst_state, stream);
                });
                if (e) return cuda_fail(e, "refinement launch");
            }
        }
    }
    // Error terms (:231-253).
    e = timed(kPassElementwise, stream, [&] {
        return launch_phase_error_terms(static_cast<const float *>(reference->data),
                                        static_cast<const float *>(moving->data), A, B, n, axes, dst_state,
                                        s->normalize_phase ? 1 : 0, static_cast<double *>(pp), dsums, stream);
    });
    if (e) return cuda_fail(e, "error terms launch");
    PcState hs;
    double sums[4];
    cudaStream_t cst = static_cast<cudaStream_t>(stream);
    CUDA_TRY(cudaMemcpyAsync(&hs, dst_state, sizeof hs, cudaMemcpyDeviceToHost, cst), "state download");
    CUDA_TRY(cudaMemcpyAsync(sums, dsums, sizeof sums, cudaMemcpyDeviceToHost, cst), "sums download");
    CUDA_TRY(cudaStreamSynchronize(cst), "synchronise");
    for (int d = 0; d < LUCEM_MAX_DIMS; ++d) result->shift[d] = 0.0;
    for (int d = 0; d < reference->ndim; ++d) {
        double v = hs.shift[d];
        if (s->upsample_factor > 1) v = std::round(v * u) / u;  // :224-226
        result->shift[d] = v;
    }
    result->phasediff = std::atan2(hs.peak_im, hs.peak_re);
    const double nn = (double)n, denom = sums[0] * sums[1];
    if (denom <= DBL_EPSILON) {
        result->error = 0.0;
    } else {
        double amp2;
        if (!s->normalize_phase) {
            amp2 = (hs.peak_re * hs.peak_re + hs.peak_im * hs.peak_im) * nn * nn;
        } else {
            const double ur = sums[2] / nn, ui = sums[3] / nn;
            amp2 = (ur * ur + ui * ui) * nn * nn;
        }
        result->error = std::sqrt(1.0 - std::min(std::max(amp2 / denom, 0.0), 1.0));
    }
    return ok();
}

void lucem_unsupervised_wiener_settings_default(lucem_unsupervised_wiener_settings *s) {
    s->num_iter = 30;
    s->burnin = 10;
    s->clip = 1;
    s->seed = 0;
}

// restore/deconvolve.rs:357-509.
lucem_status lucem_unsupervised_wiener(lucem_ctx *ctx, const lucem_tensor *in, const lucem_tensor *psf,
                                       const lucem_unsupervised_wiener_settings *settings, lucem_tensor *out,
                                       double *balance_chain, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_unsupervised_wiener_settings def;
    lucem_unsupervised_wiener_settings_default(&def);
    const lucem_unsupervised_wiener_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_tensor("input", in)) || (st = check_tensor("psf", psf)) || (st = check_tensor("output", out)))
        return st;
    // deconvolve.rs:363-381, same order.
    if (in->ndim != 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION,
                    "unsupervised_wiener input expects 2-D array, got %d-D shape %s", in->ndim, dims_str(in).c_str());
    if (psf->ndim != 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION,
                    "unsupervised_wiener psf expects 2-D array, got %d-D shape %s", psf->ndim, dims_str(psf).c_str());
    if (numel(psf) == 0) return fail(LUCEM_ERR_INVALID_WEIGHTS, "psf: PSF cannot be empty");
    if (s->num_iter <= 0 || s->burnin < 0 || s->burnin >= s->num_iter)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `num_iter`: num_iter (%lld) must be > burnin (%lld) and >= 1",
                    (long long)s->num_iter, (long long)s->burnin);
    if ((st = same_shape("input", in, "output", out)) || (st = not_aliased(in, out))) return st;
    if (in->dtype != LUCEM_F32 || psf->dtype != LUCEM_F32 || out->dtype != LUCEM_F32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "unsupervised_wiener takes f32 input, psf and output");
    if (numel(in) == 0) return ok();
    const int64_t H = in->dims[0], W = in->dims[1], n = H * W;
    // The PSF is placed on the image grid by its centre (as wiener_deconvolve).
    if (psf->dims[0] > H || psf->dims[1] > W)
        return fail(LUCEM_ERR_INVALID_WEIGHTS, "psf: PSF dimensions must not exceed image dimensions");
    void *bufs[4] = {};
    const char *names[4] = {"wiener_y", "wiener_h", "wiener_l", "wiener_x"};
    for (int i = 0; i < 4; ++i)
        if ((st = ws->get(names[i], (size_t)n * sizeof(float2_), &bufs[i]))) return st;
    float2_ *Y = static_cast<float2_ *>(bufs[0]), *Hk = static_cast<float2_ *>(bufs[1]);
    float2_ *Lk = static_cast<float2_ *>(bufs[2]), *X = static_cast<float2_ *>(bufs[3]);
    void *pp = nullptr, *pm = nullptr, *ppart = nullptr, *pst = nullptr, *pch = nullptr;
    if ((st = ws->get("uw_spec", (size_t)n * sizeof(float4_), &pp)) ||
        (st = ws->get("uw_mean", (size_t)n * sizeof(double2), &pm)) ||
        (st = ws->get("uw_part", (size_t)(3 * kRedBlocks + 2) * sizeof(double), &ppart)) ||
        (st = ws->get("uw_state", sizeof(UwState), &pst)) ||
        (st = ws->get("uw_chain", (size_t)s->num_iter * sizeof(double), &pch)))
        return st;
    // Y, H and L as in wiener_deconvolve (deconvolve.rs:383-420).
    FftSide src, dst;
    src.re = static_cast<const float *>(in->data);
    dst.c = Y;
    if ((st = fft_nd(ctx, in->dims, 2, src, dst, false, 0, ws, stream))) return st;
    auto centred_fft = [&](const float *k, int kh, int kw, float2_ *dst_c) -> lucem_status {
        int e = launch_centre_kernel(k, kh, kw, X, (int)H, (int)W, stream);
        if (e) return cuda_fail(e, "kernel centring");
        FftSide a, b;
        a.c = X;
        b.c = dst_c;
        return fft_nd(ctx, in->dims, 2, a, b, false, 0, ws, stream);
    };
    if ((st = centred_fft(static_cast<const float *>(psf->data), (int)psf->dims[0], (int)psf->dims[1], Hk))) return st;
    const bool lap3 = H >= 3 && W >= 3;
    const float lap[9] = {0, -1, 0, -1, 4, -1, 0, -1, 0}, one = 1.0f;
    int err = 0;
    void *lapd = ctx->get_or_upload(lap3 ? "wiener-laplacian-3x3" : "wiener-laplacian-1x1", lap3 ? lap : &one,
                                    lap3 ? sizeof lap : sizeof one, &err);
    if (!lapd) return cuda_fail(err, "laplacian upload");
    if ((st = centred_fft(static_cast<const float *>(lapd), lap3 ? 3 : 1, lap3 ? 3 : 1, Lk))) return st;
    // The chain (deconvolve.rs:433-483), on the device.
    float4_ *P = static_cast<float4_ *>(pp);
    double2 *mean = static_cast<double2 *>(pm);
    double *part = static_cast<double *>(ppart), *chain = static_cast<double *>(pch);
    UwState *ust = static_cast<UwState *>(pst);
    int e = timed(kPassElementwise, stream, [&] {
        return launch_uw_setup(static_cast<const float *>(in->data), Y, Hk, Lk, P, n, s->seed, part, ust, mean,
                               stream);
    });
    if (e) return cuda_fail(e, "unsupervised wiener setup");
    for (int64_t it = 0; it < s->num_iter; ++it) {
        e = timed(kPassElementwise, stream, [&] {
            return launch_uw_iteration(Y, Hk, P, n, it >= s->burnin ? 1 : 0, mean, part, ust, chain, (int)it, stream);
        });
        if (e) return cuda_fail(e, "unsupervised wiener iteration");
    }
    const int64_t count = s->num_iter - s->burnin;
    e = timed(kPassElementwise, stream,
              [&] { return launch_uw_mean(mean, n, 1.0 / (double)(count > 0 ? count : 1), X, stream); });
    if (e) return cuda_fail(e, "posterior mean");
    FftSide xs, os;
    xs.c = X;
    os.wre = static_cast<float *>(out->data);
    if ((st = fft_nd(ctx, in->dims, 2, xs, os, true, s->clip ? 1 : 0, ws, stream))) return st;
    if (balance_chain) {
        cudaStream_t cst = static_cast<cudaStream_t>(stream);
        CUDA_TRY(cudaMemcpyAsync(balance_chain, chain, (size_t)s->num_iter * sizeof(double), cudaMemcpyDeviceToHost,
                                 cst),
                 "chain download");
        CUDA_TRY(cudaStreamSynchronize(cst), "synchronise");
    }
    return ok();
}

}  // extern "C"


// ---------------------------------------------------------------------------
// Helpers shared with other translation units (internal.h).

namespace lucem {

lucem_status gaussian_blur_plan(const lucem_tensor *in, const double *sigmas, int32_t n_sigmas,
                                const lucem_gaussian_settings *settings, const lucem_tensor *out,
                                std::vector<GaussPass> *passes) {
    lucem_gaussian_settings def;
    lucem_gaussian_settings_default(&def);
    const lucem_gaussian_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_in_out(in, out))) return st;
    if ((st = check_mode(s->mode))) return st;
    return plan_passes(in->ndim, sigmas, n_sigmas, s, passes);
}

bool gaussian_fuse_last_two(const lucem_tensor *in, const std::vector<GaussPass> &passes) {
    const int nd = in->ndim;
    const size_t np = passes.size();
    return np >= 2 && passes[np - 2].axis == nd - 2 && passes[np - 1].axis == nd - 1 &&
           passes[np - 2].radius <= kFamMaxRadius && passes[np - 1].radius <= kFamMaxRadius &&
           in->dims[nd - 2] < (1 << 30) && in->dims[nd - 1] < (1 << 30);
}

std::vector<float> gaussian_pass_taps(const GaussPass &p) { return taps_f32(p.sigma, p.order, p.radius); }

void gaussian_fused_params(FamParams *fp, const lucem_tensor *view, int mode, double cval, float scale,
                           const GaussPass &rows, const GaussPass &cols, float *out) {
    init_fam(fp, view, mode, cval, scale);
    fp->n_filters = 1;
    fill_filter_taps(fp, 0, &rows, &cols);
    fp->rmax0 = fp->r0[0];
    fp->rmax1 = fp->r1[0];
    fp->n_outputs = 1;
    FamOutput &o = fp->outs[0];
    o.out = out;
    o.plane_stride = (int64_t)fp->H * fp->W;
    o.row_pitch = fp->W;
    o.combine = (int)Combine::kLinear;
    o.fa = 0;
    o.fb = -1;
    o.alpha = 1.0f;
    o.beta = 0.0f;
    o.bias = 0.0f;
}

lucem_status set_error(lucem_status st, const char *msg) { return fail(st, "%s", msg); }

}  // namespace lucem

// ---------------------------------------------------------------------------
// Gaussian-consumer operators: Hessian, shape index, structure tensor and
// the ridge filters (crates/lucem-ops/src/feature/structure.rs,
// filter/ridge.rs).  Every scale's three Hessian filters run from one staged
// tile in one launch of the fused family kernel, the per-pixel tensor math
// (tensor_ops.cuh) in its epilogue; filters wider than the fused kernel take
// the per-axis passes and the same math elementwise.

namespace {

// Outputs of one fused launch with a tensor epilogue (or none).
struct TensorOuts {
    float *o[3] = {nullptr, nullptr, nullptr};
};

lucem_status check_2d(const char *op, const lucem_tensor *in) {
    if (in->ndim != 2)
        return fail(LUCEM_ERR_INVALID_DIMENSION, "%s expects 2-D array, got %d-D shape %s", op, in->ndim,
                    dims_str(in).c_str());
    return ok();
}

lucem_status check_sigma(double sigma) {
    // gaussian.rs:96-101 (the blurs these operators run).
    if (!std::isfinite(sigma) || sigma < 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `sigma`: sigma must be finite and non-negative, got %g", sigma);
    return ok();
}

// One filter of a fused tensor launch: Gaussian of `sigma` (truncate 4) with
// derivative orders (order0 along rows, order1 along columns).
struct TensorFilter {
    double sigma;
    uint32_t order0, order1;
};

// Up to three 2-D Gaussian-derivative filters of `in` written as (a, b, c)
// into outs when tensor is kTensorNone, else combined per pixel through the
// epilogue `tensor` into outs: one fused family launch when every radius fits
// the fused kernel, else the per-axis passes into workspace arrays and the
// same epilogue elementwise.
lucem_status filters_tensor(lucem_ctx *ctx, const lucem_tensor *in, const TensorFilter *flt, int nf, int mode,
                            double cval, int tensor, float p0, float p1, int black, int first, const TensorOuts &outs,
                            lucem_workspace *ws, void *stream) {
    const int64_t n = numel(in), H = in->dims[0], W = in->dims[1];
    if (n == 0) return ok();
    int64_t r[3] = {0, 0, 0}, rmax = 0;
    for (int f = 0; f < nf; ++f) {
        r[f] = flt[f].sigma > 0.0 ? (int64_t)radius_of(4.0, flt[f].sigma) : 0;
        rmax = std::max(rmax, r[f]);
    }
    if (rmax <= kFamMaxRadius && H < (1 << 30) && W < (1 << 30)) {
        FamParams fp;
        init_fam(&fp, in, mode, cval, 1.0);
        fp.n_filters = nf;
        for (int f = 0; f < nf; ++f) {
            Pass a{0, flt[f].sigma, flt[f].order0, r[f]}, b{1, flt[f].sigma, flt[f].order1, r[f]};
            // sigma 0: the reference drops the axis (a copy, orders ignored).
            const bool on = flt[f].sigma > 0.0;
            fill_filter_taps(&fp, f, on ? &a : nullptr, on ? &b : nullptr);
            fp.rmax0 = std::max(fp.rmax0, fp.r0[f]);
            fp.rmax1 = std::max(fp.rmax1, fp.r1[f]);
        }
        fp.n_outputs = 3;
        for (int k = 0; k < 3; ++k) {
            FamOutput &o = fp.outs[k];
            o.out = outs.o[k];
            o.plane_stride = H * W;
            o.row_pitch = W;
            o.combine = (int)Combine::kLinear;
            o.fa = k < nf ? k : -1;
            o.fb = -1;
            o.alpha = 1.0f;
        }
        fp.tensor = tensor;
        fp.tensor_black = black;
        fp.tensor_first = first;
        fp.tensor_p0 = p0;
        fp.tensor_p1 = p1;
        if (lucem_status st = fam_waits(ws, &fp, stream)) return st;
        int e = timed(kPassFamily, stream, [&] { return launch_family_planes(fp, in->dtype, stream); });
        return e ? cuda_fail(e, "fused filter launch") : ok();
    }
    // Wider filters: the components by the per-axis passes, then the epilogue.
    float *comp[3] = {outs.o[0], outs.o[1], outs.o[2]};
    if (tensor != kTensorNone) {
        if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
        const char *names[3] = {"tensor_a", "tensor_b", "tensor_c"};
        for (int k = 0; k < nf; ++k) {
            void *p = nullptr;
            if (lucem_status st = ws->get(names[k], (size_t)n * sizeof(float), &p)) return st;
            comp[k] = static_cast<float *>(p);
        }
    }
    for (int f = 0; f < nf; ++f) {
        std::vector<Pass> passes = {Pass{0, flt[f].sigma, flt[f].order0, r[f]},
                                    Pass{1, flt[f].sigma, flt[f].order1, r[f]}};
        if (flt[f].sigma <= 0.0) passes.clear();
        if (lucem_status st = run_passes(ctx, in, passes, mode, cval, 1.0, comp[f], ws, stream)) return st;
    }
    if (tensor == kTensorNone) return ok();
    int e = timed(kPassElementwise, stream, [&] {
        return launch_tensor_elementwise(comp[0], comp[1], nf > 2 ? comp[2] : nullptr, outs.o[0], outs.o[1],
                                         outs.o[2], n, tensor, p0, p1, black, first, stream);
    });
    return e ? cuda_fail(e, "tensor epilogue launch") : ok();
}

// The three Hessian filters of one scale, orders (2,0), (1,1), (0,2) at
// sigma (structure.rs:26-51), through filters_tensor.
lucem_status hessian_scale(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int mode, double cval, int tensor,
                           float p0, float p1, int black, int first, const TensorOuts &outs, lucem_workspace *ws,
                           void *stream) {
    const TensorFilter h[3] = {{sigma, 2, 0}, {sigma, 1, 1}, {sigma, 0, 2}};
    return filters_tensor(ctx, in, h, 3, mode, cval, tensor, p0, p1, black, first, outs, ws, stream);
}

// Checks of the single-scale Hessian operators: 2-D input, f32 outputs of
// its shape, none aliasing the input or another output.
lucem_status check_hessian_io(const char *op, const lucem_tensor *in, double sigma, int32_t mode,
                              std::initializer_list<const lucem_tensor *> outs) {
    lucem_status st;
    if ((st = check_tensor("input", in))) return st;
    if ((st = check_2d(op, in)) || (st = check_mode(mode)) || (st = check_sigma(sigma))) return st;
    for (const lucem_tensor *o : outs) {
        if ((st = check_tensor("output", o)) || (st = same_shape("input", in, "output", o)) ||
            (st = not_aliased(in, o)) || (st = require_f32_out(o)))
            return st;
        for (const lucem_tensor *o2 : outs)
            if (o2 != o && (st = not_aliased(o, o2))) return st;
    }
    return ok();
}

}  // namespace

extern "C" {

// structure.rs:16-54.
lucem_status lucem_hessian_matrix(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                  lucem_tensor *hrr, lucem_tensor *hrc, lucem_tensor *hcc, lucem_workspace *ws,
                                  void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_hessian_io("hessian_matrix", in, sigma, mode, {hrr, hrc, hcc}))) return st;
    TensorOuts o;
    o.o[0] = static_cast<float *>(hrr->data);
    o.o[1] = static_cast<float *>(hrc->data);
    o.o[2] = static_cast<float *>(hcc->data);
    return hessian_scale(ctx, in, sigma, mode, cval, kTensorNone, 0.f, 0.f, 0, 1, o, ws, stream);
}

// structure.rs:57-83.
lucem_status lucem_hessian_det(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                               lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_hessian_io("hessian_matrix", in, sigma, mode, {out}))) return st;
    TensorOuts o;
    o.o[0] = static_cast<float *>(out->data);
    return hessian_scale(ctx, in, sigma, mode, cval, kTensorDet, 0.f, 0.f, 0, 1, o, ws, stream);
}

// structure.rs:86-97.
lucem_status lucem_hessian_eigvals(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                   lucem_tensor *eig1, lucem_tensor *eig2, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_hessian_io("hessian_matrix", in, sigma, mode, {eig1, eig2}))) return st;
    TensorOuts o;
    o.o[0] = static_cast<float *>(eig1->data);
    o.o[1] = static_cast<float *>(eig2->data);
    return hessian_scale(ctx, in, sigma, mode, cval, kTensorEigvals, 0.f, 0.f, 0, 1, o, ws, stream);
}

// structure.rs:164-191.
lucem_status lucem_shape_index(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                               lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_status st;
    if ((st = check_hessian_io("hessian_matrix", in, sigma, mode, {out}))) return st;
    TensorOuts o;
    o.o[0] = static_cast<float *>(out->data);
    return hessian_scale(ctx, in, sigma, mode, cval, kTensorShapeIndex, 0.f, 0.f, 0, 1, o, ws, stream);
}

// structure.rs:102-147: Sobel gradients (gradient.rs:71-107: [-1, 0, 1] along
// the derivative axis, [1, 2, 1] across), their outer products, each
// smoothed by the Gaussian window.  Here: both gradients and the three
// products in one fused launch (into the workspace), then the three planes'
// Gaussian blurs.
lucem_status lucem_structure_tensor(lucem_ctx *ctx, const lucem_tensor *in, double sigma, int32_t mode, double cval,
                                    lucem_tensor *arr, lucem_tensor *arc, lucem_tensor *acc, lucem_workspace *ws,
                                    void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_status st;
    if ((st = check_hessian_io("structure_tensor", in, sigma, mode, {arr, arc, acc}))) return st;
    const int64_t n = numel(in), H = in->dims[0], W = in->dims[1];
    if (n == 0) return ok();
    if (H >= (1 << 30) || W >= (1 << 30))
        return fail(LUCEM_ERR_TOO_MANY_ELEMENTS, "structure_tensor: a side of 2^30 or more");
    void *prods = nullptr;
    if ((st = ws->get("structure_products", (size_t)3 * n * sizeof(float), &prods))) return st;
    float *P = static_cast<float *>(prods);
    FamParams fp;
    init_fam(&fp, in, mode, cval, 1.0);
    fp.n_filters = 2;
    const float deriv[3] = {-1.0f, 0.0f, 1.0f}, smooth[3] = {1.0f, 2.0f, 1.0f};
    for (int f = 0; f < 2; ++f) {
        std::memset(fp.taps0[f], 0, sizeof fp.taps0[f]);
        std::memset(fp.taps1[f], 0, sizeof fp.taps1[f]);
        // Kernel radius 2 (the fused kernel's even radii): taps at 1..3.
        const float *t0 = f == 0 ? deriv : smooth, *t1 = f == 0 ? smooth : deriv;
        for (int i = 0; i < 3; ++i) {
            fp.taps0[f][i + 1] = float2_{t0[i], t0[i]};
            fp.taps1[f][i + 1] = float2_{t1[i], t1[i]};
        }
        fp.r0[f] = fp.r1[f] = fam_kernel_radius(1);
    }
    fp.rmax0 = fp.rmax1 = fam_kernel_radius(1);
    fp.n_outputs = 3;
    for (int k = 0; k < 3; ++k) {
        FamOutput &o = fp.outs[k];
        o.out = P + (size_t)k * n;
        o.plane_stride = n;
        o.row_pitch = W;
        o.combine = (int)Combine::kLinear;
        o.fa = k < 2 ? k : -1;
        o.fb = -1;
        o.alpha = 1.0f;
    }
    fp.tensor = kTensorOuter;
    if ((st = fam_waits(ws, &fp, stream))) return st;
    int e = timed(kPassFamily, stream, [&] { return launch_family_planes(fp, in->dtype, stream); });
    if (e) return cuda_fail(e, "structure tensor gradient launch");
    // The Gaussian window over each product (gaussian_blur_into, orders 0).
    const int64_t r = sigma > 0.0 ? (int64_t)radius_of(4.0, sigma) : 0;
    std::vector<Pass> passes;
    if (sigma > 0.0) passes = {Pass{0, sigma, 0, r}, Pass{1, sigma, 0, r}};
    lucem_tensor* outs[3] = {arr, arc, acc};
    for (int k = 0; k < 3; ++k) {
        lucem_tensor view = *in;
        view.data = P + (size_t)k * n;
        view.dtype = LUCEM_F32;
        if ((st = run_passes(ctx, &view, passes, mode, cval, 1.0, static_cast<float *>(outs[k]->data), ws, stream)))
            return st;
    }
    return ok();
}

// structure.rs:150-161 (symmetric_eigenvalues_2x2_into, core/eigen.rs).
lucem_status lucem_structure_tensor_eigvals(const lucem_tensor *arr, const lucem_tensor *arc, const lucem_tensor *acc,
                                            lucem_tensor *eig1, lucem_tensor *eig2, void *stream) {
    lucem_status st;
    const lucem_tensor *ins[3] = {arr, arc, acc};
    for (const lucem_tensor *t : ins)
        if ((st = check_tensor("input", t))) return st;
    if ((st = check_tensor("eig1", eig1)) || (st = check_tensor("eig2", eig2))) return st;
    for (const lucem_tensor *t : {arc, acc, (const lucem_tensor *)eig1, (const lucem_tensor *)eig2})
        if ((st = same_shape("arr", arr, "other", t))) return st;
    for (const lucem_tensor *t : {arr, arc, acc, (const lucem_tensor *)eig1, (const lucem_tensor *)eig2})
        if (t->dtype != LUCEM_F32) return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "structure_tensor_eigvals takes f32 arrays");
    for (const lucem_tensor *t : ins)
        if ((st = not_aliased(t, eig1)) || (st = not_aliased(t, eig2))) return st;
    if ((st = not_aliased(eig1, eig2))) return st;
    const int64_t n = numel(arr);
    int e = launch_tensor_elementwise(static_cast<const float *>(arr->data), static_cast<const float *>(arc->data),
                                      static_cast<const float *>(acc->data), static_cast<float *>(eig1->data),
                                      static_cast<float *>(eig2->data), nullptr, n, kTensorEigvals, 0.f, 0.f, 0, 1,
                                      stream);
    return e ? cuda_fail(e, "eigenvalue launch") : ok();
}

void lucem_ridge_settings_default(lucem_ridge_settings *s) {
    s->sigmas = nullptr;
    s->n_sigmas = 0;
    s->black_ridges = 1;
    s->mode = LUCEM_PAD_REFLECT;
    s->cval = 0.0;
    s->beta = 0.5;
    s->gamma = 15.0;
}

}  // extern "C"

namespace {

// frangi_into / sato_into / meijering_into (ridge.rs:87-245): per scale the
// Hessian eigenvalues and the scale's response folded into the running
// maximum, all in the scale's one fused launch.
lucem_status ridge_filter(lucem_ctx *ctx, const char *op, int tensor, const lucem_tensor *in,
                          const lucem_ridge_settings *settings, lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    lucem_ridge_settings def;
    lucem_ridge_settings_default(&def);
    const lucem_ridge_settings *s = settings ? settings : &def;
    static const double kDefaultSigmas[5] = {1.0, 3.0, 5.0, 7.0, 9.0};
    const double *sig = s->sigmas ? s->sigmas : kDefaultSigmas;
    const int ns = s->sigmas ? s->n_sigmas : 5;
    lucem_status st;
    if ((st = check_tensor("input", in)) || (st = check_tensor("output", out))) return st;
    if ((st = check_2d(op, in)) || (st = same_shape("input", in, "output", out)) || (st = not_aliased(in, out)))
        return st;
    if ((st = require_f32_out(out)) || (st = check_mode(s->mode))) return st;
    if (tensor == kTensorFrangi && ns <= 0)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `sigmas`: at least one sigma scale is required");
    for (int i = 0; i < ns; ++i)
        if ((st = check_sigma(sig[i]))) return st;
    const int64_t n = numel(in);
    if (n == 0) return ok();
    if (ns <= 0) {
        // The output starts at zero (ridge.rs:165-166) and no scale raises it.
        CUDA_TRY(cudaMemsetAsync(out->data, 0, (size_t)n * sizeof(float), static_cast<cudaStream_t>(stream)), "fill");
        return ok();
    }
    const float p1 = (float)(1.0 / (2.0 * std::max(s->gamma * s->gamma, 1e-12)));
    TensorOuts o;
    o.o[0] = static_cast<float *>(out->data);
    for (int i = 0; i < ns; ++i) {
        float p0 = 0.0f;
        if (tensor == kTensorFrangi) p0 = (float)(1.0 / (2.0 * std::max(s->beta * s->beta, 1e-12)));
        if (tensor == kTensorSato) p0 = (float)(sig[i] * sig[i]);
        if ((st = hessian_scale(ctx, in, sig[i], s->mode, s->cval, tensor, p0, p1, s->black_ridges ? 1 : 0,
                                i == 0 ? 1 : 0, o, ws, stream)))
            return st;
    }
    return ok();
}

}  // namespace

extern "C" {

lucem_status lucem_frangi(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                          lucem_tensor *out, lucem_workspace *ws, void *stream) {
    return ridge_filter(ctx, "frangi", kTensorFrangi, in, settings, out, ws, stream);
}

lucem_status lucem_sato(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                        lucem_tensor *out, lucem_workspace *ws, void *stream) {
    return ridge_filter(ctx, "sato", kTensorSato, in, settings, out, ws, stream);
}

lucem_status lucem_meijering(lucem_ctx *ctx, const lucem_tensor *in, const lucem_ridge_settings *settings,
                             lucem_tensor *out, lucem_workspace *ws, void *stream) {
    return ridge_filter(ctx, "meijering", kTensorMeijering, in, settings, out, ws, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Blob detectors (crates/lucem-ops/src/feature/blobs.rs): the scale stack on
// the device (one fused launch per scale), its maxima by one kernel
// (features.cu), sorting and overlap pruning on the host.

namespace {

enum class BlobKind { kLog, kDog, kDoh };

// BlobDetector::validate (blobs.rs:68-94).
lucem_status blob_validate(const lucem_blob_settings *s) {
    if (!std::isfinite(s->min_sigma) || s->min_sigma <= 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `min_sigma`: min_sigma must be positive, got %g",
                    s->min_sigma);
    if (!std::isfinite(s->max_sigma) || s->max_sigma < s->min_sigma)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `max_sigma`: max_sigma (%g) must be >= min_sigma (%g)", s->max_sigma,
                    s->min_sigma);
    if (s->num_sigma <= 0)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `num_sigma`: num_sigma must be at least 1");
    if (!(s->overlap >= 0.0 && s->overlap <= 1.0))
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `overlap`: overlap must be in 0.0..=1.0, got %g",
                    s->overlap);
    return ok();
}

// BlobDetector::sigmas (blobs.rs:96-111).
std::vector<double> blob_sigmas(const lucem_blob_settings *s) {
    if (s->num_sigma == 1 || std::fabs(s->max_sigma - s->min_sigma) <= DBL_EPSILON) return {s->min_sigma};
    std::vector<double> v((size_t)s->num_sigma);
    for (int64_t i = 0; i < s->num_sigma; ++i) {
        const double t = (double)i / (double)(s->num_sigma - 1);
        v[(size_t)i] = s->log_scale ? s->min_sigma * std::pow(s->max_sigma / s->min_sigma, t)
                                    : s->min_sigma + t * (s->max_sigma - s->min_sigma);
    }
    return v;
}

// circle_overlap_fraction (blobs.rs:114-136): the lens area of two circles of
// radius sqrt(2) sigma over the smaller circle's area.
double blob_overlap(const lucem_blob &a, const lucem_blob &b) {
    const double r1 = M_SQRT2 * a.sigma, r2 = M_SQRT2 * b.sigma;
    const double dy = (double)a.y - (double)b.y, dx = (double)a.x - (double)b.x;
    const double d = std::sqrt(dy * dy + dx * dx);
    if (d >= r1 + r2) return 0.0;
    if (d <= std::fabs(r1 - r2)) return 1.0;
    const double rmin = std::min(r1, r2);
    if (rmin <= 0.0) return 0.0;
    const double c1 = std::min(std::max((d * d + r1 * r1 - r2 * r2) / (2.0 * d * r1), -1.0), 1.0);
    const double c2 = std::min(std::max((d * d + r2 * r2 - r1 * r1) / (2.0 * d * r2), -1.0), 1.0);
    const double t1 = r1 * r1 * std::acos(c1), t2 = r2 * r2 * std::acos(c2);
    const double sq = (-d + r1 + r2) * (d + r1 - r2) * (d - r1 + r2) * (d + r1 + r2);
    const double area = t1 + t2 - 0.5 * std::sqrt(std::max(sq, 0.0));
    return area / (M_PI * rmin * rmin);
}

lucem_status blobs_run(lucem_ctx *ctx, BlobKind kind, const lucem_tensor *in, const lucem_blob_settings *settings,
                       lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    if (!n_out || (cap > 0 && !out)) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `out`: null");
    *n_out = 0;
    lucem_blob_settings def;
    lucem_blob_settings_default(&def);
    const lucem_blob_settings *s = settings ? settings : &def;
    const char *op = kind == BlobKind::kLog ? "blobs_log" : kind == BlobKind::kDog ? "blobs_dog" : "blobs_doh";
    lucem_status st;
    if ((st = check_tensor("image", in)) || (st = check_2d(op, in)) || (st = blob_validate(s))) return st;
    std::vector<double> sig;
    if (kind == BlobKind::kDog) {
        // blobs.rs:244-263: sigma, sigma * ratio, ... up to max_sigma.
        if (!std::isfinite(s->sigma_ratio) || s->sigma_ratio <= 1.0)
            return fail(LUCEM_ERR_INVALID_PARAMETER,
                        "invalid parameter `sigma_ratio`: sigma_ratio must be > 1.0, got %g", s->sigma_ratio);
        for (double v = s->min_sigma; v <= s->max_sigma * (1.0 + 1e-9); v *= s->sigma_ratio) sig.push_back(v);
        if (sig.empty()) sig.push_back(s->min_sigma);
    } else {
        sig = blob_sigmas(s);
    }
    const int64_t n = numel(in), H = in->dims[0], W = in->dims[1];
    if (n == 0) return ok();
    const int ns = (int)sig.size();
    const int64_t border = std::max<int64_t>(s->exclude_border, 1);
    if (H <= 2 * border || W <= 2 * border) return ok();
    void *pc = nullptr, *pl = nullptr, *pn = nullptr;
    const int64_t bound = blob_candidate_bound(ns, H, W);
    if ((st = ws->get("blob_stack", (size_t)ns * (size_t)n * sizeof(float), &pc)) ||
        (st = ws->get("blob_candidates", (size_t)bound * sizeof(BlobCandidate), &pl)) ||
        (st = ws->get("blob_count", sizeof(unsigned long long), &pn)))
        return st;
    float *cube = static_cast<float *>(pc);
    // The scale stack: one fused launch per scale, the reference's scaling in
    // the epilogue.
    for (int i = 0; i < ns; ++i) {
        const double sg = sig[(size_t)i];
        TensorOuts o;
        o.o[0] = cube + (size_t)i * (size_t)n;
        if (kind == BlobKind::kLog) {
            // -sigma^2 (d2/dy2 + d2/dx2) G * I (blobs.rs:219-232).
            const TensorFilter f[2] = {{sg, 2, 0}, {sg, 0, 2}};
            st = filters_tensor(ctx, in, f, 2, LUCEM_PAD_REFLECT, 0.0, kTensorScaledSum, (float)(-(sg * sg)), 1.0f, 0,
                                1, o, ws, stream);
        } else if (kind == BlobKind::kDog) {
            // (G(sigma) - G(ratio sigma)) * I / (ratio - 1) (blobs.rs:265-283).
            const TensorFilter f[2] = {{sg, 0, 0}, {sg * s->sigma_ratio, 0, 0}};
            st = filters_tensor(ctx, in, f, 2, LUCEM_PAD_REFLECT, 0.0, kTensorScaledSum,
                                (float)(1.0 / (s->sigma_ratio - 1.0)), -1.0f, 0, 1, o, ws, stream);
        } else {
            // sigma^4 det H (blobs.rs:313-339).
            const TensorFilter f[3] = {{sg, 2, 0}, {sg, 1, 1}, {sg, 0, 2}};
            st = filters_tensor(ctx, in, f, 3, LUCEM_PAD_REFLECT, 0.0, kTensorScaledDet, (float)std::pow(sg, 4.0),
                                0.0f, 0, 1, o, ws, stream);
        }
        if (st) return st;
    }
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    unsigned long long *cnt = static_cast<unsigned long long *>(pn);
    CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof *cnt, cs), "count reset");
    int e = timed(kPassElementwise, stream, [&] {
        return launch_blob_candidates(cube, ns, (int)H, (int)W, (int)border, s->threshold,
                                      static_cast<BlobCandidate *>(pl), bound, cnt, stream);
    });
    if (e) return cuda_fail(e, "blob maxima launch");
    unsigned long long count = 0;
    CUDA_TRY(cudaMemcpyAsync(&count, cnt, sizeof count, cudaMemcpyDeviceToHost, cs), "count download");
    CUDA_TRY(cudaStreamSynchronize(cs), "synchronise");
    const size_t nc = (size_t)std::min<unsigned long long>(count, (unsigned long long)bound);
    std::vector<BlobCandidate> cand(nc);
    if (nc) {
        CUDA_TRY(cudaMemcpyAsync(cand.data(), pl, nc * sizeof(BlobCandidate), cudaMemcpyDeviceToHost, cs),
                 "candidate download");
        CUDA_TRY(cudaStreamSynchronize(cs), "synchronise");
    }
    // blobs.rs:183-200: response descending, then y, x (the reference's stable
    // sort keeps scale order on full ties); then the greedy overlap pruning.
    std::sort(cand.begin(), cand.end(), [](const BlobCandidate &a, const BlobCandidate &b) {
        if (a.response != b.response) return a.response > b.response;
        if (a.y != b.y) return a.y < b.y;
        if (a.x != b.x) return a.x < b.x;
        return a.s < b.s;
    });
    // The greedy pass checks each candidate against the blobs kept so far.
    // Two blobs overlap only closer than r1 + r2 <= 2 sqrt(2) max sigma, so
    // the kept blobs are bucketed on a grid of that cell and a candidate
    // meets only those of its 3 x 3 cells: the same decisions as checking
    // every kept blob (a zero overlap never exceeds the threshold).
    std::vector<lucem_blob> kept;
    // Cells no smaller than the overlap reach; no more cells than about
    // four per candidate (a large image with small sigmas stays bounded).
    const double reach = 2.0 * M_SQRT2 * *std::max_element(sig.begin(), sig.end());
    const double cell = std::max(reach, std::sqrt((double)H * (double)W /
                                                  (double)std::max<size_t>(1024, 4 * cand.size())));
    const int64_t gx = std::max<int64_t>(1, (int64_t)std::ceil((double)W / cell));
    const int64_t gy = std::max<int64_t>(1, (int64_t)std::ceil((double)H / cell));
    std::vector<std::vector<int32_t>> grid((size_t)(gx * gy));
    for (const BlobCandidate &c : cand) {
        const lucem_blob b{c.y, c.x, sig[(size_t)c.s], (double)c.response};
        const int64_t cy = std::min<int64_t>(gy - 1, (int64_t)((double)c.y / cell));
        const int64_t cx = std::min<int64_t>(gx - 1, (int64_t)((double)c.x / cell));
        bool drop = false;
        for (int64_t yy = std::max<int64_t>(0, cy - 1); yy <= std::min<int64_t>(gy - 1, cy + 1) && !drop; ++yy)
            for (int64_t xx = std::max<int64_t>(0, cx - 1); xx <= std::min<int64_t>(gx - 1, cx + 1) && !drop; ++xx)
                for (int32_t k : grid[(size_t)(yy * gx + xx)])
                    if (blob_overlap(b, kept[(size_t)k]) > s->overlap) {
                        drop = true;
                        break;
                    }
        if (!drop) {
            grid[(size_t)(cy * gx + cx)].push_back((int32_t)kept.size());
            kept.push_back(b);
        }
    }
    *n_out = (int64_t)kept.size();
    for (int64_t i = 0; i < std::min<int64_t>(cap, (int64_t)kept.size()); ++i) out[i] = kept[(size_t)i];
    return ok();
}

}  // namespace

extern "C" {

void lucem_blob_settings_default(lucem_blob_settings *s) {
    s->min_sigma = 1.0;
    s->max_sigma = 30.0;
    s->num_sigma = 10;
    s->sigma_ratio = 1.6;
    s->threshold = 0.1;
    s->overlap = 0.5;
    s->log_scale = 0;
    s->exclude_border = 1;
}

lucem_status lucem_blobs_log(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream) {
    return blobs_run(ctx, BlobKind::kLog, in, settings, out, cap, n_out, ws, stream);
}

lucem_status lucem_blobs_dog(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream) {
    return blobs_run(ctx, BlobKind::kDog, in, settings, out, cap, n_out, ws, stream);
}

lucem_status lucem_blobs_doh(lucem_ctx *ctx, const lucem_tensor *in, const lucem_blob_settings *settings,
                             lucem_blob *out, int64_t cap, int64_t *n_out, lucem_workspace *ws, void *stream) {
    return blobs_run(ctx, BlobKind::kDoh, in, settings, out, cap, n_out, ws, stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Pyramids (crates/lucem-ops/src/transform/pyramid.rs): the Gaussian blur of
// the fused family path and the resize's resampling (features.cu).

namespace {

// Pyramid::resolved_sigma (pyramid.rs:115-132) and the orders built here.
lucem_status pyramid_sigma(const lucem_pyramid_settings *s, double *sigma) {
    if (!std::isfinite(s->downscale) || s->downscale <= 1.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `downscale`: pyramid scale factor must be > 1.0, got %g", s->downscale);
    const double sg = s->sigma < 0.0 ? 2.0 * s->downscale / 6.0 : s->sigma;
    if (!std::isfinite(sg))
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `sigma`: sigma must be non-negative and finite, got %g", sg);
    if (s->order < 0 || s->order > 5)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `order`: spline order must be in 0..=5, got %d",
                    s->order);
    if (s->order > 1)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `order`: orders 2..=5 (B-spline prefiltered) are not built; use 0 or 1");
    *sigma = sg;
    return check_mode(s->mode);
}

// gaussian_blur_into with the pyramid's sigma, mode and cval, into out (f32).
lucem_status pyramid_blur(lucem_ctx *ctx, const lucem_tensor *in, double sigma, const lucem_pyramid_settings *s,
                          float *out, lucem_workspace *ws, void *stream) {
    std::vector<Pass> passes;
    if (sigma > 0.0) {
        const int64_t r = (int64_t)radius_of(4.0, sigma);
        passes = {Pass{0, sigma, 0, r}, Pass{1, sigma, 0, r}};
    }
    return run_passes(ctx, in, passes, s->mode, s->cval, 1.0, out, ws, stream);
}

// resize (warp.rs:207-251) without anti-aliasing: the inverse map
// y = (H / OH) oy + (H / OH - 1) / 2, likewise x, in f32.
lucem_status pyramid_resample(const float *in, int64_t H, int64_t W, float *out, int64_t OH, int64_t OW,
                              const lucem_pyramid_settings *s, void *stream) {
    const double sy = (double)H / (double)OH, sx = (double)W / (double)OW;
    int e = timed(kPassElementwise, stream, [&] {
        return launch_resample(in, (int)H, (int)W, out, (int)OH, (int)OW, (float)sy, (float)(0.5 * (sy - 1.0)),
                               (float)sx, (float)(0.5 * (sx - 1.0)), s->order, s->mode, (float)s->cval, stream);
    });
    return e ? cuda_fail(e, "resample launch") : ok();
}

lucem_status pyramid_io(const char *op, const lucem_tensor *in, const lucem_tensor *out) {
    lucem_status st;
    if ((st = check_tensor("image", in)) || (st = check_tensor("output", out))) return st;
    if ((st = check_2d(op, in)) || (st = check_2d(op, out)) || (st = require_f32_out(out)) ||
        (st = not_aliased(in, out)))
        return st;
    return ok();
}

}  // namespace

extern "C" {

void lucem_pyramid_settings_default(lucem_pyramid_settings *s) {
    s->downscale = 2.0;
    s->sigma = -1.0;
    s->order = 1;
    s->mode = LUCEM_PAD_REFLECT;
    s->cval = 0.0;
}

// pyramid.rs:135-168.
lucem_status lucem_pyramid_reduce(lucem_ctx *ctx, const lucem_tensor *in, const lucem_pyramid_settings *settings,
                                  lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_pyramid_settings def;
    lucem_pyramid_settings_default(&def);
    const lucem_pyramid_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = pyramid_io("pyramid_reduce", in, out))) return st;
    double sigma;
    if ((st = pyramid_sigma(s, &sigma))) return st;
    const int64_t H = in->dims[0], W = in->dims[1];
    const int64_t OH = std::max<int64_t>(1, (int64_t)std::ceil((double)H / s->downscale));
    const int64_t OW = std::max<int64_t>(1, (int64_t)std::ceil((double)W / s->downscale));
    if (out->dims[0] != OH || out->dims[1] != OW)
        return fail(LUCEM_ERR_SHAPE_MISMATCH, "output shape %s does not match the reduced shape [%lld, %lld]",
                    dims_str(out).c_str(), (long long)OH, (long long)OW);
    if (H == 0 || W == 0) return ok();
    void *pb = nullptr;
    if ((st = ws->get("pyramid_blur", (size_t)(H * W) * sizeof(float), &pb))) return st;
    if ((st = pyramid_blur(ctx, in, sigma, s, static_cast<float *>(pb), ws, stream))) return st;
    return pyramid_resample(static_cast<const float *>(pb), H, W, static_cast<float *>(out->data), OH, OW, s, stream);
}

// pyramid.rs:171-208 (the output shape given by `out`).
lucem_status lucem_pyramid_expand(lucem_ctx *ctx, const lucem_tensor *in, const lucem_pyramid_settings *settings,
                                  lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_pyramid_settings def;
    lucem_pyramid_settings_default(&def);
    const lucem_pyramid_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = pyramid_io("pyramid_expand", in, out))) return st;
    if (in->dtype != LUCEM_F32) return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "pyramid_expand takes an f32 image");
    double sigma;
    if ((st = pyramid_sigma(s, &sigma))) return st;
    const int64_t H = in->dims[0], W = in->dims[1], OH = out->dims[0], OW = out->dims[1];
    if (OH == 0 || OW == 0)
        return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `output_shape`: output_shape dimensions must be >= 1");
    if (H == 0 || W == 0) return ok();
    void *pu = nullptr;
    if ((st = ws->get("pyramid_up", (size_t)(OH * OW) * sizeof(float), &pu))) return st;
    if ((st = pyramid_resample(static_cast<const float *>(in->data), H, W, static_cast<float *>(pu), OH, OW, s,
                               stream)))
        return st;
    lucem_tensor up = *out;
    up.data = pu;
    return pyramid_blur(ctx, &up, sigma, s, static_cast<float *>(out->data), ws, stream);
}

// pyramid.rs:247-262: one band L = fine - expand(coarse).
lucem_status lucem_laplacian_band(lucem_ctx *ctx, const lucem_tensor *fine, const lucem_tensor *coarse,
                                  const lucem_pyramid_settings *settings, lucem_tensor *out, lucem_workspace *ws,
                                  void *stream) {
    lucem_status st;
    if ((st = check_tensor("fine", fine)) || (st = check_tensor("output", out))) return st;
    if ((st = same_shape("fine", fine, "output", out)) || (st = not_aliased(fine, out))) return st;
    if (fine->dtype != LUCEM_F32) return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "laplacian bands take f32 levels");
    if ((st = lucem_pyramid_expand(ctx, coarse, settings, out, ws, stream))) return st;
    // elementwise::linear_combination_into(fine, expanded, 1, -1, 0).
    int e = timed(kPassElementwise, stream, [&] {
        return launch_linear_comb(static_cast<const float *>(fine->data), static_cast<const float *>(out->data),
                                  static_cast<float *>(out->data), numel(fine), 1.0f, -1.0f, 0.0f, stream);
    });
    return e ? cuda_fail(e, "band combine launch") : ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Canny (crates/lucem-ops/src/feature/canny.rs:47-165).  One fused family
// launch gives the Sobel gradients of the smoothed image with the magnitude
// and the direction sector in its epilogue; one kernel suppresses the
// non-maxima and reduces the maximum magnitude; four launches do the
// hysteresis (features.cu).

namespace {

// Correlating with a then with b is correlating with their full convolution
// (offsets add): the Gaussian's 2 r + 1 taps and a 3-tap Sobel stencil make
// 2 r + 3 taps.
std::vector<double> compose3(const std::vector<double> &g, const double (&s)[3]) {
    std::vector<double> c(g.size() + 2, 0.0);
    for (size_t k = 0; k < g.size(); ++k)
        for (int j = 0; j < 3; ++j) c[k + (size_t)j] += g[k] * s[j];
    return c;
}

// The gradient launch over `src`: filter 0 differentiates along rows (the
// reference's gy), filter 1 along columns (gx), each axis' taps given with
// radius `R`; the epilogue writes |g| and the sector.
lucem_status canny_gradient_launch(const lucem_tensor *src, int mode, double cval, const std::vector<double> &ty0,
                                   const std::vector<double> &ty1, const std::vector<double> &tx0,
                                   const std::vector<double> &tx1, int R, float *mag, float *sector,
                                   lucem_workspace *ws, void *stream) {
    FamParams fp;
    init_fam(&fp, src, mode, cval, 1.0);
    fp.n_filters = 2;
    const int kr = fam_kernel_radius(R);
    const std::vector<double> *t[2][2] = {{&ty0, &ty1}, {&tx0, &tx1}};
    for (int f = 0; f < 2; ++f) {
        std::memset(fp.taps0[f], 0, sizeof fp.taps0[f]);
        std::memset(fp.taps1[f], 0, sizeof fp.taps1[f]);
        for (size_t i = 0; i < t[f][0]->size(); ++i) {
            const float a = (float)(*t[f][0])[i], b = (float)(*t[f][1])[i];
            fp.taps0[f][i + (size_t)(kr - R)] = float2_{a, a};
            fp.taps1[f][i + (size_t)(kr - R)] = float2_{b, b};
        }
        fp.r0[f] = fp.r1[f] = kr;
    }
    fp.rmax0 = fp.rmax1 = kr;
    fp.n_outputs = 3;
    float *outs[3] = {mag, sector, nullptr};
    const int64_t n = (int64_t)fp.H * fp.W;
    for (int k = 0; k < 3; ++k) {
        FamOutput &o = fp.outs[k];
        o.out = outs[k];
        o.plane_stride = n;
        o.row_pitch = fp.W;
        o.combine = (int)Combine::kLinear;
        o.fa = k < 2 ? k : -1;
        o.fb = -1;
        o.alpha = 1.0f;
    }
    fp.tensor = kTensorCannyGrad;
    if (lucem_status st = fam_waits(ws, &fp, stream)) return st;
    int e = timed(kPassFamily, stream, [&] { return launch_family_planes(fp, src->dtype, stream); });
    return e ? cuda_fail(e, "canny gradient launch") : ok();
}

}  // namespace

extern "C" {

void lucem_canny_settings_default(lucem_canny_settings *s) {
    s->sigma = 1.0;
    s->has_low = 0;
    s->low_threshold = 0.0;
    s->has_high = 0;
    s->high_threshold = 0.0;
    s->use_quantiles = 0;
    s->mode = LUCEM_PAD_REFLECT;
    s->cval = 0.0;
}

lucem_status lucem_canny(lucem_ctx *ctx, const lucem_tensor *in, const lucem_canny_settings *settings,
                         lucem_tensor *out, lucem_workspace *ws, void *stream) {
    TimerScope timer_scope(ws);
    if (!ctx) return fail(LUCEM_ERR_INVALID_HANDLE, "null context");
    if (!ws) return fail(LUCEM_ERR_INVALID_HANDLE, "a workspace is required");
    lucem_canny_settings def;
    lucem_canny_settings_default(&def);
    const lucem_canny_settings *s = settings ? settings : &def;
    lucem_status st;
    if ((st = check_tensor("image", in)) || (st = check_2d("canny", in))) return st;
    if (!std::isfinite(s->sigma) || s->sigma < 0.0)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `sigma`: sigma must be non-negative and finite, got %g", s->sigma);
    if ((st = check_mode(s->mode))) return st;
    // The output: a u32 edge map of the image's shape.
    if (!out) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `output`: null tensor");
    if (out->dtype != LUCEM_U32)
        return fail(LUCEM_ERR_UNSUPPORTED_DTYPE, "canny writes a u32 edge map, got element type %d", out->dtype);
    if ((st = same_shape("image", in, "output", out))) return st;
    const int64_t n = numel(in), H = in->dims[0], W = in->dims[1];
    if (n == 0) return ok();
    if (!out->data) return fail(LUCEM_ERR_INVALID_PARAMETER, "invalid parameter `output`: null data pointer");
    {
        const uintptr_t a0 = reinterpret_cast<uintptr_t>(in->data), a1 = a0 + (uintptr_t)n * dtype_size(in->dtype);
        const uintptr_t b0 = reinterpret_cast<uintptr_t>(out->data), b1 = b0 + (uintptr_t)n * 4u;
        if (a0 < b1 && b0 < a1)
            return fail(LUCEM_ERR_ALIASED_BUFFERS, "input and output arrays must not share the same device buffer");
    }
    if (H >= (1 << 30) || W >= (1 << 30))
        return fail(LUCEM_ERR_TOO_MANY_ELEMENTS, "canny: a side of 2^30 or more");
    void *pm = nullptr, *ps = nullptr, *pn = nullptr, *px = nullptr;
    if ((st = ws->get("canny_mag", (size_t)n * sizeof(float), &pm)) ||
        (st = ws->get("canny_sector", (size_t)n * sizeof(float), &ps)) ||
        (st = ws->get("canny_nms", (size_t)n * sizeof(float), &pn)) || (st = ws->get("canny_max", 64, &px)))
        return st;
    float *mag = static_cast<float *>(pm), *sector = static_cast<float *>(ps), *nms = static_cast<float *>(pn);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);

    // Gaussian pre-smoothing (truncate 4; sigma 0 leaves the image as it is),
    // then the Sobel stencils (gradient.rs:71-107).
    const double deriv[3] = {-1.0, 0.0, 1.0}, smooth[3] = {1.0, 2.0, 1.0};
    const int64_t r = s->sigma > 0.0 ? (int64_t)radius_of(4.0, s->sigma) : 0;
    std::vector<double> g((size_t)(2 * r + 1), 1.0);
    if (s->sigma > 0.0) gaussian_taps(s->sigma, 0, r, g.data());
    // For the reflect, mirror and wrap extensions, the smoothed image's
    // extension is the smoothing of the input's (a symmetric kernel on a
    // symmetric or periodic signal), so the stencils compose with the
    // Gaussian into one filter over the input.  The constant and nearest
    // extensions do not commute with the blur: those smooth first, as the
    // reference does.
    const bool compose = (s->mode == LUCEM_PAD_REFLECT || s->mode == LUCEM_PAD_MIRROR || s->mode == LUCEM_PAD_WRAP) &&
                         r + 1 <= kFamMaxRadius;
    if (compose) {
        const std::vector<double> gd = compose3(g, deriv), gs = compose3(g, smooth);
        st = canny_gradient_launch(in, s->mode, s->cval, gd, gs, gs, gd, (int)r + 1, mag, sector, ws, stream);
    } else {
        // The smoothed image goes through the nms slot (free until the
        // suppression writes it).
        std::vector<Pass> passes;
        if (s->sigma > 0.0) passes = {Pass{0, s->sigma, 0, r}, Pass{1, s->sigma, 0, r}};
        if ((st = run_passes(ctx, in, passes, s->mode, s->cval, 1.0, nms, ws, stream))) return st;
        lucem_tensor view = *in;
        view.data = nms;
        view.dtype = LUCEM_F32;
        const std::vector<double> d(deriv, deriv + 3), sm(smooth, smooth + 3);
        st = canny_gradient_launch(&view, s->mode, s->cval, d, sm, sm, d, 1, mag, sector, ws, stream);
    }
    if (st) return st;

    unsigned int *max_bits = static_cast<unsigned int *>(px);
    CUDA_TRY(cudaMemsetAsync(max_bits, 0, sizeof *max_bits, cs), "maximum reset");
    int e = timed(kPassElementwise, stream,
                  [&] { return launch_canny_nms(mag, sector, nms, (int)H, (int)W, max_bits, stream); });
    if (e) return cuda_fail(e, "non-maximum suppression launch");

    uint32_t *edges = static_cast<uint32_t *>(out->data);
    // The sector slot is free after the suppression: it holds the labels.
    uint32_t *labels = reinterpret_cast<uint32_t *>(sector);
    if (!s->has_low && !s->has_high) {
        // Both thresholds by default (canny.rs:108-116): high >= low always,
        // so they are computed on the device from the maximum, no host
        // round trip (the call stays asynchronous and capturable).
        double *thr = reinterpret_cast<double *>(static_cast<char *>(px) + 16);
        e = timed(kPassElementwise, stream, [&] {
            int r = launch_canny_thresholds(max_bits, s->use_quantiles ? 1 : 0, thr, stream);
            return r ? r : launch_canny_hysteresis(nms, (int)H, (int)W, thr, 0.0, 0.0, labels, edges, stream);
        });
        return e ? cuda_fail(e, "hysteresis launch") : ok();
    }
    // Thresholds (canny.rs:108-121); the maximum is needed unless both
    // thresholds are given as values.
    double max_mag = 0.0;
    if (!(s->has_low && s->has_high && !s->use_quantiles)) {
        unsigned int bits = 0;
        CUDA_TRY(cudaMemcpyAsync(&bits, max_bits, sizeof bits, cudaMemcpyDeviceToHost, cs), "maximum download");
        CUDA_TRY(cudaStreamSynchronize(cs), "synchronise");
        float m;
        std::memcpy(&m, &bits, sizeof m);
        max_mag = std::max((double)m, 0.0);
    }
    double low = s->has_low ? s->low_threshold : 0.1 * max_mag;
    double high = s->has_high ? s->high_threshold : 0.2 * max_mag;
    if (s->use_quantiles) {
        low *= max_mag;
        high *= max_mag;
    }
    if (high < low)
        return fail(LUCEM_ERR_INVALID_PARAMETER,
                    "invalid parameter `high_threshold`: high_threshold (%g) must be >= low_threshold (%g)", high,
                    low);
    // No strong pixel can exist unless high > 0; with low <= 0 nothing grows
    // from them, so the mask is the strong pixels themselves (the kernels
    // apply both rules).
    e = timed(kPassElementwise, stream, [&] {
        return launch_canny_hysteresis(nms, (int)H, (int)W, nullptr, low, high, labels, edges, stream);
    });
    return e ? cuda_fail(e, "hysteresis launch") : ok();
}

}  // extern "C"
