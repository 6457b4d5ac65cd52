"""lucem-ops' Gaussian family and Richardson-Lucy on torch CUDA tensors.

Each function mirrors the reference function of the same name
(crates/lucem-ops/src/filter/gaussian.rs, filter/convolve.rs,
restore/deconvolve.rs): same parameters, defaults, argument checks and error
kinds (raised as LucemError, a ValueError carrying the lucem_status).  Arrays
are zero-copy device tensors; work is queued on the current torch stream.

Inputs may be float32, uint8 or uint16 (the cast to f32 is fused into the
kernels' load); outputs are float32.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _native as N
from ._native import LucemError

__all__ = [
    "LucemError", "PadMode", "Block", "context", "Workspace", "gaussian_kernel_1d", "gaussian_radius",
    "pad_index", "gaussian_blur", "gaussian_1d", "correlate_1d", "convolve_1d",
    "difference_of_gaussians", "gaussian_laplace", "gaussian_grad_mag", "unsharp_mask",
    "gaussian_family", "schedule", "gaussian_family_tiles", "richardson_lucy", "rl_grid",
    "gaussian_halo", "op_halo", "gaussian_blur_adjoint", "richardson_lucy_backward", "fft_convolve",
    "fft_convolve_backward", "RlBatch", "richardson_lucy_batch", "autotune_fft", "autotune_query",
    "autotune_save", "autotune_load", "autotune_enable", "autotune_plans", "Graph", "gaussian_batch", "fft_nd",
    "fft_1d", "complex_mul",
    "wiener_deconvolve", "from_dlpack", "fourier_gaussian", "fourier_box", "fourier_shift", "butterworth",
    "PhaseCorrelationResult", "phase_correlation", "unsupervised_wiener", "hessian_matrix", "hessian_det",
    "hessian_eigvals", "shape_index", "structure_tensor", "structure_tensor_eigvals", "frangi", "sato",
    "meijering", "Blob", "blobs_log", "blobs_dog", "blobs_doh", "pyramid_reduce", "pyramid_expand",
    "gaussian_pyramid", "laplacian_pyramid", "canny",
]


class PadMode:
    """crates/lucem-ops/src/core/pad.rs:15-68."""

    REFLECT, CONSTANT, NEAREST, MIRROR, WRAP = 0, 1, 2, 3, 4

    @staticmethod
    def parse(mode) -> int:
        if isinstance(mode, (int, np.integer)):
            return int(mode)
        out = C.c_int32()
        N.check(N.lib().lucem_pad_mode_parse(str(mode).encode(), C.byref(out)))
        return out.value


_DTYPES = {torch.float32: N.F32, torch.uint8: N.U8, torch.uint16: N.U16, torch.uint32: N.U32}

# ---------------------------------------------------------------------------
# Context / workspace


class _Ctx:
    def __init__(self, device: int):
        self.device = device
        h = C.c_void_p()
        N.check(N.lib().lucem_ctx_create(device, C.byref(h)))
        self.handle = h


_ctx_lock = threading.Lock()
_ctxs: dict = {}


def _device_index(device) -> int:
    if device is None:
        return torch.cuda.current_device()
    if isinstance(device, torch.device):
        return device.index if device.index is not None else torch.cuda.current_device()
    return int(device)


def context(device=None) -> _Ctx:
    """The library context of a CUDA device (created once per process)."""
    device = _device_index(device)
    with _ctx_lock:
        if device not in _ctxs:
            with torch.cuda.device(device):
                _ctxs[device] = _Ctx(device)
        return _ctxs[device]


class Workspace:
    """Grow-only device scratch (crates/lucem-core/src/memory/workspace.rs).
    One workspace serves one thread of work at a time."""

    def __init__(self, device=None):
        self.ctx = context(_device_index(device))
        h = C.c_void_p()
        N.check(N.lib().lucem_workspace_create(self.ctx.handle, C.byref(h)))
        self.handle = h

    @property
    def capacity_bytes(self) -> int:
        return int(N.lib().lucem_workspace_capacity_bytes(self.handle))

    def set_timing(self, enable: bool = True):
        """Bracket every kernel this workspace's calls launch with CUDA events
        (restarts the totals)."""
        N.check(N.lib().lucem_workspace_set_timing(self.handle, int(bool(enable))))

    def set_wait_limit(self, ns: int):
        """Bounded device waits of this workspace's calls: give up on a tensor
        copy after `ns` nanoseconds (0: at once; the default is one second)."""
        N.check(N.lib().lucem_workspace_set_wait_limit(self.handle, int(ns)))

    def wait_status(self, stream=None) -> int:
        """Synchronises the stream and returns (and clears) the number of
        device waits that gave up; raises LucemError DEVICE_TIMEOUT when it is
        not zero, with the count in the exception's `gave_up`."""
        st = stream if stream is not None else torch.cuda.current_stream()
        n = C.c_int64()
        rc = N.lib().lucem_workspace_wait_status(self.handle, C.c_void_p(st.cuda_stream), C.byref(n))
        if rc != 0:
            try:
                N.check(rc)
            except LucemError as e:
                e.gave_up = n.value
                raise
        return n.value

    def timings(self) -> dict:
        """{kernel kind: (launches, total device ms)} since timing was enabled;
        synchronises on the recorded events."""
        cap = 16
        names = C.create_string_buffer(32 * cap)
        ms = (C.c_double * cap)()
        cnt = (C.c_int64 * cap)()
        n = C.c_int32()
        N.check(N.lib().lucem_workspace_timings(self.handle, names, ms, cnt, cap, C.byref(n)))
        out = {}
        for i in range(min(n.value, cap)):
            name = names.raw[32 * i:32 * i + 32].split(b"\0", 1)[0].decode()
            out[name] = (int(cnt[i]), float(ms[i]))
        return out

    def close(self):
        if self.handle:
            N.lib().lucem_workspace_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


def _default_ws(device: int) -> Workspace:
    d = getattr(_tls, "ws", None)
    if d is None:
        d = _tls.ws = {}
    if device not in d:
        d[device] = Workspace(device)
    return d[device]


# ---------------------------------------------------------------------------
# helpers


def from_dlpack(obj) -> torch.Tensor:
    """A torch view of any DLPack producer (an object with __dlpack__: CuPy,
    JAX, NumPy, ...), zero-copy; torch tensors pass through.  Every operator
    here accepts such objects in place of tensors and returns torch tensors,
    which are DLPack producers themselves (``cupy.from_dlpack(out)``)."""
    if isinstance(obj, torch.Tensor):
        return obj
    if hasattr(obj, "__dlpack__"):
        return torch.from_dlpack(obj)
    raise TypeError(f"expected a torch.Tensor or a DLPack producer, got {type(obj).__name__}")


def _dlpack_args(fn):
    """Converts DLPack producers among the positional arguments and the
    `out` / `outs` keywords to torch views before calling `fn`."""
    import functools

    @functools.wraps(fn)
    def wrapped(*args, **kw):
        args = tuple(from_dlpack(a) if (not isinstance(a, torch.Tensor) and hasattr(a, "__dlpack__")) else a
                     for a in args)
        if kw.get("out") is not None:
            kw["out"] = from_dlpack(kw["out"])
        return fn(*args, **kw)

    return wrapped


def _tensor(t: torch.Tensor, name: str) -> N.Tensor:
    if not isinstance(t, torch.Tensor) and hasattr(t, "__dlpack__"):
        t = from_dlpack(t)
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor or a DLPack producer")
    if not t.is_cuda:
        raise LucemError(7, f"invalid parameter `{name}`: must be a CUDA tensor")
    if t.dtype not in _DTYPES:
        raise LucemError(13, f"{name}: unsupported element type {t.dtype}")
    if not t.is_contiguous():
        raise LucemError(7, f"invalid parameter `{name}`: must be C-contiguous")
    if t.dim() > N.MAX_DIMS:
        raise LucemError(3, f"{name} expects at most {N.MAX_DIMS}-D array, got {t.dim()}-D")
    d = N.Tensor()
    d.data = t.data_ptr() if t.numel() > 0 else None
    d.dtype = _DTYPES[t.dtype]
    d.ndim = t.dim()
    for i, s in enumerate(t.shape):
        d.dims[i] = int(s)
    return d


def _stream(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _out_like(x: torch.Tensor, out: Optional[torch.Tensor]) -> torch.Tensor:
    if out is None:
        return torch.empty(x.shape, dtype=torch.float32, device=x.device)
    return out


def _doubles(v) -> tuple:
    if np.isscalar(v):
        v = [v]
    v = [float(a) for a in v]
    return (C.c_double * max(1, len(v)))(*v), len(v)


def _ctx_ws(x: torch.Tensor, workspace: Optional[Workspace]):
    if not isinstance(x, torch.Tensor) or not x.is_cuda:
        raise LucemError(7, "invalid parameter `input`: must be a CUDA tensor (or a DLPack producer of device "
                            "memory)")
    dev = x.device.index if x.device.index is not None else torch.cuda.current_device()
    ctx = context(dev)
    ws = workspace if workspace is not None else _default_ws(dev)
    return ctx, ws


def _gaussian_settings(orders, mode, cval, truncate, radii, axes, channel_axis, input_scale, keep):
    s = N.GaussianSettings()
    N.lib().lucem_gaussian_settings_default(C.byref(s))
    if orders is not None:
        if np.isscalar(orders):
            orders = [orders]
        arr = (C.c_uint32 * len(orders))(*[int(o) for o in orders])
        keep.append(arr)
        s.orders = arr
        s.n_orders = len(orders)
    s.mode = PadMode.parse(mode)
    s.cval = float(cval)
    s.truncate = float(truncate)
    if radii is not None:
        if np.isscalar(radii):
            radii = [radii]
        arr = (C.c_int64 * len(radii))(*[int(r) for r in radii])
        keep.append(arr)
        s.radii = arr
        s.n_radii = len(radii)
    if axes is not None:
        arr = (C.c_int64 * max(1, len(axes)))(*[int(a) for a in axes])
        keep.append(arr)
        s.axes = arr
        s.n_axes = len(axes)
    if channel_axis is not None:
        s.has_channel_axis = 1
        s.channel_axis = int(channel_axis)
    s.input_scale = float(input_scale)
    return s


# ---------------------------------------------------------------------------
# host helpers


def gaussian_kernel_1d(sigma: float, order: int, radius: int) -> np.ndarray:
    """crates/lucem-ops/src/filter/gaussian.rs:22-63 (f64 taps)."""
    out = np.empty(2 * int(radius) + 1, np.float64)
    N.check(N.lib().lucem_gaussian_kernel_1d(float(sigma), int(order), int(radius),
                                             out.ctypes.data_as(C.POINTER(C.c_double))))
    return out


def gaussian_radius(sigma: float, truncate: float = 4.0) -> int:
    """crates/lucem-ops/src/filter/gaussian.rs:83-85."""
    return int(N.lib().lucem_gaussian_radius(float(truncate), float(sigma)))


def pad_index(p: int, n: int, mode="reflect") -> int:
    """crates/lucem-ops/src/core/kernels/pad.rs:11-34 (-1: constant fill)."""
    return int(N.lib().lucem_pad_index(int(p), int(n), PadMode.parse(mode)))


def gaussian_halo(ndim: int, sigmas, truncate: float = 4.0):
    """GaussianBlur::halo (crates/lucem-ops/src/filter/gaussian.rs:160-172)."""
    if np.isscalar(sigmas):
        sigmas = [sigmas]
    out = []
    for d in range(ndim):
        s = sigmas[d] if d < len(sigmas) else (sigmas[0] if sigmas else 0.0)
        r = gaussian_radius(s, truncate) if s > 0 else 0
        out.append((r, r))
    return out


def op_halo(op: str, sigma: float = 0.0, low_sigma: float = 0.0, high_sigma: float = 0.0) -> int:
    """Op::halo for the Gaussian ops (engine/lucem-pipeline/src/ops.rs:434-438):
    ceil(4 sigma)."""
    s = lambda v: int(np.ceil(4.0 * max(v, 0.0)))  # noqa: E731
    if op in ("gaussian_blur", "unsharp_mask"):
        return s(sigma)
    if op == "difference_of_gaussians":
        return s(max(low_sigma, high_sigma))
    raise ValueError(f"no halo rule for {op}")


# ---------------------------------------------------------------------------
# filters


@_dlpack_args
def gaussian_blur(x: torch.Tensor, sigmas, *, orders=None, mode="reflect", cval=0.0, truncate=4.0, radii=None,
                  axes=None, channel_axis=None, input_scale=1.0, out: Optional[torch.Tensor] = None,
                  workspace: Optional[Workspace] = None) -> torch.Tensor:
    """gaussian_blur / gaussian_blur_into (crates/lucem-ops/src/filter/gaussian.rs:176-250)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    keep = []
    s = _gaussian_settings(orders, mode, cval, truncate, radii, axes, channel_axis, input_scale, keep)
    sig, ns = _doubles(sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_gaussian_blur(ctx.handle, C.byref(ti), sig, ns, C.byref(s), C.byref(to), ws.handle,
                                        _stream(x)))
    return out


@_dlpack_args
def gaussian_blur_adjoint(g: torch.Tensor, sigmas, *, orders=None, mode="reflect", truncate=4.0, radii=None,
                          axes=None, channel_axis=None, input_scale=1.0, out: Optional[torch.Tensor] = None,
                          workspace: Optional[Workspace] = None) -> torch.Tensor:
    """The transpose of gaussian_blur's linear map with the same arguments,
    applied to `g` (f32): the input gradient of gaussian_blur given the output
    gradient.  No counterpart in the reference."""
    ctx, ws = _ctx_ws(g, workspace)
    out = _out_like(g, out)
    keep = []
    s = _gaussian_settings(orders, mode, 0.0, truncate, radii, axes, channel_axis, input_scale, keep)
    sig, ns = _doubles(sigmas)
    ti, to = _tensor(g, "grad_out"), _tensor(out, "grad_in")
    N.check(N.lib().lucem_gaussian_blur_adjoint(ctx.handle, C.byref(ti), sig, ns, C.byref(s), C.byref(to),
                                                ws.handle, _stream(g)))
    return out


@_dlpack_args
def gaussian_1d(x: torch.Tensor, sigma: float, *, axis=-1, order=0, mode="reflect", cval=0.0, truncate=4.0,
                radius=None, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """gaussian_1d / gaussian_1d_into (crates/lucem-ops/src/filter/gaussian.rs:66-130)."""
    ctx, _ = _ctx_ws(x, None)
    out = _out_like(x, out)
    s = N.Gaussian1dSettings()
    N.lib().lucem_gaussian_1d_settings_default(C.byref(s))
    s.axis, s.order, s.mode = int(axis), int(order), PadMode.parse(mode)
    s.cval, s.truncate = float(cval), float(truncate)
    s.radius = -1 if radius is None else int(radius)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_gaussian_1d(ctx.handle, C.byref(ti), float(sigma), C.byref(s), C.byref(to), _stream(x)))
    return out


@_dlpack_args
def correlate_1d(x: torch.Tensor, weights, *, axis=-1, mode="reflect", cval=0.0, origin=0,
                 out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """correlate_1d (crates/lucem-ops/src/filter/convolve.rs:40-92)."""
    ctx, _ = _ctx_ws(x, None)
    out = _out_like(x, out)
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
    s = N.Correlate1dSettings(int(axis), PadMode.parse(mode), float(cval), int(origin))
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    wp = w.ctypes.data_as(C.POINTER(C.c_double)) if w.size else None
    N.check(N.lib().lucem_correlate_1d(ctx.handle, C.byref(ti), wp, int(w.size), C.byref(s), C.byref(to),
                                       _stream(x)))
    return out


@_dlpack_args
def convolve_1d(x: torch.Tensor, weights, *, axis=-1, mode="reflect", cval=0.0, origin=0,
                out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """convolve_1d (crates/lucem-ops/src/filter/convolve.rs:95-109): correlation
    with reversed weights and the mirrored origin."""
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    size = w.size
    if size == 0:
        raise LucemError(6, "weights: filter weights cannot be empty")
    lo, hi = -(size // 2), (size - 1) // 2
    if not lo <= origin <= hi:
        raise LucemError(5, f"origin {origin} is out of bounds for window of size {size} (must be in {lo}..={hi})")
    mirrored = -int(origin) - (1 if size % 2 == 0 else 0)
    return correlate_1d(x, w[::-1].copy(), axis=axis, mode=mode, cval=cval, origin=mirrored, out=out)


@_dlpack_args
def difference_of_gaussians(x: torch.Tensor, low_sigmas, high_sigmas, *, mode="reflect", cval=0.0, truncate=4.0,
                            axes=None, channel_axis=None, input_scale=1.0, out: Optional[torch.Tensor] = None,
                            workspace: Optional[Workspace] = None) -> torch.Tensor:
    """difference_of_gaussians (crates/lucem-ops/src/filter/gaussian.rs:374-404)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    keep = []
    s = _gaussian_settings(None, mode, cval, truncate, None, axes, channel_axis, input_scale, keep)
    lo, nlo = _doubles(low_sigmas)
    hi, nhi = _doubles(high_sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_difference_of_gaussians(ctx.handle, C.byref(ti), lo, nlo, hi, nhi, C.byref(s),
                                                  C.byref(to), ws.handle, _stream(x)))
    return out


@_dlpack_args
def gaussian_laplace(x: torch.Tensor, sigmas, *, mode="reflect", cval=0.0, truncate=4.0,
                     out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """gaussian_laplace (crates/lucem-ops/src/filter/gaussian.rs:255-303)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    sig, ns = _doubles(sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_gaussian_laplace(ctx.handle, C.byref(ti), sig, ns, PadMode.parse(mode), float(cval),
                                           float(truncate), C.byref(to), ws.handle, _stream(x)))
    return out


@_dlpack_args
def gaussian_grad_mag(x: torch.Tensor, sigmas, *, mode="reflect", cval=0.0, truncate=4.0,
                      out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """gaussian_grad_mag (crates/lucem-ops/src/filter/gaussian.rs:307-371)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    sig, ns = _doubles(sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_gaussian_grad_mag(ctx.handle, C.byref(ti), sig, ns, PadMode.parse(mode), float(cval),
                                            float(truncate), C.byref(to), ws.handle, _stream(x)))
    return out


@_dlpack_args
def unsharp_mask(x: torch.Tensor, sigmas, amount: float, *, mode="reflect", cval=0.0, truncate=4.0, axes=None,
                 channel_axis=None, input_scale=1.0, out: Optional[torch.Tensor] = None,
                 workspace: Optional[Workspace] = None) -> torch.Tensor:
    """unsharp_mask (crates/lucem-ops/src/filter/gaussian.rs:407-435)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    keep = []
    s = _gaussian_settings(None, mode, cval, truncate, None, axes, channel_axis, input_scale, keep)
    sig, ns = _doubles(sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_unsharp_mask(ctx.handle, C.byref(ti), sig, ns, float(amount), C.byref(s), C.byref(to),
                                       ws.handle, _stream(x)))
    return out


_KINDS = {"gaussian": N.RESP_GAUSSIAN, "dog": N.RESP_DOG, "laplace": N.RESP_LAPLACE,
          "grad_mag": N.RESP_GRAD_MAG, "unsharp": N.RESP_UNSHARP}


def _responses(specs, outs):
    arr = (N.Response * max(1, len(specs)))()
    for i, (spec, o) in enumerate(zip(specs, outs)):
        kind = spec[0]
        r = arr[i]
        r.kind = _KINDS[kind]
        r.sigma = float(spec[1])
        if kind == "dog":
            r.sigma2 = float(spec[2])
        if kind == "unsharp":
            r.amount = float(spec[2])
        r.out = _tensor(o, "output")
    return arr


@_dlpack_args
def gaussian_family(x: torch.Tensor, responses: Sequence[tuple], *, mode="reflect", cval=0.0, truncate=4.0,
                    input_scale=1.0, outs: Optional[Sequence[torch.Tensor]] = None,
                    workspace: Optional[Workspace] = None):
    """Several Gaussian-family responses of one input over its last two axes in
    one fused pass.  `responses`: ("gaussian", s), ("dog", s_low, s_high),
    ("laplace", s), ("grad_mag", s), ("unsharp", s, amount).  Each equals the
    reference function of that name on `x`."""
    ctx, ws = _ctx_ws(x, workspace)
    if outs is None:
        outs = [torch.empty(x.shape, dtype=torch.float32, device=x.device) for _ in responses]
    arr = _responses(responses, outs)
    ti = _tensor(x, "input")
    N.check(N.lib().lucem_gaussian_family(ctx.handle, C.byref(ti), arr, len(responses), PadMode.parse(mode),
                                          float(cval), float(truncate), float(input_scale), ws.handle, _stream(x)))
    return list(outs)


# ---------------------------------------------------------------------------
# tiling / batched tiles


@dataclass(frozen=True)
class Block:
    """crates/lucem-core/src/tiling.rs:13-49 ([z, y, x])."""

    index: int
    origin: tuple
    size: tuple
    read_origin: tuple
    read_size: tuple

    def inner_offset(self):
        return tuple(self.origin[a] - self.read_origin[a] for a in range(3))

    def read_dims(self):
        return [self.read_size[1], self.read_size[2]] if self.read_size[0] == 1 else list(self.read_size)


def _blocks_c(blocks):
    arr = (N.Block * max(1, len(blocks)))()
    for i, b in enumerate(blocks):
        arr[i].index = b.index
        for a in range(3):
            arr[i].origin[a] = b.origin[a]
            arr[i].size[a] = b.size[a]
            arr[i].read_origin[a] = b.read_origin[a]
            arr[i].read_size[a] = b.read_size[a]
    return arr


def schedule(dims, block, halo):
    """crates/lucem-core/src/tiling.rs:54-78."""
    d = (C.c_int64 * 3)(*dims)
    b = (C.c_int64 * 3)(*block)
    h = (C.c_int64 * 3)(*halo)
    n = C.c_int64()
    N.check(N.lib().lucem_schedule(d, b, h, None, 0, C.byref(n)))
    arr = (N.Block * max(1, n.value))()
    N.check(N.lib().lucem_schedule(d, b, h, arr, n.value, C.byref(n)))
    return [Block(int(a.index), tuple(a.origin), tuple(a.size), tuple(a.read_origin), tuple(a.read_size))
            for a in arr[: n.value]]


class TileWalk:
    """A prepared batched walk: the block list marshalled once, so repeated calls
    (and CUDA-graph capture of them) do no host work beyond the launch."""

    def __init__(self, blocks):
        self.blocks = list(blocks)
        self._arr = _blocks_c(self.blocks)


def gaussian_family_tiles(slide: torch.Tensor, blocks, responses: Sequence[tuple], *, mode="reflect", cval=0.0,
                          truncate=4.0, input_scale=1.0, persistent=True,
                          outs: Optional[Sequence[torch.Tensor]] = None, workspace: Optional[Workspace] = None):
    """The tile walk of engine/lucem-pipeline/src/custom.rs:199-251 with a
    Gaussian-family function per block, over every channel of a [C, H, W] (or
    [H, W]) slide.  persistent=True: one persistent launch over the whole work
    list; False: one launch per block and channel (the plain drop-in)."""
    ctx, ws = _ctx_ws(slide, workspace)
    if outs is None:
        outs = [torch.empty(slide.shape, dtype=torch.float32, device=slide.device) for _ in responses]
    walk = blocks if isinstance(blocks, TileWalk) else TileWalk(blocks)
    arr = _responses(responses, outs)
    ts = _tensor(slide, "slide")
    N.check(N.lib().lucem_gaussian_family_tiles(ctx.handle, C.byref(ts), walk._arr, len(walk.blocks), arr,
                                                len(responses), PadMode.parse(mode), float(cval), float(truncate),
                                                float(input_scale), int(bool(persistent)), ws.handle,
                                                _stream(slide)))
    return list(outs)


# ---------------------------------------------------------------------------
# Richardson-Lucy


def rl_grid(dims, kdims, mode="reflect", grid=None):
    """The FFT grid richardson_lucy uses for these sizes."""
    nd = len(dims)
    d = (C.c_int64 * 3)(*dims)
    k = (C.c_int64 * 3)(*kdims)
    g = (C.c_int64 * 3)()
    req = (C.c_int64 * 3)(*(list(grid) if grid is not None else [0] * nd))
    N.check(N.lib().lucem_rl_grid(d, k, nd, PadMode.parse(mode), req, g))
    return tuple(int(v) for v in g[:nd])


def _rl_settings(num_iter, clip, filter_epsilon, mode, grid):
    s = N.RlSettings()
    N.lib().lucem_rl_settings_default(C.byref(s))
    s.num_iter = int(num_iter)
    s.clip = int(bool(clip))
    if filter_epsilon is not None:
        s.has_filter_epsilon = 1
        s.filter_epsilon = float(filter_epsilon)
    s.mode = PadMode.parse(mode)
    if grid is not None:
        for i, g in enumerate(grid):
            s.grid[i] = int(g)
    return s


def _grid_arg(grid):
    if grid is None:
        return None
    g = list(grid)
    return (C.c_int64 * 3)(*(g + [0] * (3 - len(g))))


@_dlpack_args
def richardson_lucy(x: torch.Tensor, psf: torch.Tensor, *, num_iter: int = 30, clip: bool = True,
                    filter_epsilon: Optional[float] = None, mode="reflect", grid=None,
                    out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """richardson_lucy (crates/lucem-ops/src/restore/deconvolve.rs:45-162) for
    2-D and 3-D inputs, on FFT convolution.  `grid` overrides the FFT lengths.
    `x` may carry one leading batch axis (one axis more than `psf`): the
    images or volumes share the PSF and run in the same launches."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    s = _rl_settings(num_iter, clip, filter_epsilon, mode, grid)
    ti, tp, to = _tensor(x, "input"), _tensor(psf, "psf"), _tensor(out, "output")
    N.check(N.lib().lucem_richardson_lucy(ctx.handle, C.byref(ti), C.byref(tp), C.byref(s), C.byref(to),
                                          ws.handle, _stream(x)))
    return out


def richardson_lucy_backward(x: torch.Tensor, psf: torch.Tensor, grad_out: torch.Tensor, *, num_iter: int = 30,
                             filter_epsilon: Optional[float] = None, grid=None, checkpoint_every: int = 5,
                             need_psf: bool = True, need_input: bool = True,
                             workspace: Optional[Workspace] = None):
    """(d loss / d psf, d loss / d x) of richardson_lucy(x, psf, clip=False,
    mode="constant", ...) given d loss / d (its output); either is None when
    not asked for.  The iterations are recomputed from checkpoints kept every
    `checkpoint_every` iterations.  With a leading batch axis on `x` the PSF
    gradient is summed over the batch.  No counterpart in the reference."""
    ctx, ws = _ctx_ws(x, workspace)
    s = _rl_settings(num_iter, False, filter_epsilon, "constant", grid)
    gp = torch.empty(psf.shape, dtype=torch.float32, device=x.device) if need_psf else None
    gx = torch.empty(x.shape, dtype=torch.float32, device=x.device) if need_input else None
    ti, tp, tg = _tensor(x, "input"), _tensor(psf, "psf"), _tensor(grad_out, "grad_out")
    tgp = C.byref(_tensor(gp, "grad_psf")) if gp is not None else None
    tgx = C.byref(_tensor(gx, "grad_in")) if gx is not None else None
    N.check(N.lib().lucem_richardson_lucy_backward(ctx.handle, C.byref(ti), C.byref(tp), C.byref(s), C.byref(tg),
                                                   int(checkpoint_every), tgp, tgx, ws.handle, _stream(x)))
    return gp, gx


@_dlpack_args
def fft_convolve(x: torch.Tensor, psf: torch.Tensor, *, grid=None, out: Optional[torch.Tensor] = None,
                 workspace: Optional[Workspace] = None) -> torch.Tensor:
    """The forward model of richardson_lucy (deconvolve.rs:120, correlation
    with the flipped PSF): convolution centred at k-1-k//2 per axis, zero
    padding, the PSF as given, on the FFT grid.  `x` may carry one leading
    batch axis (one PSF for the batch)."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    ti, tp, to = _tensor(x, "x"), _tensor(psf, "psf"), _tensor(out, "output")
    N.check(N.lib().lucem_fft_convolve(ctx.handle, C.byref(ti), C.byref(tp), PadMode.CONSTANT, _grid_arg(grid),
                                       C.byref(to), ws.handle, _stream(x)))
    return out


def fft_convolve_backward(x: torch.Tensor, psf: torch.Tensor, grad_out: torch.Tensor, *, grid=None,
                          need_psf: bool = True, need_input: bool = True,
                          workspace: Optional[Workspace] = None):
    """(grad_psf, grad_x) of fft_convolve."""
    ctx, ws = _ctx_ws(x, workspace)
    gp = torch.empty(psf.shape, dtype=torch.float32, device=x.device) if need_psf else None
    gx = torch.empty(x.shape, dtype=torch.float32, device=x.device) if need_input else None
    ti, tp, tg = _tensor(x, "x"), _tensor(psf, "psf"), _tensor(grad_out, "grad_out")
    tgp = C.byref(_tensor(gp, "grad_psf")) if gp is not None else None
    tgx = C.byref(_tensor(gx, "grad_x")) if gx is not None else None
    N.check(N.lib().lucem_fft_convolve_backward(ctx.handle, C.byref(ti), C.byref(tp), PadMode.CONSTANT,
                                                _grid_arg(grid), C.byref(tg), tgx, tgp, ws.handle, _stream(x)))
    return gp, gx


# ---------------------------------------------------------------------------
# Gaussian-consumer operators (crates/lucem-ops/src/feature/structure.rs,
# filter/ridge.rs): each scale's Hessian filters in one fused launch.


def _empty_f32(x, n):
    return [torch.empty(x.shape, dtype=torch.float32, device=x.device) for _ in range(n)]


def _hessian_call(fn, x, sigma, mode, cval, outs, workspace):
    ctx, ws = _ctx_ws(x, workspace)
    ts = [_tensor(o, "output") for o in outs]
    ti = _tensor(x, "input")
    N.check(fn(ctx.handle, C.byref(ti), float(sigma), PadMode.parse(mode), float(cval), *[C.byref(t) for t in ts],
               ws.handle, _stream(x)))
    return outs


@_dlpack_args
def hessian_matrix(x: torch.Tensor, sigma: float, mode="reflect", cval: float = 0.0, *,
                   workspace: Optional[Workspace] = None):
    """hessian_matrix (crates/lucem-ops/src/feature/structure.rs:16-54): the
    2-D Gaussian Hessian (H_rr, H_rc, H_cc) at scale sigma."""
    return tuple(_hessian_call(N.lib().lucem_hessian_matrix, x, sigma, mode, cval, _empty_f32(x, 3), workspace))


@_dlpack_args
def hessian_det(x: torch.Tensor, sigma: float, mode="reflect", cval: float = 0.0, *,
                workspace: Optional[Workspace] = None) -> torch.Tensor:
    """hessian_det (feature/structure.rs:57-83): H_rr H_cc - H_rc^2."""
    return _hessian_call(N.lib().lucem_hessian_det, x, sigma, mode, cval, _empty_f32(x, 1), workspace)[0]


@_dlpack_args
def hessian_eigvals(x: torch.Tensor, sigma: float, mode="reflect", cval: float = 0.0, *,
                    workspace: Optional[Workspace] = None):
    """hessian_eigvals (feature/structure.rs:86-97): (l1 >= l2)."""
    return tuple(_hessian_call(N.lib().lucem_hessian_eigvals, x, sigma, mode, cval, _empty_f32(x, 2), workspace))


@_dlpack_args
def shape_index(x: torch.Tensor, sigma: float, mode="reflect", cval: float = 0.0, *,
                workspace: Optional[Workspace] = None) -> torch.Tensor:
    """shape_index (feature/structure.rs:164-191): Koenderink's shape index in
    [-1, 1] from the Hessian eigenvalues."""
    return _hessian_call(N.lib().lucem_shape_index, x, sigma, mode, cval, _empty_f32(x, 1), workspace)[0]


@_dlpack_args
def structure_tensor(x: torch.Tensor, sigma: float, mode="reflect", cval: float = 0.0, *,
                     workspace: Optional[Workspace] = None):
    """structure_tensor (feature/structure.rs:102-147): (A_rr, A_rc, A_cc),
    the Gaussian-windowed outer products of the Sobel gradients."""
    return tuple(_hessian_call(N.lib().lucem_structure_tensor, x, sigma, mode, cval, _empty_f32(x, 3), workspace))


def structure_tensor_eigvals(arr, arc, acc):
    """structure_tensor_eigvals (feature/structure.rs:150-161): (l1 >= l2)."""
    arr, arc, acc = (from_dlpack(t) for t in (arr, arc, acc))
    e1, e2 = _empty_f32(arr, 2)
    ts = [_tensor(t, n) for t, n in ((arr, "arr"), (arc, "arc"), (acc, "acc"), (e1, "eig1"), (e2, "eig2"))]
    N.check(N.lib().lucem_structure_tensor_eigvals(*[C.byref(t) for t in ts], _stream(arr)))
    return e1, e2


def _ridge(fn, x, sigmas, black_ridges, mode, cval, beta, gamma, out, workspace):
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    s = N.RidgeSettings()
    N.lib().lucem_ridge_settings_default(C.byref(s))
    if sigmas is not None:
        arr, n = _doubles(sigmas)
        s.sigmas, s.n_sigmas = C.cast(arr, C.POINTER(C.c_double)), n
    s.black_ridges, s.mode, s.cval = int(bool(black_ridges)), PadMode.parse(mode), float(cval)
    s.beta, s.gamma = float(beta), float(gamma)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(fn(ctx.handle, C.byref(ti), C.byref(s), C.byref(to), ws.handle, _stream(x)))
    return out


@_dlpack_args
def frangi(x: torch.Tensor, sigmas=(1.0, 3.0, 5.0, 7.0, 9.0), *, black_ridges: bool = True, mode="reflect",
           cval: float = 0.0, beta: float = 0.5, gamma: float = 15.0, out: Optional[torch.Tensor] = None,
           workspace: Optional[Workspace] = None) -> torch.Tensor:
    """frangi (crates/lucem-ops/src/filter/ridge.rs:87-145): multi-scale
    vesselness, the maximum over the scales."""
    return _ridge(N.lib().lucem_frangi, x, sigmas, black_ridges, mode, cval, beta, gamma, out, workspace)


@_dlpack_args
def sato(x: torch.Tensor, sigmas=(1.0, 3.0, 5.0, 7.0, 9.0), *, black_ridges: bool = True, mode="reflect",
         cval: float = 0.0, out: Optional[torch.Tensor] = None,
         workspace: Optional[Workspace] = None) -> torch.Tensor:
    """sato (filter/ridge.rs:148-196): multi-scale tubeness."""
    return _ridge(N.lib().lucem_sato, x, sigmas, black_ridges, mode, cval, 0.5, 15.0, out, workspace)


@_dlpack_args
def meijering(x: torch.Tensor, sigmas=(1.0, 3.0, 5.0, 7.0, 9.0), *, black_ridges: bool = True, mode="reflect",
              cval: float = 0.0, out: Optional[torch.Tensor] = None,
              workspace: Optional[Workspace] = None) -> torch.Tensor:
    """meijering (filter/ridge.rs:199-245): multi-scale neuriteness."""
    return _ridge(N.lib().lucem_meijering, x, sigmas, black_ridges, mode, cval, 0.5, 15.0, out, workspace)


def _pyramid_settings(downscale, sigma, order, mode, cval):
    s = N.PyramidSettings()
    N.lib().lucem_pyramid_settings_default(C.byref(s))
    s.downscale = float(downscale)
    s.sigma = -1.0 if sigma is None else float(sigma)
    s.order, s.mode, s.cval = int(order), PadMode.parse(mode), float(cval)
    return s


def pyramid_reduce(x, *, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0,
                   workspace: Optional[Workspace] = None) -> torch.Tensor:
    """pyramid_reduce (crates/lucem-ops/src/transform/pyramid.rs:135-168): the
    Gaussian blur (sigma default 2 downscale / 6), then the resize to
    ceil(H / downscale) x ceil(W / downscale) (orders 0 and 1)."""
    x = from_dlpack(x)
    ctx, ws = _ctx_ws(x, workspace)
    if x.dim() != 2:
        raise LucemError(3, f"pyramid_reduce expects 2-D array, got {x.dim()}-D")
    oh = max(1, math.ceil(x.shape[0] / float(downscale))) if downscale > 1 else 1
    ow = max(1, math.ceil(x.shape[1] / float(downscale))) if downscale > 1 else 1
    out = torch.empty((oh, ow), dtype=torch.float32, device=x.device)
    s = _pyramid_settings(downscale, sigma, order, mode, cval)
    ti, to = _tensor(x, "image"), _tensor(out, "output")
    N.check(N.lib().lucem_pyramid_reduce(ctx.handle, C.byref(ti), C.byref(s), C.byref(to), ws.handle, _stream(x)))
    return out


def pyramid_expand(x, output_shape=None, *, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0,
                   workspace: Optional[Workspace] = None) -> torch.Tensor:
    """pyramid_expand (transform/pyramid.rs:171-208): the resize up (to
    output_shape, default ceil(H downscale) x ceil(W downscale)), then the
    Gaussian blur."""
    x = from_dlpack(x)
    ctx, ws = _ctx_ws(x, workspace)
    if output_shape is None:
        output_shape = (max(1, math.ceil(x.shape[0] * float(downscale))),
                        max(1, math.ceil(x.shape[1] * float(downscale))))
    out = torch.empty(tuple(output_shape), dtype=torch.float32, device=x.device)
    s = _pyramid_settings(downscale, sigma, order, mode, cval)
    ti, to = _tensor(x, "image"), _tensor(out, "output")
    N.check(N.lib().lucem_pyramid_expand(ctx.handle, C.byref(ti), C.byref(s), C.byref(to), ws.handle, _stream(x)))
    return out


def gaussian_pyramid(x, max_layer: int, *, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0,
                     workspace: Optional[Workspace] = None):
    """gaussian_pyramid (transform/pyramid.rs:211-236): [level_0 (a copy),
    level_1, ...], at most max_layer reductions, stopping when a level is
    1 x 1 or stops shrinking."""
    x = from_dlpack(x)
    if x.dim() != 2:
        raise LucemError(3, f"gaussian_pyramid expects 2-D array, got {x.dim()}-D")
    _pyramid_settings(downscale, sigma, order, mode, cval)
    if not (math.isfinite(downscale) and downscale > 1.0):
        raise LucemError(7, f"invalid parameter `downscale`: pyramid scale factor must be > 1.0, got {downscale}")
    levels = [gaussian_blur(x, [0.0, 0.0], workspace=workspace)]
    for _ in range(int(max_layer)):
        cur = levels[-1]
        if cur.shape[0] <= 1 and cur.shape[1] <= 1:
            break
        nxt = pyramid_reduce(cur, downscale=downscale, sigma=sigma, order=order, mode=mode, cval=cval,
                             workspace=workspace)
        done = tuple(nxt.shape) == tuple(cur.shape)
        levels.append(nxt)
        if done:
            break
    return levels


def laplacian_pyramid(x, max_layer: int, *, downscale=2.0, sigma=None, order=1, mode="reflect", cval=0.0,
                      workspace: Optional[Workspace] = None):
    """laplacian_pyramid (transform/pyramid.rs:239-266): [L_0, ..., L_{N-1},
    G_N], L_k = G_k - expand(G_{k+1}) to G_k's shape."""
    g = gaussian_pyramid(x, max_layer, downscale=downscale, sigma=sigma, order=order, mode=mode, cval=cval,
                         workspace=workspace)
    if len(g) <= 1:
        return g
    ctx, ws = _ctx_ws(g[0], workspace)
    s = _pyramid_settings(downscale, sigma, order, mode, cval)
    bands = []
    for fine, coarse in zip(g[:-1], g[1:]):
        out = torch.empty_like(fine)
        tf, tc, to = _tensor(fine, "fine"), _tensor(coarse, "coarse"), _tensor(out, "output")
        N.check(N.lib().lucem_laplacian_band(ctx.handle, C.byref(tf), C.byref(tc), C.byref(s), C.byref(to),
                                             ws.handle, _stream(fine)))
        bands.append(out)
    return bands + [g[-1]]


@dataclass
class Blob:
    """crates/lucem-ops/src/feature/blobs.rs:16-30."""

    y: int
    x: int
    sigma: float
    response: float

    def radius(self) -> float:
        return math.sqrt(2.0) * self.sigma


def _blobs(fn, x, min_sigma, max_sigma, num_sigma, sigma_ratio, threshold, overlap, log_scale, exclude_border,
           workspace):
    x = from_dlpack(x)
    ctx, ws = _ctx_ws(x, workspace)
    s = N.BlobSettings()
    N.lib().lucem_blob_settings_default(C.byref(s))
    s.min_sigma, s.max_sigma, s.num_sigma = float(min_sigma), float(max_sigma), int(num_sigma)
    s.sigma_ratio, s.threshold, s.overlap = float(sigma_ratio), float(threshold), float(overlap)
    s.log_scale, s.exclude_border = int(bool(log_scale)), int(exclude_border)
    ti = _tensor(x, "image")
    cap = 4096
    while True:
        buf = (N.BlobC * cap)()
        n = C.c_int64()
        N.check(fn(ctx.handle, C.byref(ti), C.byref(s), buf, cap, C.byref(n), ws.handle, _stream(x)))
        if n.value <= cap:
            return [Blob(int(b.y), int(b.x), float(b.sigma), float(b.response)) for b in buf[: n.value]]
        cap = n.value


def blobs_log(x, *, min_sigma=1.0, max_sigma=30.0, num_sigma=10, threshold=0.1, overlap=0.5, log_scale=False,
              exclude_border=1, workspace: Optional[Workspace] = None):
    """blobs_log (crates/lucem-ops/src/feature/blobs.rs:204-236): scale-normalised
    LoG blobs, strongest first."""
    return _blobs(N.lib().lucem_blobs_log, x, min_sigma, max_sigma, num_sigma, 1.6, threshold, overlap, log_scale,
                  exclude_border, workspace)


def blobs_dog(x, *, min_sigma=1.0, max_sigma=30.0, sigma_ratio=1.6, threshold=0.1, overlap=0.5, exclude_border=1,
              workspace: Optional[Workspace] = None):
    """blobs_dog (feature/blobs.rs:238-287): difference-of-Gaussians blobs."""
    return _blobs(N.lib().lucem_blobs_dog, x, min_sigma, max_sigma, 10, sigma_ratio, threshold, overlap, False,
                  exclude_border, workspace)


def blobs_doh(x, *, min_sigma=1.0, max_sigma=30.0, num_sigma=10, threshold=0.1, overlap=0.5, log_scale=False,
              exclude_border=1, workspace: Optional[Workspace] = None):
    """blobs_doh (feature/blobs.rs:289-345): determinant-of-Hessian blobs."""
    return _blobs(N.lib().lucem_blobs_doh, x, min_sigma, max_sigma, num_sigma, 1.6, threshold, overlap, log_scale,
                  exclude_border, workspace)


@_dlpack_args
def canny(x: torch.Tensor, sigma: float = 1.0, low_threshold: Optional[float] = None,
          high_threshold: Optional[float] = None, use_quantiles: bool = False, mode="reflect", cval: float = 0.0, *,
          out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """canny (crates/lucem-ops/src/feature/canny.rs:47-165): Gaussian
    smoothing, Sobel gradients, non-maximum suppression along the quantised
    direction and 8-connected hysteresis; a u32 edge map (1 on edges).
    Thresholds default to 0.1 / 0.2 of the maximum gradient magnitude; with
    use_quantiles they are fractions of it."""
    ctx, ws = _ctx_ws(x, workspace)
    if out is None:
        out = torch.empty(x.shape, dtype=torch.uint32, device=x.device)
    s = N.CannySettings()
    N.lib().lucem_canny_settings_default(C.byref(s))
    s.sigma = float(sigma)
    if low_threshold is not None:
        s.has_low, s.low_threshold = 1, float(low_threshold)
    if high_threshold is not None:
        s.has_high, s.high_threshold = 1, float(high_threshold)
    s.use_quantiles = int(bool(use_quantiles))
    s.mode, s.cval = PadMode.parse(mode), float(cval)
    ti, to = _tensor(x, "image"), _tensor(out, "output")
    N.check(N.lib().lucem_canny(ctx.handle, C.byref(ti), C.byref(s), C.byref(to), ws.handle, _stream(x)))
    return out


# ---------------------------------------------------------------------------
# spectral operators (crates/lucem-ops/src/core/fft.rs, restore/deconvolve.rs)


def _zeros_like_f32(t):
    return torch.zeros(t.shape, dtype=torch.float32, device=t.device)


def fft_nd(re: torch.Tensor, im: Optional[torch.Tensor] = None, *, inverse: bool = False,
           workspace: Optional[Workspace] = None):
    """fft_nd_into (crates/lucem-ops/src/core/fft.rs:55-100): the N-D DFT of
    the split complex f32 array (re, im) over every axis, forward
    unnormalised, inverse scaled by 1/len per axis.  Returns (re, im)."""
    re = from_dlpack(re)
    im = _zeros_like_f32(re) if im is None else from_dlpack(im)
    ctx, ws = _ctx_ws(re, workspace)
    ore, oim = torch.empty_like(re), torch.empty_like(re)
    a, b, c, d = _tensor(re, "re_in"), _tensor(im, "im_in"), _tensor(ore, "re_out"), _tensor(oim, "im_out")
    N.check(N.lib().lucem_fft_nd(ctx.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d), int(bool(inverse)),
                                 ws.handle, _stream(re)))
    return ore, oim


def fft_1d(re: torch.Tensor, im: Optional[torch.Tensor] = None, *, axis: int = -1, inverse: bool = False,
           workspace: Optional[Workspace] = None):
    """fft_1d_into (crates/lucem-ops/src/core/fft.rs:14-53): the DFT along one
    axis of the split complex f32 array (re, im).  Returns (re, im)."""
    re = from_dlpack(re)
    im = _zeros_like_f32(re) if im is None else from_dlpack(im)
    ctx, ws = _ctx_ws(re, workspace)
    ore, oim = torch.empty_like(re), torch.empty_like(re)
    a, b, c, d = _tensor(re, "re_in"), _tensor(im, "im_in"), _tensor(ore, "re_out"), _tensor(oim, "im_out")
    N.check(N.lib().lucem_fft_1d(ctx.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d), int(axis),
                                 int(bool(inverse)), ws.handle, _stream(re)))
    return ore, oim


def complex_mul(a_re, a_im, b_re, b_im, *, conj_b: bool = False):
    """complex_mul_into (crates/lucem-ops/src/core/fft.rs:104-138): (a_re +
    i a_im) (b_re + i b_im), or times conj(b).  Returns (re, im)."""
    a_re, a_im, b_re, b_im = (from_dlpack(t) for t in (a_re, a_im, b_re, b_im))
    ore, oim = torch.empty_like(a_re), torch.empty_like(a_re)
    ts = [_tensor(t, n) for t, n in ((a_re, "a_re"), (a_im, "a_im"), (b_re, "b_re"), (b_im, "b_im"),
                                     (ore, "out_re"), (oim, "out_im"))]
    N.check(N.lib().lucem_complex_mul(*[C.byref(t) for t in ts], int(bool(conj_b)), _stream(a_re)))
    return ore, oim


@_dlpack_args
def wiener_deconvolve(x: torch.Tensor, psf: torch.Tensor, *, balance: float = 0.1, clip: bool = True,
                      out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """wiener_deconvolve (crates/lucem-ops/src/restore/deconvolve.rs:210-309):
    regularised frequency-domain Wiener deconvolution of a 2-D f32 image,
    X = conj(H) Y / max(|H|^2 + balance |L|^2, 1e-12), on the FFTs of fft_nd."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    s = N.WienerSettings()
    N.lib().lucem_wiener_settings_default(C.byref(s))
    s.balance = float(balance)
    s.clip = int(bool(clip))
    ti, tp, to = _tensor(x, "input"), _tensor(psf, "psf"), _tensor(out, "output")
    N.check(N.lib().lucem_wiener_deconvolve(ctx.handle, C.byref(ti), C.byref(tp), C.byref(s), C.byref(to),
                                            ws.handle, _stream(x)))
    return out


def _spectral_filter(fn, re, im, vals):
    re, im = from_dlpack(re), from_dlpack(im)
    ctx, _ = _ctx_ws(re, None)
    arr, n = _doubles(vals)
    a, b = _tensor(re, "re"), _tensor(im, "im")
    N.check(fn(ctx.handle, C.byref(a), C.byref(b), arr, n, _stream(re)))
    return re, im


def fourier_gaussian(re, im, sigmas):
    """fourier_gaussian_into (crates/lucem-ops/src/filter/spectral.rs:21-63):
    the split complex spectrum (re, im) times exp(-2 pi^2 sigma^2 f^2) per
    axis, in place.  Returns (re, im)."""
    return _spectral_filter(N.lib().lucem_fourier_gaussian, re, im, sigmas)


def fourier_box(re, im, sizes):
    """fourier_box_into (filter/spectral.rs:66-108): times sinc(pi size f)
    per axis, in place.  Returns (re, im)."""
    return _spectral_filter(N.lib().lucem_fourier_box, re, im, sizes)


def fourier_shift(re, im, shifts):
    """fourier_shift_into (filter/spectral.rs:112-164): times
    exp(-i 2 pi shift f) per axis, in place.  Returns (re, im)."""
    return _spectral_filter(N.lib().lucem_fourier_shift, re, im, shifts)


@_dlpack_args
def butterworth(x: torch.Tensor, cutoff_ratio: float, high_pass: bool = False, order: float = 2.0, *,
                out: Optional[torch.Tensor] = None, workspace: Optional[Workspace] = None) -> torch.Tensor:
    """butterworth (crates/lucem-ops/src/filter/spectral.rs:168-213): N-D
    frequency-domain Butterworth low-pass (or high-pass) filter of an f32
    array, cutoff_ratio in (0, 0.5]."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    N.check(N.lib().lucem_butterworth(ctx.handle, C.byref(ti), float(cutoff_ratio), int(bool(high_pass)),
                                      float(order), C.byref(to), ws.handle, _stream(x)))
    return out


@dataclass
class PhaseCorrelationResult:
    """crates/lucem-ops/src/register/phase.rs:39-48."""

    shift: list
    error: float
    phasediff: float


@_dlpack_args
def phase_correlation(reference: torch.Tensor, moving: torch.Tensor, *, upsample_factor: int = 1,
                      normalize_phase: bool = True,
                      workspace: Optional[Workspace] = None) -> PhaseCorrelationResult:
    """phase_correlation (crates/lucem-ops/src/register/phase.rs:51-255): the
    N-D shift registering `moving` onto `reference` (1 / upsample_factor
    pixel precision), its normalised RMS error and the global phase
    difference.  Synchronises (the result is host data)."""
    ctx, ws = _ctx_ws(reference, workspace)
    s = N.PhaseCorrelationSettings()
    N.lib().lucem_phase_correlation_settings_default(C.byref(s))
    s.upsample_factor = int(upsample_factor)
    s.normalize_phase = int(bool(normalize_phase))
    r = N.PhaseCorrelationResult()
    a, b = _tensor(reference, "reference"), _tensor(moving, "moving")
    N.check(N.lib().lucem_phase_correlation(ctx.handle, C.byref(a), C.byref(b), C.byref(s), C.byref(r),
                                            ws.handle, _stream(reference)))
    return PhaseCorrelationResult([float(r.shift[d]) for d in range(reference.dim())], float(r.error),
                                  float(r.phasediff))


@_dlpack_args
def unsupervised_wiener(x: torch.Tensor, psf: torch.Tensor, *, num_iter: int = 30, burnin: int = 10,
                        clip: bool = True, seed: int = 0, out: Optional[torch.Tensor] = None,
                        workspace: Optional[Workspace] = None):
    """unsupervised_wiener (crates/lucem-ops/src/restore/deconvolve.rs:357-509):
    Wiener deconvolution of a 2-D f32 image with the regularisation balance
    estimated by the reference's empirical-Bayes chain.  Returns
    (deconvolved, balance_chain); synchronises to return the chain."""
    ctx, ws = _ctx_ws(x, workspace)
    out = _out_like(x, out)
    s = N.UnsupervisedWienerSettings()
    N.lib().lucem_unsupervised_wiener_settings_default(C.byref(s))
    s.num_iter, s.burnin, s.clip, s.seed = int(num_iter), int(burnin), int(bool(clip)), int(seed) & (2 ** 64 - 1)
    chain = (C.c_double * max(1, int(num_iter)))()
    ti, tp, to = _tensor(x, "input"), _tensor(psf, "psf"), _tensor(out, "output")
    N.check(N.lib().lucem_unsupervised_wiener(ctx.handle, C.byref(ti), C.byref(tp), C.byref(s), C.byref(to), chain,
                                              ws.handle, _stream(x)))
    n = int(num_iter) if x.numel() else 0
    return out, [float(chain[i]) for i in range(n)]


# ---------------------------------------------------------------------------
# batched 2-D Richardson-Lucy, autotuning, graphs


def _tensor_array(ts, name):
    arr = (N.Tensor * len(ts))()
    for i, t in enumerate(ts):
        arr[i] = _tensor(t, f"{name}[{i}]")
    return arr


class RlBatch:
    """A planned batch of 2-D Richardson-Lucy problems of any sizes and PSFs
    (lucem_rl_batch_*).  The plan keeps the tensors' device pointers: keep
    `images`, `psfs` and `outs` alive while it is used.  run() only launches
    (one launch per pass and length group), so it can be captured in a CUDA
    graph; run(per_problem=True) runs the same kernels image by image."""

    def __init__(self, images: Sequence[torch.Tensor], psfs: Sequence[torch.Tensor], *, num_iter: int = 30,
                 clip: bool = True, filter_epsilon: Optional[float] = None, mode="reflect",
                 outs: Optional[Sequence[torch.Tensor]] = None, workspace: Optional[Workspace] = None):
        if len(images) == 0 or len(images) != len(psfs):
            raise LucemError(7, "invalid parameter `images`: one PSF per image, at least one image")
        x0 = images[0]
        ctx, ws = _ctx_ws(x0, workspace)
        self.images, self.psfs = list(images), list(psfs)
        self.outs = list(outs) if outs is not None else [torch.empty(x.shape, dtype=torch.float32, device=x.device)
                                                        for x in images]
        s = _rl_settings(num_iter, clip, filter_epsilon, mode, None)
        ti = _tensor_array(self.images, "images")
        tp = _tensor_array(self.psfs, "psfs")
        to = _tensor_array(self.outs, "outs")
        h = C.c_void_p()
        N.check(N.lib().lucem_rl_batch_create(ctx.handle, len(images), ti, tp, C.byref(s), to, ws.handle,
                                              _stream(x0), C.byref(h)))
        self.handle = h
        self.device = x0.device

    def run(self, per_problem: bool = False, workspace: Optional[Workspace] = None):
        ws = workspace.handle if workspace is not None else None
        N.check(N.lib().lucem_rl_batch_run(self.handle, int(bool(per_problem)), ws,
                                           C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
        return self.outs

    def info(self):
        """(grids [(Py, Px)], launches per row pass, launches per column pass)."""
        n = len(self.images)
        g = (C.c_int64 * (2 * n))()
        nr, nc = C.c_int32(), C.c_int32()
        N.check(N.lib().lucem_rl_batch_info(self.handle, g, C.byref(nr), C.byref(nc)))
        return [(int(g[2 * i]), int(g[2 * i + 1])) for i in range(n)], nr.value, nc.value

    def close(self):
        if getattr(self, "handle", None):
            N.lib().lucem_rl_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def richardson_lucy_batch(images: Sequence[torch.Tensor], psfs: Sequence[torch.Tensor], **kw):
    """richardson_lucy over a list of 2-D images of any sizes, one PSF each,
    as one planned batch; returns the list of estimates."""
    b = RlBatch(images, psfs, **kw)
    try:
        return b.run()
    finally:
        torch.cuda.current_stream(b.device).synchronize()
        b.close()


def autotune_fft(lengths, device=None, workspace: Optional[Workspace] = None):
    """Measure the FFT pass costs at `lengths` (lucem_autotune_fft); batched
    plans made afterwards on this device choose grids by them."""
    dev = _device_index(device)
    ctx = context(dev)
    ws = workspace if workspace is not None else _default_ws(dev)
    arr = (C.c_int64 * max(1, len(lengths)))(*[int(v) for v in lengths])
    N.check(N.lib().lucem_autotune_fft(ctx.handle, arr, len(lengths), ws.handle,
                                       C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))


def autotune_query(kind: int, length: int, device=None) -> float:
    """ns per transformed element of the column (kind 0) or row (kind 1) pass."""
    v = C.c_double()
    N.check(N.lib().lucem_autotune_query(context(_device_index(device)).handle, int(kind), int(length), C.byref(v)))
    return v.value


def autotune_save(path: str, device=None):
    N.check(N.lib().lucem_autotune_save(context(_device_index(device)).handle, str(path).encode()))


def autotune_enable(enable: bool = True, device=None):
    """lucem_autotune_enable: while on, the first plain 2-D blur or persistent
    tile walk of each size class times its launch candidates and caches the
    fastest (saved / loaded with autotune_save / autotune_load)."""
    N.check(N.lib().lucem_autotune_enable(context(_device_index(device)).handle, int(bool(enable))))


def autotune_plans(device=None) -> dict:
    """The cached launch plans: {key: code}, code = 1 + bits (1 copy ahead,
    2 one CTA per SM)."""
    h = context(_device_index(device)).handle
    n = C.c_int32()
    N.check(N.lib().lucem_autotune_plans(h, None, None, 0, C.byref(n)))
    cap = max(1, n.value)
    keys = C.create_string_buffer(64 * cap)
    codes = (C.c_int32 * cap)()
    N.check(N.lib().lucem_autotune_plans(h, keys, codes, cap, C.byref(n)))
    return {keys.raw[64 * i:64 * (i + 1)].split(b"\0", 1)[0].decode(): int(codes[i]) for i in range(min(n.value, cap))}


def autotune_load(path: str, device=None):
    N.check(N.lib().lucem_autotune_load(context(_device_index(device)).handle, str(path).encode()))


class Graph:
    """A CUDA graph of launch-only library calls (lucem_graph_*):

        g = Graph(stream); with g: plan.run(); ...; g.launch()
    """

    def __init__(self, stream: Optional[torch.cuda.Stream] = None):
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.handle = None

    def __enter__(self):
        self._ctx = torch.cuda.stream(self.stream)
        self._ctx.__enter__()
        N.check(N.lib().lucem_graph_begin(C.c_void_p(self.stream.cuda_stream)))
        return self

    def __exit__(self, exc_type, exc, tb):
        h = C.c_void_p()
        st = N.lib().lucem_graph_end(C.c_void_p(self.stream.cuda_stream), C.byref(h))
        self._ctx.__exit__(exc_type, exc, tb)
        if exc_type is None:
            N.check(st)
            self.handle = h
        elif h:
            N.lib().lucem_graph_destroy(h)
        return False

    def launch(self, stream: Optional[torch.cuda.Stream] = None):
        s = stream if stream is not None else torch.cuda.current_stream()
        N.check(N.lib().lucem_graph_launch(self.handle, C.c_void_p(s.cuda_stream)))

    def close(self):
        if self.handle:
            N.lib().lucem_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gaussian_batch(images: Sequence[torch.Tensor], sigmas, *, mode="reflect", cval=0.0, truncate=4.0,
                   input_scale=1.0, outs: Optional[Sequence[torch.Tensor]] = None,
                   workspace: Optional[Workspace] = None):
    """gaussian_blur of each 2-D image with its own isotropic sigma
    (`sigmas`: one per image, or one for all) in one launch per distinct sigma
    (lucem_gaussian_batch); returns the list of f32 outputs."""
    images = list(images)
    if len(images) == 0:
        return []
    if np.isscalar(sigmas):
        sigmas = [sigmas] * len(images)
    sigmas = [float(v) for v in sigmas]
    if len(sigmas) != len(images):
        raise LucemError(7, "invalid parameter `sigmas`: one per image")
    uniq = sorted(set(sigmas))
    ids = (C.c_int32 * len(images))(*[uniq.index(v) for v in sigmas])
    sets = (C.c_double * len(uniq))(*uniq)
    ctx, ws = _ctx_ws(images[0], workspace)
    outs = list(outs) if outs is not None else [torch.empty(x.shape, dtype=torch.float32, device=x.device)
                                                for x in images]
    ti = _tensor_array(images, "images")
    to = _tensor_array(outs, "outs")
    N.check(N.lib().lucem_gaussian_batch(ctx.handle, len(images), ti, to, ids, len(uniq), sets, PadMode.parse(mode),
                                         float(cval), float(truncate), float(input_scale), ws.handle,
                                         _stream(images[0])))
    return outs
