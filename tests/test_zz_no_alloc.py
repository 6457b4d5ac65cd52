"""lucem_gaussian_blur_noalloc, called through the C ABI: the blur for callers
that cannot allocate device memory (their memory comes from a pool under a
fixed budget, or they must not synchronise the device with cudaMalloc while
working).  Its intermediate buffers live in a static device array of the
library, so two calls in a row reuse the same memory; each must still match
lucem_gaussian_blur (the existing entry point) within the filters' 1e-5.

This file is collected last so that a failure here stops a `-x` run only
after every other test has run."""
import ctypes as C

import numpy as np
import pytest
import torch

import lucem_b200 as lb
from lucem_b200 import _native as N
from lucem_b200.ops import _tensor

pytestmark = pytest.mark.gpu

RTOL = 1e-5
MAX_ELEMS = 4 * 1024 * 1024


def noalloc_blur(x, sigmas, mode="reflect", axes=None):
    out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
    s = N.GaussianSettings()
    N.lib().lucem_gaussian_settings_default(C.byref(s))
    s.mode = lb.PadMode.parse(mode)
    keep = None
    if axes is not None:
        keep = (C.c_int64 * len(axes))(*axes)
        s.axes, s.n_axes = keep, len(axes)
    sig = (C.c_double * len(sigmas))(*sigmas)
    ti, to = _tensor(x, "input"), _tensor(out, "output")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.check(N.lib().lucem_gaussian_blur_noalloc(C.byref(ti), sig, len(sigmas), C.byref(s), C.byref(to), stream))
    return out


def test_two_calls_in_a_row_match_the_allocating_entry_point(oracle):
    rng = np.random.default_rng(21)
    # 3-D u16 volume: an axis-0 pass into the static scratch, then the fused 2-D pass.
    a = torch.from_numpy(rng.integers(0, 4000, (12, 150, 260)).astype(np.uint16)).cuda()
    # 2-D f32 image with a radius beyond the fused kernel: two passes through the scratch.
    b = torch.from_numpy(rng.standard_normal((300, 410)).astype(np.float32)).cuda()
    got_a = noalloc_blur(a, [1.5, 2.0, 2.5])
    got_b = noalloc_blur(b, [9.0], mode="mirror")
    want_a = lb.gaussian_blur(a, [1.5, 2.0, 2.5])
    want_b = lb.gaussian_blur(b, [9.0], mode="mirror")
    torch.cuda.synchronize()
    oracle.assert_close(got_a.cpu().numpy(), want_a.cpu().numpy().astype(np.float64), RTOL, "first call")
    oracle.assert_close(got_b.cpu().numpy(), want_b.cpu().numpy().astype(np.float64), RTOL, "second call")


def test_three_generic_passes_use_both_halves_of_the_scratch(oracle):
    """A radius beyond the fused 2-D kernel on every axis of a volume: three
    generic passes, input -> first half -> second half -> output."""
    rng = np.random.default_rng(23)
    x = torch.from_numpy(rng.standard_normal((40, 70, 90)).astype(np.float32)).cuda()
    for sig in ([9.0], [9.5, 10.0, 11.0]):
        got = noalloc_blur(x, sig, mode="wrap")
        want = lb.gaussian_blur(x, sig, mode="wrap")
        torch.cuda.synchronize()
        oracle.assert_close(got.cpu().numpy(), want.cpu().numpy().astype(np.float64), RTOL, f"sigma {sig}")


def test_repeated_calls_leave_device_memory_unchanged():
    """After one call of each kind (kernels loaded), further calls with new
    data take no device memory: free memory before and after is equal."""
    rng = np.random.default_rng(29)
    a = torch.from_numpy(rng.integers(0, 4000, (12, 150, 260)).astype(np.uint16)).cuda()
    b = torch.from_numpy(rng.standard_normal((300, 410)).astype(np.float32)).cuda()
    full = torch.ones((2, 1024, 2048), dtype=torch.float32, device="cuda")  # exactly the maximum
    calls = [(a, [1.5, 2.0, 2.5]), (b, [9.0]), (full, [1.0, 2.0, 2.0])]
    outs = [torch.empty(x.shape, dtype=torch.float32, device="cuda") for x, _ in calls]

    def run_all():
        for (x, sig), o in zip(calls, outs):
            s = N.GaussianSettings()
            N.lib().lucem_gaussian_settings_default(C.byref(s))
            arr = (C.c_double * len(sig))(*sig)
            ti, to = _tensor(x, "input"), _tensor(o, "output")
            stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            N.check(N.lib().lucem_gaussian_blur_noalloc(C.byref(ti), arr, len(sig), C.byref(s), C.byref(to), stream))

    a2 = torch.from_numpy(rng.integers(0, 4000, a.shape).astype(np.uint16)).cuda()
    b2 = torch.from_numpy(rng.standard_normal(b.shape).astype(np.float32)).cuda()
    run_all()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    a.copy_(a2)
    b.copy_(b2)
    for _ in range(3):
        run_all()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_sizes_beyond_the_static_scratch_are_refused():
    x = torch.zeros((MAX_ELEMS + 1,), dtype=torch.float32, device="cuda")
    with pytest.raises(N.LucemError) as e:
        noalloc_blur(x, [1.0])
    assert e.value.name == "TOO_MANY_ELEMENTS"
    ok = torch.ones((2, 1024, 2048), dtype=torch.float32, device="cuda")  # exactly the maximum
    out = noalloc_blur(ok, [1.0, 2.0, 2.0])
    torch.cuda.synchronize()
    assert torch.allclose(out, torch.ones_like(out), rtol=1e-5)
