"""The C-ABI library: it loads without a GPU, exports every function
include/lucem_b200.h declares, and its host-only helpers and argument checks
behave as the reference's.  CPU only (no device work is started)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from lucem_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "lucem_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lucem_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = N.lib()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)
    assert lib.lucem_abi_version() == 1


def test_taps_radius_and_pad_index_match_the_oracle(oracle):
    import lucem_b200 as lb

    for sigma, order, radius in ((2.0, 0, 8), (1.0, 1, 4), (3.0, 2, 12), (0.7, 3, 3), (2.5, 5, 10), (1.0, 0, 0)):
        np.testing.assert_array_equal(lb.gaussian_kernel_1d(sigma, order, radius),
                                      oracle.gaussian_kernel_1d(sigma, order, radius))
    for s in (0.0, 0.3, 1.0, 2.0, 3.0, 4.0, 2.125):
        assert lb.gaussian_radius(s) == oracle.resolved_radius(4.0, s)
    for n in (1, 2, 7):
        for p in range(-20, 25):
            for m in range(5):
                assert lb.pad_index(p, n, m) == oracle.pad_index(p, n, m)


def test_pad_mode_names():
    """crates/lucem-ops/src/core/pad.rs:128-138."""
    from lucem_b200.ops import PadMode

    assert PadMode.parse("reflect") == 0
    assert PadMode.parse("grid-mirror") == 0
    assert PadMode.parse(" Constant ") == 1
    assert PadMode.parse("edge") == 2
    assert PadMode.parse("mirror") == 3
    assert PadMode.parse("periodic") == 4
    with pytest.raises(N.LucemError) as e:
        PadMode.parse("invalid")
    assert e.value.name == "UNKNOWN_PAD_MODE"


def test_schedule_covers_the_image_exactly_once():
    """crates/lucem-core/src/tiling.rs:101-131."""
    import lucem_b200 as lb

    dims = (5, 70, 130)
    blocks = lb.schedule(dims, (2, 32, 64), (1, 4, 4))
    hits = np.zeros(dims, np.int32)
    for b in blocks:
        hits[b.origin[0]:b.origin[0] + b.size[0], b.origin[1]:b.origin[1] + b.size[1],
             b.origin[2]:b.origin[2] + b.size[2]] += 1
        for a in range(3):
            assert b.read_origin[a] + b.read_size[a] <= dims[a] and b.read_origin[a] <= b.origin[a]
    assert (hits == 1).all()
    assert [b.index for b in blocks] == list(range(len(blocks)))
    b = lb.schedule((1, 10, 10), (1, 4, 4), (0, 2, 2))[0]
    assert b.read_dims() == [6, 6] and b.inner_offset() == (0, 0, 0)
    assert lb.schedule((0, 5, 5), (1, 2, 2), (0, 1, 1)) == []


def test_slide_schedule_matches_the_tile_walk_geometry():
    """The batched-tile workload: 1024 blocks with a 32 px halo over a
    34560 x 24960 slide: 34 x 25 blocks, edge blocks 768 tall / 384 wide."""
    import lucem_b200 as lb

    blocks = lb.schedule((1, 34560, 24960), (1, 1024, 1024), (0, 32, 32))
    assert len(blocks) == 34 * 25
    sizes = {(b.size[1], b.size[2]) for b in blocks}
    assert sizes == {(1024, 1024), (1024, 384), (768, 1024), (768, 384)}


def test_fft_lengths_and_rl_grid():
    import lucem_b200 as lb

    lib = N.lib()
    assert lib.lucem_fft_good_length(1021, 0) == 1024
    assert lib.lucem_fft_good_length(1025, 0) == 1029  # 3 * 7^3
    assert lib.lucem_fft_good_length(1029, 1) == 1050
    # zero padding needs n + k/2, the other modes n + 2 (k/2); the automatic
    # length is the cheapest m * 2^k above the need by the default pass costs
    # (power-of-two register kernels 1; Stockham 5 for columns, 2.7 for rows)
    assert lb.rl_grid((64, 512, 512), (31, 15, 15), mode="constant") == (128, 1024, 1024)
    assert lb.rl_grid((40, 53), (7, 5), mode="reflect") == (64, 60)   # 60 * 2.7 < 128 * 1
    assert lb.rl_grid((3000, 3000), (9, 9), mode="constant") == (3072, 3072)
    assert lb.rl_grid((64, 512, 512), (31, 15, 15), mode="constant", grid=(128, 1024, 1024)) == (128, 1024, 1024)
    assert lb.rl_grid((100, 200), (9, 9), mode="reflect") == (128, 256)
    with pytest.raises(N.LucemError) as e:
        lb.rl_grid((64, 512, 512), (31, 15, 15), mode="constant", grid=(64, 1024, 1024))
    assert e.value.name == "INVALID_PARAMETER"
    with pytest.raises(N.LucemError):
        lb.rl_grid((10, 10), (3, 3), mode="constant", grid=(13, 12))  # 13 is not 2/3/5/7-smooth


def test_calls_without_a_context_are_refused_before_any_device_work():
    lib = N.lib()
    t = N.Tensor()
    t.dtype, t.ndim = N.F32, 2
    t.dims[0] = t.dims[1] = 4
    sig = (C.c_double * 1)(2.0)
    st = lib.lucem_gaussian_blur(None, C.byref(t), sig, 1, None, C.byref(t), None, None)
    assert N.STATUS_NAMES[st] == "INVALID_HANDLE"
    assert b"context" in lib.lucem_last_error_message()
    st = lib.lucem_richardson_lucy(None, C.byref(t), C.byref(t), None, C.byref(t), None, None)
    assert N.STATUS_NAMES[st] == "INVALID_HANDLE"


def test_library_is_built_for_sm100a():
    """The build compiles every source for sm_100a only."""
    from lucem_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(N.LIB_PATH)


def test_header_compiles_as_c99_and_cpp():
    """include/lucem_b200.h is plain C: a C99 and a C++ translation unit
    include it without warnings."""
    import shutil
    import subprocess

    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "lucem_b200.h")
    for cc, args in (("gcc", ["-x", "c", "-std=c99"]), ("g++", ["-x", "c++", "-std=c++17"])):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not available")
        r = subprocess.run([cc, "-fsyntax-only", "-Wall", "-Wextra", "-Werror", *args, hdr],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
