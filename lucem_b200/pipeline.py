"""The pipeline's operator stage for this path: lucem-pipeline's `Op`
(engine/lucem-pipeline/src/ops.rs:97-203) restricted to the Gaussian-family,
ridge and deconvolution operators, plus the Richardson-Lucy node the
reference does not have, and the Python `run_op` / `run_chain` of
bindings/python/lucem-py-core/src/ops.rs:124-167.

An operator is the reference's JSON spec, `{"op": "gaussian_blur",
"sigma": 2.0}` (tag `op`, snake_case, unknown fields refused).  `Op.halo()`,
`Op.validate()` and `Op.at_downsample()` follow ops.rs:434-452, 695-760 and
456-520.  `run_op` / `run_chain` take DLPack producers of device memory
zero-copy and leave results on the device (the reference copies NumPy arrays
in and out, lib.rs:42-45); NumPy inputs are uploaded once, as the raw integer
type where they are integers (u8 / u16 go to the device at their own width
and are converted to f32 inside the first kernel's tile load, with
`input_scale` fused), and results come back as NumPy.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np
import torch

from . import ops as _ops
from .ops import LucemError, from_dlpack

__all__ = ["Op", "parse_op", "ridge_sigmas", "catalog", "run_op", "run_chain", "OP_FIELDS"]

# op tag -> (field -> type, default); the reference's field names and order.
OP_FIELDS: Dict[str, Dict[str, tuple]] = {
    "gaussian_blur": {"sigma": (float, 2.0)},
    "unsharp_mask": {"sigma": (float, 1.0), "amount": (float, 1.0)},
    "difference_of_gaussians": {"low_sigma": (float, 1.0), "high_sigma": (float, 3.0)},
    "frangi": {"sigma_min": (float, 1.0), "sigma_max": (float, 5.0), "black_ridges": (bool, False)},
    "sato": {"sigma_min": (float, 1.0), "sigma_max": (float, 5.0), "black_ridges": (bool, False)},
    # No counterpart in the reference's Op enum: Richardson-Lucy with a
    # Gaussian PSF of `psf_sigma` (support 2 ceil(3 sigma) + 1, unit sum),
    # zero padding, the reference's RichardsonLucy settings otherwise.
    "richardson_lucy": {"num_iter": (int, 30), "psf_sigma": (float, 2.0), "clip": (bool, False),
                        "filter_epsilon": (float, 1e-6)},
}

_TITLES = {"gaussian_blur": "Gaussian blur", "unsharp_mask": "Unsharp mask",
           "difference_of_gaussians": "Difference of Gaussians", "frangi": "Frangi", "sato": "Sato",
           "richardson_lucy": "Richardson-Lucy"}


def ridge_sigmas(min_s: float, max_s: float) -> List[float]:
    """engine/lucem-pipeline/src/ops.rs:969-975: five scales from min to max
    (one when they are equal)."""
    if abs(max_s - min_s) < 1e-6:
        return [min_s]
    return [min_s + (max_s - min_s) * (i / 4.0) for i in range(5)]


@dataclass
class Op:
    """One operator and its parameters (ops.rs:97-203)."""

    op: str
    params: Dict[str, object] = field(default_factory=dict)

    def title(self) -> str:
        return _TITLES[self.op]

    def spec(self) -> str:
        return json.dumps({"op": self.op, **self.params})

    def validate(self) -> None:
        """ops.rs:695-760 (the arms of these operators); raises ValueError."""
        p = self.params

        def pos(name, v):
            if not (math.isfinite(v) and v > 0.0):
                raise ValueError(f"{name} must be a positive number")

        if self.op == "gaussian_blur":
            pos("sigma", p["sigma"])
        elif self.op == "unsharp_mask":
            pos("sigma", p["sigma"])
            if not math.isfinite(p["amount"]):
                raise ValueError("amount must be a number")
        elif self.op == "difference_of_gaussians":
            pos("low sigma", p["low_sigma"])
            pos("high sigma", p["high_sigma"])
            if p["high_sigma"] <= p["low_sigma"]:
                raise ValueError("high sigma must be larger than low sigma")
        elif self.op in ("frangi", "sato"):
            pos("sigma min", p["sigma_min"])
            pos("sigma max", p["sigma_max"])
            if p["sigma_max"] < p["sigma_min"]:
                raise ValueError("sigma max must be ≥ sigma min")
        elif self.op == "richardson_lucy":
            if p["num_iter"] < 1:
                raise ValueError("num_iter must be at least 1")
            pos("psf sigma", p["psf_sigma"])
            pos("filter epsilon", p["filter_epsilon"])

    def halo(self) -> int:
        """ops.rs:434-452: ceil(4 sigma) of the widest Gaussian.  The
        Richardson-Lucy node: each iteration correlates twice with a PSF of
        radius ceil(3 sigma), so a tile's owned pixels depend on input up to
        2 num_iter ceil(3 sigma) away (the halo that makes tiled equal whole)."""
        p = self.params
        s = lambda v: int(math.ceil(4.0 * max(v, 0.0)))  # noqa: E731
        if self.op in ("gaussian_blur", "unsharp_mask"):
            return s(p["sigma"])
        if self.op == "difference_of_gaussians":
            return s(max(p["low_sigma"], p["high_sigma"]))
        if self.op in ("frangi", "sato"):
            return s(p["sigma_max"])
        if self.op == "richardson_lucy":
            return 2 * int(p["num_iter"]) * int(math.ceil(3.0 * p["psf_sigma"]))
        return 0

    def at_downsample(self, ds: float) -> "Op":
        """ops.rs:456-520: sizes given in level-0 pixels, scaled to a level
        whose pixels are `ds` level-0 pixels (at least 0.3 px)."""
        ds = max(ds, 1e-9)
        s = lambda v: max(v / ds, 0.3)  # noqa: E731
        p = dict(self.params)
        if self.op in ("gaussian_blur", "unsharp_mask"):
            p["sigma"] = s(p["sigma"])
        elif self.op == "difference_of_gaussians":
            lo, hi = s(p["low_sigma"]), s(p["high_sigma"])
            p["low_sigma"], p["high_sigma"] = lo, max(hi, lo * 1.01)
        elif self.op in ("frangi", "sato"):
            lo, hi = s(p["sigma_min"]), s(p["sigma_max"])
            p["sigma_min"], p["sigma_max"] = lo, max(hi, lo)
        elif self.op == "richardson_lucy":
            p["psf_sigma"] = s(p["psf_sigma"])
        return Op(self.op, p)

    def psf(self) -> np.ndarray:
        """The Richardson-Lucy node's PSF: a unit-sum isotropic Gaussian on
        2 ceil(3 sigma) + 1 samples per side."""
        sg = float(self.params["psf_sigma"])
        r = int(math.ceil(3.0 * sg))
        ax = np.arange(-r, r + 1, dtype=np.float64)
        g = np.exp(-(ax[:, None] ** 2 + ax[None, :] ** 2) / (2.0 * sg * sg))
        return (g / g.sum()).astype(np.float32)

    def run(self, x: torch.Tensor, *, input_scale: float = 1.0, workspace=None) -> torch.Tensor:
        """ops.rs:778-800 (these operators' arms), on a 2-D device image."""
        self.validate()
        p = self.params
        if x.dim() != 2:
            raise LucemError(3, f"{self.title()}: input must be a 2-D image, got {x.dim()}-D")
        kw = {"workspace": workspace}
        if self.op == "gaussian_blur":
            return _ops.gaussian_blur(x, [p["sigma"], p["sigma"]], input_scale=input_scale, **kw)
        if self.op == "unsharp_mask":
            return _ops.unsharp_mask(x, [p["sigma"], p["sigma"]], p["amount"], input_scale=input_scale, **kw)
        if self.op == "difference_of_gaussians":
            return _ops.difference_of_gaussians(x, [p["low_sigma"]] * 2, [p["high_sigma"]] * 2,
                                                input_scale=input_scale, **kw)
        # The ridge filters and Richardson-Lucy take f32: integer input is
        # cast (and scaled) on the device first.
        if input_scale != 1.0 or x.dtype != torch.float32:
            x = _ops.gaussian_blur(x, [0.0, 0.0], input_scale=input_scale, **kw)
        if self.op in ("frangi", "sato"):
            fn = _ops.frangi if self.op == "frangi" else _ops.sato
            return fn(x, ridge_sigmas(p["sigma_min"], p["sigma_max"]), black_ridges=p["black_ridges"], **kw)
        psf = torch.from_numpy(self.psf()).to(x.device)
        return _ops.richardson_lucy(x, psf, num_iter=int(p["num_iter"]), clip=bool(p["clip"]),
                                    filter_epsilon=float(p["filter_epsilon"]), mode="constant", **kw)


def parse_op(spec) -> Op:
    """A JSON spec (or dict) -> Op, with serde's tag / deny_unknown_fields /
    defaulted-field rules of the reference's `Op` (ops.rs:97-99)."""
    d = json.loads(spec) if isinstance(spec, str) else dict(spec)
    tag = d.pop("op", None)
    if tag is None:
        raise ValueError("missing field `op`")
    if tag not in OP_FIELDS:
        raise ValueError(f"unknown variant `{tag}`, expected one of {sorted(OP_FIELDS)}")
    fields = OP_FIELDS[tag]
    unknown = [k for k in d if k not in fields]
    if unknown:
        raise ValueError(f"unknown field `{unknown[0]}`, expected one of {list(fields)}")
    params = {}
    for name, (ty, default) in fields.items():
        if name not in d:
            raise ValueError(f"missing field `{name}`")
        v = d[name]
        if ty is bool and not isinstance(v, bool):
            raise ValueError(f"invalid type for `{name}`: expected a boolean")
        if ty is int and (isinstance(v, bool) or not isinstance(v, int) or v < 0):
            raise ValueError(f"invalid type for `{name}`: expected an unsigned integer")
        if ty is float and (isinstance(v, bool) or not isinstance(v, (int, float))):
            raise ValueError(f"invalid type for `{name}`: expected a number")
        params[name] = ty(v)
    return Op(tag, params)


def catalog() -> List[Op]:
    """These operators with their default parameters (ops.rs:978-...)."""
    return [Op(tag, {k: v[1] for k, v in f.items()}) for tag, f in OP_FIELDS.items()]


def _to_device(a, device):
    """A DLPack producer of device memory -> a zero-copy torch view; a NumPy
    array -> one upload at its own element width (f32, u8 or u16)."""
    if isinstance(a, torch.Tensor) or (hasattr(a, "__dlpack__") and not isinstance(a, np.ndarray)):
        return from_dlpack(a), False
    arr = np.ascontiguousarray(a)
    if arr.dtype not in (np.float32, np.uint8, np.uint16):
        arr = arr.astype(np.float32)
    return torch.from_numpy(arr).to(device), True


def run_op(spec, inputs: Sequence, *, input_scale: float = 1.0, device=None):
    """bindings/python/lucem-py-core/src/ops.rs:124-141 run_op: one operator on
    one image.  Device inputs (DLPack) stay on the device and the result is a
    device tensor; a NumPy input is uploaded once (integers at their own
    width, the cast and `input_scale` fused into the first kernel) and the
    result comes back as NumPy."""
    op = parse_op(spec)
    if len(inputs) != 1:
        raise ValueError(f"{op.title()} takes 1 input(s), {len(inputs)} given")
    return run_chain([spec], inputs[0], input_scale=input_scale, device=device)


def run_chain(specs: Sequence, x, *, input_scale: float = 1.0, device=None):
    """ops.rs:144-167 run_chain: one-input operators in order on one image,
    staying on the device between them (one upload, one download for NumPy
    input; none for device input)."""
    ops_ = [parse_op(s) for s in specs]
    if not ops_:
        raise ValueError("a chain needs at least one operator")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    t, from_host = _to_device(x, dev)
    for i, op in enumerate(ops_):
        t = op.run(t, input_scale=input_scale if i == 0 else 1.0)
    return t.cpu().numpy() if from_host else t
