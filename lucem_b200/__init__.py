"""lucem_b200 -- B200 (sm_100a) implementation of lucem-ops' separable
Gaussian family and Richardson-Lucy deconvolution behind lucem's operator
interface.

    import lucem_b200 as lb
    y = lb.gaussian_blur(x_cuda_u16, 2.0)                    # f32 out
    est = lb.richardson_lucy(obs, psf, num_iter=50, clip=False,
                             filter_epsilon=1e-6, mode="constant")

The kernels live in liblucem_b200.so (C ABI: include/lucem_b200.h); this
package is its host-side mirror of the reference's Python/Rust operator API.
"""
from .ops import *  # noqa: F401,F403
from .ops import __all__ as _ops_all
from . import synth  # noqa: F401
from . import autograd  # noqa: F401

__all__ = list(_ops_all) + ["synth", "autograd"]
