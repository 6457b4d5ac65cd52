"""The pipeline stage (lucem_b200.pipeline): the reference's Op JSON rules
(engine/lucem-pipeline/src/ops.rs:97-203 with serde's tag, snake_case and
deny_unknown_fields), validate (ops.rs:695-760), halo (ops.rs:434-452),
at_downsample (ops.rs:456-520) and ridge_sigmas (ops.rs:969-975).  Host
logic only: no GPU."""
import json

import pytest

from lucem_b200 import pipeline as P


def test_parse_round_trip_and_defaults():
    for op in P.catalog():
        back = P.parse_op(op.spec())
        assert back == op
        back.validate()


def test_parse_refuses_what_serde_refuses():
    with pytest.raises(ValueError, match="unknown variant"):
        P.parse_op('{"op": "median", "radius": 2}')
    with pytest.raises(ValueError, match="unknown field"):
        P.parse_op('{"op": "gaussian_blur", "sigma": 2.0, "mode": "reflect"}')
    with pytest.raises(ValueError, match="missing field `sigma`"):
        P.parse_op('{"op": "gaussian_blur"}')
    with pytest.raises(ValueError, match="missing field `op`"):
        P.parse_op('{"sigma": 2.0}')
    with pytest.raises(ValueError, match="boolean"):
        P.parse_op('{"op": "frangi", "sigma_min": 1, "sigma_max": 2, "black_ridges": 1}')
    with pytest.raises(ValueError, match="unsigned integer"):
        P.parse_op('{"op": "richardson_lucy", "num_iter": -3, "psf_sigma": 1.0, "clip": false, '
                   '"filter_epsilon": 1e-6}')
    # integers are numbers
    assert P.parse_op('{"op": "gaussian_blur", "sigma": 2}').params["sigma"] == 2.0


def test_validate_messages():
    bad = [('{"op": "gaussian_blur", "sigma": 0}', "sigma must be a positive number"),
           ('{"op": "difference_of_gaussians", "low_sigma": 3, "high_sigma": 2}', "high sigma must be larger"),
           ('{"op": "sato", "sigma_min": 3, "sigma_max": 2, "black_ridges": true}', "sigma max must be"),
           ('{"op": "richardson_lucy", "num_iter": 0, "psf_sigma": 1.0, "clip": false, "filter_epsilon": 1e-6}',
            "num_iter must be at least 1")]
    for spec, msg in bad:
        with pytest.raises(ValueError, match=msg):
            P.parse_op(spec).validate()


def test_halo_like_the_reference():
    """ops.rs:434-452: ceil(4 sigma) of the widest Gaussian; the halo of sigma
    2 is 8 (bindings/python/tests/test_runtime_io.py:28)."""
    h = lambda s: P.parse_op(s).halo()  # noqa: E731
    assert h('{"op": "gaussian_blur", "sigma": 2.0}') == 8
    assert h('{"op": "gaussian_blur", "sigma": 1.1}') == 5
    assert h('{"op": "unsharp_mask", "sigma": 0.5, "amount": 1.0}') == 2
    assert h('{"op": "difference_of_gaussians", "low_sigma": 1, "high_sigma": 3}') == 12
    assert h('{"op": "frangi", "sigma_min": 1, "sigma_max": 4.2, "black_ridges": false}') == 17
    assert h('{"op": "richardson_lucy", "num_iter": 5, "psf_sigma": 1.5, "clip": false, '
             '"filter_epsilon": 1e-6}') == 2 * 5 * 5


def test_at_downsample_and_ridge_sigmas():
    op = P.parse_op('{"op": "difference_of_gaussians", "low_sigma": 1.0, "high_sigma": 1.2}')
    d = op.at_downsample(8.0)
    assert d.params["low_sigma"] == 0.3 and d.params["high_sigma"] == pytest.approx(0.303)
    f = P.parse_op('{"op": "frangi", "sigma_min": 2, "sigma_max": 8, "black_ridges": true}').at_downsample(2.0)
    assert (f.params["sigma_min"], f.params["sigma_max"]) == (1.0, 4.0)
    assert P.ridge_sigmas(1.0, 5.0) == [1.0, 2.0, 3.0, 4.0, 5.0]
    assert P.ridge_sigmas(2.0, 2.0) == [2.0]
    assert json.loads(op.spec())["op"] == "difference_of_gaussians"
