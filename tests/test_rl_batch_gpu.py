"""Batched uneven 2-D Richardson-Lucy (lucem_rl_batch_*) against the oracle:
every problem of a batch equals the oracle's Richardson-Lucy on that problem
(FP64 FFT form for zero padding, the direct f32 restatement of the reference
for the other modes), tolerance 1e-4 (assert_close semantics).  The batched
run, the per-problem run and a CUDA-graph replay give identical bits."""
import numpy as np
import pytest
import torch

import lucem_b200 as lb

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().astype(np.float64)


def problems(seed, n, lo, hi, kmax=9):
    rng = np.random.default_rng(seed)
    obs, psfs = [], []
    for i in range(n):
        h, w = int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1))
        kh, kw = int(rng.integers(1, kmax + 1)), int(rng.integers(1, kmax + 1))
        obs.append(rng.uniform(0.5, 2.0, (h, w)).astype(np.float32))
        psfs.append(rng.uniform(0.1, 1.0, (kh, kw)).astype(np.float32))
    return obs, psfs


def test_uneven_batch_zero_padding_against_fp64(oracle):
    obs, psfs = problems(1, 14, 12, 140)
    b = lb.RlBatch([dev(o) for o in obs], [dev(p) for p in psfs], num_iter=8, clip=False, filter_epsilon=1e-6,
                   mode="constant")
    outs = b.run()
    for i, (o, p) in enumerate(zip(obs, psfs)):
        want = oracle.richardson_lucy_fft64(o, p, num_iter=8, clip=False, filter_epsilon=1e-6)
        oracle.assert_close(host(outs[i]), want, RTOL, f"problem {i} {o.shape} psf {p.shape}")
    b.close()


@pytest.mark.parametrize("mode", ["reflect", "wrap", "nearest"])
def test_uneven_batch_extension_modes_against_direct(oracle, mode):
    obs, psfs = problems(2, 6, 10, 48, kmax=7)
    b = lb.RlBatch([dev(o) for o in obs], [dev(p) for p in psfs], num_iter=5, clip=True, filter_epsilon=1e-6,
                   mode=mode)
    outs = b.run()
    for i, (o, p) in enumerate(zip(obs, psfs)):
        want = oracle.richardson_lucy(o, p, num_iter=5, clip=True, filter_epsilon=1e-6, mode=mode)
        oracle.assert_close(host(outs[i]), want.astype(np.float64), RTOL, f"{mode} problem {i}")
    b.close()


def test_large_problems_use_the_fast_lengths(oracle):
    rng = np.random.default_rng(3)
    shapes = [(500, 1000), (1000, 500), (250, 250), (700, 300)]
    obs = [rng.uniform(0.5, 2.0, s).astype(np.float32) for s in shapes]
    psfs = [lb.synth.gaussian_psf((13, 13), (2.0, 2.0)).astype(np.float32) for _ in shapes]
    b = lb.RlBatch([dev(o) for o in obs], [dev(p) for p in psfs], num_iter=4, clip=False, filter_epsilon=1e-6,
                   mode="constant")
    grids, _, _ = b.info()
    assert all(gy >= s[0] + 6 and gx >= s[1] + 6 for (gy, gx), s in zip(grids, shapes))
    outs = b.run()
    for i, (o, p) in enumerate(zip(obs, psfs)):
        want = oracle.richardson_lucy_fft64(o, p, num_iter=4, clip=False, filter_epsilon=1e-6)
        oracle.assert_close(host(outs[i]), want, RTOL, f"problem {i} {shapes[i]} grid {grids[i]}")
    b.close()


def test_batched_per_problem_and_graph_runs_agree():
    obs, psfs = problems(4, 9, 20, 90)
    xs, ps = [dev(o) for o in obs], [dev(p) for p in psfs]
    b = lb.RlBatch(xs, ps, num_iter=6, clip=False, filter_epsilon=1e-6, mode="constant")
    a = [host(t) for t in b.run()]
    c = [host(t) for t in b.run(per_problem=True)]
    for u, v in zip(a, c):
        assert np.array_equal(u, v)
    for t in b.outs:
        t.zero_()
    g = lb.Graph()
    with g:
        b.run()
    g.launch()
    g.launch()
    d = [host(t) for t in b.outs]
    for u, v in zip(a, d):
        assert np.array_equal(u, v)
    g.close()
    b.close()


def test_equal_lengths_share_one_launch():
    obs = [np.full((64, 100), 1.0, np.float32)] * 5 + [np.full((30, 40), 1.0, np.float32)] * 3
    psfs = [np.ones((5, 5), np.float32)] * 8
    b = lb.RlBatch([dev(o) for o in obs], [dev(p) for p in psfs], num_iter=1, clip=False, mode="constant")
    grids, nrow, ncol = b.info()
    assert len(set(grids)) == 2 and nrow == len({g[1] for g in grids}) and ncol == len({g[0] for g in grids})
    b.close()


def test_batch_argument_errors():
    x, p = dev(np.ones((8, 8))), dev(np.ones((3, 3)))
    with pytest.raises(lb.LucemError):
        lb.RlBatch([x], [p, p])
    with pytest.raises(lb.LucemError):
        lb.RlBatch([dev(np.ones((4, 8, 8)))], [dev(np.ones((1, 3, 3)))])
    with pytest.raises(lb.LucemError):
        lb.RlBatch([x], [p], num_iter=0)


def test_autotune_table_round_trip(tmp_path):
    lb.autotune_fft([64, 96, 128, 250])
    for kind in (0, 1):
        for n in (64, 96, 128, 250):
            assert lb.autotune_query(kind, n) > 0
    path = tmp_path / "tune.txt"
    lb.autotune_save(str(path))
    assert len([l for l in path.read_text().splitlines() if not l.startswith("#")]) >= 8
    lb.autotune_load(str(path))
    bad = tmp_path / "bad.txt"
    bad.write_text("0 64 -1\n")
    with pytest.raises(lb.LucemError):
        lb.autotune_load(str(bad))
    with pytest.raises(lb.LucemError):
        lb.autotune_fft([97])
