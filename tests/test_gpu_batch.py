"""Batched ensemble (mplb_batch_*): many periodic D2Q9 FP32-deviation
lattices of uneven size advanced by one launch per step.

Each lattice in a batch must evolve exactly as the same lattice stepped alone
through its own handle (same device function, same arguments), so the
comparisons here are bitwise.  Convergence retirement is checked the same
way: a lattice that leaves the work table after s steps equals a lone
lattice stepped s times."""
import numpy as np
import pytest

from multiphaselb_b200 import Batch, Lattice, MplbError, abi, cases

pytestmark = pytest.mark.gpu

SHAPES = [((32, 32), 8.0, 0.8), ((48, 40), 10.0, 0.7), ((64, 32), 9.0, 0.9), ((40, 56), 12.0, 0.65),
          ((96, 64), 14.0, 0.85)]


def ensemble():
    return [cases.bubble_case(abi.D2Q9, dims=d, radius=r, width=4.0, t_ratio=t, name=f"b{i}")
            for i, (d, r, t) in enumerate(SHAPES)]


def lone(case, steps):
    with Lattice(case, path=abi.PATH_FUSED, precision=abi.FP32_DEV) as lat:
        lat.upload_case()
        lat.initialize()
        for s in steps:
            lat.step(s)
        return lat.download()


def lone_run(case, steps, K):
    """A lone lattice through the same equilibrium-run procedure (checks and
    FP32 momentum resets every K steps), held for exactly `steps` steps."""
    with Lattice(case, path=abi.PATH_FUSED, precision=abi.FP32_DEV) as lat:
        lat.upload_case()
        lat.initialize()
        got, _ = lat.run_to_equilibrium(steps, K, 0.0)
        assert got == steps
        return lat.download()


def make(cs):
    lats = []
    for c in cs:
        lat = Lattice(c, path=abi.PATH_FUSED, precision=abi.FP32_DEV)
        lat.upload_case()
        lat.initialize()
        lats.append(lat)
    return lats


def same(a, b, ctx):
    for k in ("rho", "U", "f", "Fi"):
        assert np.array_equal(a[k], b[k]), (ctx, k, float(np.abs(a[k] - b[k]).max()))


@pytest.mark.parametrize("tile", [1, 2, 3, 4])
def test_batch_steps_match_lone_lattices(gpu_lib, tile):
    cs = ensemble()
    want = [lone(c, [7]) for c in cs]
    lats = make(cs)
    with Batch(lats, tile_config=tile) as b:
        b.step(7)
        info = b.info()
        assert info["tile_config"] == tile - 1
        assert info["nodes"] == sum(c.n for c in cs)
        for c, lat, w in zip(cs, lats, want):
            same(lat.download(), w, (c.name, tile))
            assert lat.info()["current_time"] == 7
    for lat in lats:
        lat.close()


def test_batch_then_handle_steps(gpu_lib):
    """Odd batch steps, then the handles' own steps, then the batch again."""
    cs = ensemble()
    want = [lone(c, [12]) for c in cs]
    lats = make(cs)
    with Batch(lats) as b:
        b.step(5)
        for lat in lats:
            lat.step(2)
        b.step(5)
        for c, lat, w in zip(cs, lats, want):
            same(lat.download(), w, c.name)
        info = b.info()
        assert 0 <= info["tile_config"] < len(info["tiles"])
        assert all(ms > 0 for ms in info["tile_ms"]), info
    for lat in lats:
        lat.close()


def test_batch_run_retires_converged_lattices(gpu_lib):
    """Run to a loose tolerance: each lattice's step count is a whole number of
    check intervals, converged ones report a rate under tol, and every
    lattice's state is that of a lone lattice run through the same
    equilibrium procedure for as many steps."""
    cs = ensemble()
    lats = make(cs)
    K, tol, max_steps = 100, 2e-5, 3000
    with Batch(lats, check_interval=K, tol=tol) as b:
        steps, rate, conv = b.run(max_steps)
        info = b.info()
    print(steps, rate, conv)
    assert conv == int((rate < tol).sum())
    assert conv >= 1
    assert len(set(steps.tolist())) > 1, "expected lattices to retire at different steps"
    for s, r in zip(steps, rate):
        assert s % K == 0 and 0 < s <= max_steps
        assert r >= 0
        if r >= tol:
            assert s == max_steps
    assert info["graph_launches"] == max(steps) // K
    for c, lat, s in zip(cs, lats, steps):
        same(lat.download(), lone_run(c, int(s), K), c.name)
        lat.close()


def test_batch_rejects_ineligible(gpu_lib):
    ok = cases.bubble_case(abi.D2Q9, dims=(32, 32), radius=8.0, width=4.0)
    good = make([ok])[0]
    bad = {
        "fp64": Lattice(ok, path=abi.PATH_FUSED, precision=abi.FP64),
        "d3q15": Lattice(cases.bubble_case(abi.D3Q15, dims=(16, 16, 16), radius=5.0, width=3.0),
                         path=abi.PATH_FUSED, precision=abi.FP32_DEV),
        "walls": Lattice(cases.column_case(16, 32), path=abi.PATH_FUSED, precision=abi.FP32_DEV),
    }
    for name, lat in bad.items():
        with pytest.raises(MplbError) as e:
            Batch([good, lat])
        assert e.value.code == abi.E_UNSUPPORTED, name
        lat.close()
    with pytest.raises(MplbError) as e:
        Batch([good, good])
    assert e.value.code == abi.E_ARG
    with pytest.raises(MplbError) as e:
        Batch([good], check_interval=3)
    assert e.value.code == abi.E_ARG
    good.close()


def test_batch_run_retires_diverged_lattice(gpu_lib):
    cs = ensemble()[:3]
    cs[1].rho = cs[1].rho.copy()
    cs[1].rho[5] = np.nan
    lats = make(cs)
    with Batch(lats, check_interval=20, tol=1e-30) as b:
        steps, rate, conv = b.run(200)
    assert conv == 0
    assert steps[1] == 20 and np.isinf(rate[1])
    assert steps[0] == 200 and steps[2] == 200 and np.isfinite(rate[0]) and np.isfinite(rate[2])
    for lat in lats:
        lat.close()
