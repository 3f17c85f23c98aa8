"""The TMA-staged D3Q15 kernel (k_fused_d3q15_tma) against the oracle, bit for bit.

It takes fully periodic D3Q15 boxes without boundary programs whose x and y
extents are multiples of its tile (tile candidates 7 = 32 x 4, 8 = 32 x 8,
9 = 32 x 16 and 10 = 64 x 8).  Tiles inside the box stage each plane with
tensor copies; tiles on a face (their pull boxes wrap around the periodic
faces) take row copies.  The lattices here hold both kinds: 96 x 24 in xy
has interior tiles for the first two shapes, 192 x 48 for all four.
"""
import numpy as np
import pytest

from multiphaselb_b200 import Lattice, abi, cases
from tests.helpers import assert_same, run_checker

pytestmark = pytest.mark.gpu

TMA_CANDIDATES = (7, 8, 9, 10)  # tile_config values (1-based) of the TMA kernel
TMA_TILES = {7: (32, 4), 8: (32, 8), 9: (32, 16), 10: (64, 8)}


def takes(case, tile):
    tx, ty = TMA_TILES[tile]
    return case.dims[0] % tx == 0 and case.dims[1] % ty == 0


def periodic_cases():
    base = cases.bubble_case(abi.D3Q15, 96, 8.0, 3.0, 0.75, dims=(96, 24, 10))
    out = {"bubble_96x24x10": cases.perturbed(base, du=1e-3)}
    # node-varying temperature (psi reads T per node), gravity and an external force
    c = cases.perturbed(base, du=2e-3, drho=1e-3)
    rng = np.random.Generator(np.random.PCG64(11))
    c.T = c.T * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, size=c.n))
    c.eos = dict(c.eos, g=(0.0, -1e-5, 2e-6), fext=(1e-6, 0.0, -1e-6), rho_0=0.0)
    c.name = "bubble_Tnoise_force_96x24x10"
    out[c.name] = c
    # the surface-tension term (xuMRTSurfaceTension) from the same psi ring
    s = cases.perturbed(base, du=1e-3)
    s.f = dict(s.f, surface_tension=1, kappa_st=0.4)
    s.name = "bubble_st_96x24x10"
    out[s.name] = s
    # a box whose every tile lies on a face (per-element copies only), odd z
    e = cases.perturbed(cases.bubble_case(abi.D3Q15, 32, 4.0, 2.0, 0.75, dims=(32, 8, 7)), du=1e-3)
    out["bubble_32x8x7"] = e
    # interior and face tiles of every candidate, node-varying T and forces
    w = cases.perturbed(cases.bubble_case(abi.D3Q15, 192, 10.0, 3.0, 0.75, dims=(192, 48, 6)), du=2e-3, drho=1e-3)
    w.T = w.T * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, size=w.n))
    w.eos = dict(w.eos, g=(0.0, -1e-5, 2e-6), fext=(1e-6, 0.0, -1e-6), rho_0=0.0)
    w.name = "bubble_Tnoise_force_192x48x6"
    out[w.name] = w
    return out


PAIRS = [(name, tile) for name, case in periodic_cases().items() for tile in TMA_CANDIDATES if takes(case, tile)]


def run(case, steps, tile):
    with Lattice(case, path=abi.PATH_FUSED, tile_config=tile) as lat:
        lat.upload_case()
        lat.initialize()
        lat.step(steps)
        out = lat.download()
        return out, lat.info()


@pytest.mark.parametrize("name,tile", PAIRS)
def test_tma_kernel_matches_oracle(gpu_lib, name, tile):
    case = periodic_cases()[name]
    steps = 30
    got, info = run(case, steps, tile)
    assert info["path"] == abi.PATH_FUSED and info["tile_config"] == tile - 1
    assert_same(got, run_checker("port", case, steps), fields=("rho", "U", "T", "Fi", "Ft", "S", "f"),
                ctx=f"{name} TMA candidate {tile}")


def test_tma_kernel_stepwise_and_autotuned(gpu_lib):
    """Single steps with downloads in between (the lazily rebuilt reference
    state around every step), and the autotuner's pick, against the oracle."""
    case = periodic_cases()["bubble_Tnoise_force_192x48x6"]
    want = run_checker("port", case, 7)
    for tile in TMA_CANDIDATES + (0,):
        with Lattice(case, path=abi.PATH_FUSED, tile_config=tile) as lat:
            lat.upload_case()
            lat.initialize()
            for _ in range(7):
                lat.step(1)
                lat.download()
            assert_same(lat.download(), want, fields=("rho", "U", "Fi", "Ft", "f"), ctx=f"stepwise tile {tile}")
            if tile == 0:
                info = lat.info()
                assert all(info["tile_ms"][c - 1] > 0 for c in TMA_CANDIDATES), info["tile_ms"]


def test_tma_candidates_refuse_other_lattices(gpu_lib):
    """A lattice the TMA kernel does not take (x extent not a multiple of 32)
    refuses the forced candidate with an argument error."""
    case = cases.perturbed(cases.bubble_case(abi.D3Q15, 10, 3.0, 2.0, 0.75, dims=(10, 8, 6)), du=1e-3)
    with Lattice(case, path=abi.PATH_FUSED, tile_config=7) as lat:
        lat.upload_case()
        lat.initialize()
        with pytest.raises(RuntimeError, match="does not take this lattice"):
            lat.step(1)


def test_tma_kernel_fullsize_bubble(gpu_lib):
    """The 192^3 workload on every TMA candidate: equal to the oracle after
    one step and to the general kernel after 20."""
    case = cases.standard_cases()["bubble_d3q15_192"]()
    want1 = run_checker("port", case, 1)
    gen, _ = run(case, 20, 3)  # 32 x 4 general kernel
    for tile in TMA_CANDIDATES:
        got1, _ = run(case, 1, tile)
        assert_same(got1, want1, fields=("rho", "U", "Fi", "Ft", "f"), ctx=f"192^3 TMA {tile} vs oracle")
        got, _ = run(case, 20, tile)
        assert_same(got, gen, fields=("rho", "U", "Fi", "Ft", "f"), ctx=f"192^3 TMA {tile} vs general, 20 steps")
