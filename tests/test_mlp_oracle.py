"""CPU checks of the warm-start network's oracle and the library's host-side
feature normalisation (no GPU calls)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0.0, 0.3, mo.NPARAM)
    X = rng.uniform(-1, 1, (40, mo.NIN))
    Y = rng.uniform(0, 1.5, 40)
    _, g = mo.loss_and_grad64(p, X, Y)
    idx = np.concatenate([rng.choice(mo.NPARAM, 60, replace=False),
                          [mo.OFF[k][0] for k in mo.OFF]])
    fd = mo.finite_difference(p, X, Y, idx)
    assert np.max(np.abs(fd - g[idx])) <= 1e-7 * np.max(np.abs(g[idx]))


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.001953125, 1.0029296875, -2.5, 3.0e-3], dtype=np.float32)
    r = mo.bf16(x)
    # bf16 keeps 8 significant bits: at most half a spacing (2^-8 relative) away
    for v, q in zip(x, r):
        lo = np.float32(q)
        assert abs(float(v) - float(lo)) <= abs(float(v)) * 2 ** -8
    assert mo.bf16(np.float32(1 + 2 ** -8))[()] == 1.0           # tie -> even (1.0)
    assert mo.bf16(np.float32(1 + 3 * 2 ** -8))[()] == 1 + 2 ** -6  # tie -> even (1 + 2^-6)


def test_features_match_library_host_code():
    from multiphaselb_b200 import warmstart
    rng = np.random.default_rng(5)
    for _ in range(300):
        t, R = rng.uniform(0.5, 1.0), rng.uniform(4.0, 200.0)
        r = rng.uniform(0.0, 3.0 * R)
        a, b = rng.choice([1.0, 0.5]), rng.choice([4.0, 2.0])
        want = np.ravel(mo.features(t, a, b, r, R)).astype(np.float32)
        got = warmstart.features(t, a, b, r, R)
        assert np.array_equal(got, want), (t, a, b, r, R, got, want)


def test_flat_interface_features_match_library_host_code():
    """R = +inf: r is the signed distance to a flat interface (liquid bands,
    mplb_mlp_init_column); the curvature input is -1 (k = 0)."""
    from multiphaselb_b200 import warmstart
    rng = np.random.default_rng(6)
    for _ in range(300):
        t, d = rng.uniform(0.5, 1.0), rng.uniform(-40.0, 40.0)
        want = np.ravel(mo.features(t, 1.0, 4.0, d, np.inf)).astype(np.float32)
        got = warmstart.features(t, 1.0, 4.0, d, np.inf)
        assert np.array_equal(got, want), (t, d, got, want)
        assert got[4] == -1.0
        assert got[3] == mo.bf16(np.float32(np.clip(d / 5.0, -6.0, 6.0) / 6.0))
