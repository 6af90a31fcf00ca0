"""PBE in the CPU oracle (CPU only). The reference has no PBE, so this pins the
restatement by its own properties: complex-step derivatives against central
differences, the large-gradient limit (exchange -> (1 + kappa) x Slater, gradient
correction of correlation -> -eps_c), spin-exchange symmetry, homogeneity of the
exchange part and the uniform-gas limit against the reference's VWN5 LDA."""
import numpy as np
import pytest

from oracle import oracle

KAPPA = 0.804


def pts(n=60, seed=3):
    rng = np.random.default_rng(seed)
    ra = 10 ** rng.uniform(-4, 1.5, n)
    rb = ra * 10 ** rng.uniform(-1, 1, n)
    gaa = 10 ** rng.uniform(-6, 2, n) * ra ** (8 / 3)
    gbb = 10 ** rng.uniform(-6, 2, n) * rb ** (8 / 3)
    gab = np.sqrt(gaa * gbb) * rng.uniform(-1, 1, n)
    return ra, rb, gaa, gab, gbb


def test_derivatives_match_central_differences():
    ra, rb, gaa, gab, gbb = pts()
    out = oracle.functional("PBE", ra, rb, gaa, gab, gbb)
    x = np.stack([ra, rb, gaa, gab, gbb], axis=1)
    for k in range(5):
        h = 1e-6 * np.abs(x[:, k]) + 1e-14
        xp, xm = x.copy(), x.copy()
        xp[:, k] += h
        xm[:, k] -= h
        fp = oracle.functional("PBE", *xp.T)[:, 0]
        fm = oracle.functional("PBE", *xm.T)[:, 0]
        fd = (fp - fm) / (2 * h)
        scale = np.abs(out[:, 0]) / np.maximum(np.abs(x[:, k]), 1e-300) + np.abs(out[:, 1 + k])
        assert np.all(np.abs(out[:, 1 + k] - fd) <= 1e-6 * scale), k


def test_large_gradient_limit_is_scaled_slater_exchange():
    ra, rb, _, _, _ = pts(seed=4)
    big = 1e24
    f = oracle.functional("PBE", ra, rb, big, 0.0 * ra, big)[:, 0]
    sl = np.array([oracle.component("Slater", a, b, 0, 0, 0)[0] for a, b in zip(ra, rb)])
    assert np.allclose(f, (1.0 + KAPPA) * sl, rtol=1e-8, atol=0)


def test_spin_exchange_symmetry():
    ra, rb, gaa, gab, gbb = pts(seed=5)
    a = oracle.functional("PBE", ra, rb, gaa, gab, gbb)
    b = oracle.functional("PBE", rb, ra, gbb, gab, gaa)
    assert np.allclose(a[:, 0], b[:, 0], rtol=1e-13, atol=0)
    assert np.allclose(a[:, 1], b[:, 2], rtol=1e-12, atol=0)
    assert np.allclose(a[:, 3], b[:, 5], rtol=1e-12, atol=0)


def test_exchange_homogeneity():
    """f_x(l^3 rho, l^8 gamma) = l^4 f_x: correlation removed through the large-gradient
    limit (where it vanishes), so this checks the exchange enhancement's s scaling."""
    ra, rb, gaa, gab, gbb = pts(seed=6)
    lam = 1.7
    big = 1e24
    f1 = oracle.functional("PBE", ra, rb, big, 0 * ra, big)[:, 0]
    f2 = oracle.functional("PBE", lam ** 3 * ra, lam ** 3 * rb, big, 0 * ra, big)[:, 0]
    assert np.allclose(f2, lam ** 4 * f1, rtol=1e-8, atol=0)


def test_uniform_gas_close_to_reference_lda():
    """gamma = 0: PBE reduces to Slater exchange + PW92 correlation; PW92 and the
    reference's VWN5 are two fits of the same Monte Carlo data (within ~1 %)."""
    ra, rb, _, _, _ = pts(seed=7)
    rb = ra.copy()
    f_pbe = oracle.functional("PBE", ra, rb, 0 * ra, 0 * ra, 0 * ra)[:, 0]
    f_svwn = oracle.functional("SVWN", ra, rb, 0 * ra, 0 * ra, 0 * ra)[:, 0]
    sl = np.array([oracle.component("Slater", a, b, 0, 0, 0)[0] for a, b in zip(ra, rb)])
    ec_pbe, ec_vwn = f_pbe - sl, f_svwn - sl
    assert np.all(ec_pbe < 0)
    assert np.allclose(ec_pbe, ec_vwn, rtol=2e-2, atol=0)


def test_pbe_is_a_gga_in_the_quadrature(water2):
    from conftest import shell_table
    sh = shell_table(water2)
    r = oracle.xc("PBE", sh, water2["grid"][:500, :4], water2["PA"])
    assert r["rho"].shape[1] == 4 and np.isfinite(r["exc"]) and r["exc"] < 0
