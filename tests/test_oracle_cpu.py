"""The float64 oracle and the shared sampler, pinned against the reference engine's golden vectors:
the Philox and splitmix known answers of its tests (tests/test_util.cpp:159-171), its sampler and blur
outputs (run from its own code, tests/golden), and its renders (tests/golden/golden_renders.npz)."""

import json
import os

import numpy as np
import pytest

import oracle
from conftest import coupler_steep_mask, BASE, GOLDEN, golden, lsb_stats, sc, setup_f64

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0, 200, 0, 0), (0x5EED, 0), (0x15CECB3F, 0xF63DFA39, 0x3EC2DC0E, 0xF78F6C18)),
]


def test_philox_known_answers():
    for ctr, key, want in KAT:
        got = oracle.philox(np.array(ctr, np.uint32), np.array(key, np.uint32))[0]
        assert tuple(int(v) for v in got) == want
    # the vectorised numpy copy used to make the synthetic frames agrees
    x = sc.philox_np(np.array([0], np.uint64), np.array([200], np.uint64), 0x5EED)
    assert int(x[0]) == 0x15CECB3F


def test_splitmix_seed_sequence():
    assert oracle.splitmix(4) == [0x4ABEA221, 0x23148989, 0x609DFE03, 0xDEB12800]


def test_philox_uniform_edges():
    L = oracle.lib()
    assert L.orc_uniform(0) == 0.5 * 2.0 ** -24
    assert L.orc_uniform(0xFFFFFEFF) < 1.0
    assert L.orc_uniform(0xFFFFFFFF) == 1.0


def ulp_err(a, b64):
    a = np.asarray(a, np.float64)
    b32 = b64.astype(np.float32)
    spacing = np.spacing(np.abs(b32)).astype(np.float64)
    return np.abs(a - b64) / spacing


def test_elementary_functions_error_bounds():
    L = oracle.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-80, 80, 20000)), rng.uniform(0.5, 2.0, 20000), [1e-40, 3e-39, 1.0, 2.0]])
    xs = xs.astype(np.float32)
    got = np.array([L.orc_logf(float(x)) for x in xs], np.float32)
    ref = np.log(xs.astype(np.float64))
    nz = np.abs(ref) > 1e-3
    assert ulp_err(got[nz], ref[nz]).max() <= 2.0
    assert np.abs(got[~nz] - ref[~nz]).max() <= 2e-10
    ex = rng.uniform(-100, 88, 20000).astype(np.float32)
    got = np.array([L.orc_expf(float(x)) for x in ex], np.float32)
    want = np.exp(ex.astype(np.float64))
    normal = want > 1.2e-38
    assert ulp_err(got[normal], want[normal]).max() <= 2.0
    cx = rng.uniform(0, 2 * np.pi, 20000).astype(np.float32)
    got = np.array([L.orc_cosf(float(x)) for x in cx], np.float32)
    assert np.abs(got - np.cos(cx.astype(np.float64))).max() <= 2e-7
    assert L.orc_logf(0.0) == -np.inf and np.isnan(L.orc_logf(-1.0))
    assert L.orc_expf(-200.0) == 0.0 and L.orc_expf(100.0) == np.inf
    # the sampler's lgamma takes log(2 pi) as a constant: the sampler's own log of SPK_TWO_PI, bit for bit
    two_pi = np.float32(6.283185307179586)
    assert np.float32(L.orc_logf(float(two_pi))).view(np.uint32) == 0x3FEB3F8F


def test_sampler_against_reference():
    g = golden("golden_sampler.npz")
    counts = oracle.poisson(g["lam"], int(g["stream"]), int(g["seed"]))
    mism = int((counts != g["counts"]).sum())
    # the reference's own tolerance between two binary32 samplers: 100 per 20000 draws (tests/test_fx.cpp:565)
    assert mism <= 100 * g["lam"].size // 20000, mism
    logn = oracle.lognormal(g["lam"].size, float(g["mean"]), float(g["sd"]), int(g["stream"]), int(g["seed"]))
    assert ulp_err(logn, g["lognormal"].astype(np.float64)).max() <= 16  # tests/test_fx.cpp:566


@pytest.mark.parametrize("lam", [0.5, 3.0, 9.99, 10.0, 37.0, 600.0, 2500.0])
def test_poisson_moments(lam):
    n = 100000
    k = oracle.poisson(np.full(n, lam, np.float32), 3, 11).astype(np.float64)
    assert abs(k.mean() - lam) < 5 * np.sqrt(lam / n) + 1e-3
    assert abs(k.var() - lam) < 6 * lam * np.sqrt(2.0 / n) + 0.02 * lam


def test_poisson_zero_and_nan():
    k = oracle.poisson(np.array([0.0, np.nan], np.float32), 0, 0)
    assert k[0] == 0.0 and k[1] == 0.0


def test_gaussian_against_reference():
    g = golden("golden_gaussian.npz")
    plane = g["plane"]
    for k in range(3):
        sig = g[f"s{k}_sigma"]
        mine = oracle.gaussian(plane, sig)
        for mode in (0, 1):
            ref = g[f"s{k}_mode{mode}"].astype(np.float64)
            rel = np.abs(mine - ref) / np.maximum(np.abs(ref), 1e-6)
            for c in range(3):
                tol = 1e-5 if sig[c] >= 3 else 2e-6  # tests/test_fx.cpp:200
                assert rel[..., c].max() <= tol, (k, mode, c, rel[..., c].max())


@pytest.mark.parametrize("sigma", [3.0, 4.6, 13.9, 127.6, 261.0, 0.65, 1.5, 2.9])
def test_gaussian_flat_field_and_dc_gain(sigma):
    plane = np.full((41, 53, 3), 0.37)
    out = oracle.gaussian(plane, (sigma, sigma, sigma))
    assert np.abs(out - 0.37).max() < 1e-9  # binary64 state; the reference allows 2e-6 (tests/test_fx.cpp:340)


def test_fir_impulse_equals_taps():
    plane = np.zeros((31, 31, 3))
    plane[15, 15, :] = 1.0
    sigma = 1.5
    out = oracle.gaussian(plane, (sigma, sigma, sigma))
    r = int(np.floor(3 * sigma + 0.5))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    np.testing.assert_allclose(out[15 - r:16 + r, 15 - r:16 + r, 0], np.outer(k, k), atol=1e-15)


def test_render_against_reference_golden(lib, resources):
    meta = json.load(open(os.path.join(GOLDEN, "golden_renders.json")))
    g = golden("golden_renders.npz")
    img = g["image"]
    w, h = meta["width"], meta["height"]
    assert np.array_equal(img, sc.synthetic_image(w, h, meta["seed"]))
    pitch = 35000.0 / max(w, h)
    for name, case in meta["cases"].items():
        f64 = setup_f64(lib, resources, case["delta"], pitch)["f64"]
        hal = case["halation"]
        o = oracle.Oracle(f64, seed=0x4ABEA221, halation=(hal[0], hal[1]) if hal else None)
        out, neg = o.render(img)
        ref = g[f"{name}_rgba"]
        s = lsb_stats(out, ref[0])
        if not case["delta"].get("grain_active", True):
            assert s["max"] <= 1, (name, s)
            np.testing.assert_allclose(neg, g[f"{name}_negative"], rtol=0, atol=2e-5)
            out2, _ = o.print(neg, print_exposure=meta["exposures"][1])
            assert lsb_stats(out2, ref[1])["max"] <= 1, name
        else:
            # grain: the binary64 lambdas flip a few Poisson counts against the reference's binary32 ones;
            # the developed density agrees everywhere else and on average
            dn = np.abs(neg - g[f"{name}_negative"])
            assert np.median(dn) < 1e-5 and abs(neg.mean() - g[f"{name}_negative"].mean()) < 1e-3, name
            assert s["frac_gt1"] < 0.5, (name, s)
        assert (out[..., 3] == 65535).all()


@pytest.mark.parametrize("amount", [0.5, 1.0, 4.0])
def test_couplers_against_reference(lib, resources, ref, ref_engine, amount):
    """DIR couplers (reference src/film/develop.cpp:203-226): the float64 oracle's render against the
    reference engine itself, without grain: the negatives within 2e-5 and the RGBA within 1 LSB16, except
    where the pre-inverted curve is steep (coupler_steep_mask); there within its slope times 4 binary32
    rounding steps of the log exposure. At the schema's largest amount (4) y0 is flat but for one step, and
    the negative holds channels at zero density: the print's gamut compression of those saturated colours
    parts binary32 from binary64 by a few LSB16 on a handful of pixels."""
    import ctypes
    w, h = 160, 120
    img = sc.synthetic_image(w, h, 3)
    delta = dict(BASE, grain_active=False, dir_couplers_active=True, dir_couplers_amount=amount)
    out = np.zeros((1, h, w, 4), np.uint16)
    neg = np.zeros((h, w, 3), np.float32)
    ex = (ctypes.c_double * 1)(1.0)
    z = (ctypes.c_double * 3)(0, 0, 0)
    ref.check(ref.lib.spkref_render(ref_engine.h, img.ctypes.data_as(sc.FP), w, h, json.dumps(delta).encode(), 0, z,
                                    z, z, ex, 1, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                    neg.ctypes.data_as(sc.FP)))
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert f64["couplers"]["active"]
    got, neg64 = oracle.Oracle(f64).render(img)
    steep, slope = coupler_steep_mask(f64, neg64)
    assert steep.mean() < 0.01
    dn = np.abs(neg64 - neg)
    assert dn[~steep].max() <= 2e-5
    assert dn[steep].max(initial=0) <= slope * 4 * 2.0 ** -23 * 4
    flat = ~steep.any(-1)
    st = lsb_stats(got[flat][None], out[0][flat][None])
    if amount <= 1.0:
        assert st["max"] <= 1, st
    else:
        assert st["frac_gt1"] <= 1e-3 and st["max"] <= 8, st
    # the couplers change the negative
    plain, neg_plain = oracle.Oracle(setup_f64(lib, resources, dict(delta, dir_couplers_active=False),
                                               35000.0 / max(w, h))["f64"]).render(img)
    assert np.abs(neg_plain - neg64).max() > 1e-2
