"""Parity of the CUDA render path with the oracles, through the C ABI (marked gpu: needs a B200).

  * against the reference engine itself (its stage code and kernels run on the CPU, oracle/_ref, or the
    stored golden renders): every pixel within 1 LSB16 without grain;
  * against the float64 oracle with the grain held as fixed noise (the device's own Poisson counts):
    the final RGBA16 within 1 LSB16 on (nearly) every pixel;
  * the sampler, Philox and the blurs at the stage level.
"""

import json
import os

import numpy as np
import pytest

import oracle
from conftest import BASE, GOLDEN, coupler_steep_mask, golden, lsb_stats, sc, setup_f64

pytestmark = pytest.mark.gpu
CFG1 = ([((1, 1, 1), (8, 8, 8)), ((1, 1, 1), (40, 40, 40))], (0.02, 0.02, 0.02))
FIRST_SEED = 0x4ABEA221  # the first draw of a pipeline's seed sequence


def render_pair(engine, img, delta, halation=None, exposure2=1.2):
    with engine.open(img, delta) as s:
        if halation:
            s.set_halation(*halation)
        a, meta = s.render("full")
        s.set_params({"print_exposure": exposure2})
        b, meta2 = s.reprint("full")
        assert meta["reprint"] == 0 and meta["negative_was_cached"] == 0
        assert meta2["reprint"] == 1 and meta2["negative_was_cached"] == 1
        return a, b


def test_golden_renders(engine):
    meta = json.load(open(os.path.join(GOLDEN, "golden_renders.json")))
    g = golden("golden_renders.npz")
    img = g["image"]
    for name, case in meta["cases"].items():
        hal = case["halation"]
        a, b = render_pair(engine, img, case["delta"], (hal[0], hal[1]) if hal else None, meta["exposures"][1])
        ref = g[f"{name}_rgba"]
        if not case["delta"].get("grain_active", True):
            assert lsb_stats(a, ref[0])["max"] <= 1, name
            assert lsb_stats(b, ref[1])["max"] <= 1, name
        else:
            # grain against the reference's own draws: its sampler's host log and exp flip a few Poisson
            # counts against ours (the fixed-noise float64 gates hold the same renders to 1 LSB16); measured
            # 12.7 % of the channels of this 64 x 48 frame for the preset, less with the cfg1 halation
            assert lsb_stats(a, ref[0])["frac_gt1"] < 0.15, name
        assert (a[..., 3] == 65535).all()


@pytest.mark.parametrize("w,h", [(256, 192), (97, 61), (3, 2), (1, 17)])
def test_no_grain_within_one_lsb_of_reference(engine, ref, ref_engine, w, h):
    import ctypes
    img = sc.synthetic_image(w, h, 3)
    delta = dict(BASE, grain_active=False)
    a, b = render_pair(engine, img, delta)
    out = np.zeros((2, h, w, 4), np.uint16)
    neg = np.zeros((h, w, 3), np.float32)
    ex = (ctypes.c_double * 2)(1.0, 1.2)
    z = (ctypes.c_double * 3)(0, 0, 0)
    ref.check(ref.lib.spkref_render(ref_engine.h, img.ctypes.data_as(sc.FP), w, h, json.dumps(delta).encode(), 0, z,
                                    z, z, ex, 2, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                    neg.ctypes.data_as(sc.FP)))
    assert lsb_stats(a, out[0])["max"] <= 1
    assert lsb_stats(b, out[1])["max"] <= 1


@pytest.mark.parametrize("case", ["nograin", "grain_preset", "grain_cfg1"])
def test_fp64_gate_fixed_noise(engine, lib, resources, case):
    w, h = 512, 512
    img = sc.synthetic_image(w, h, 0)
    delta = dict(BASE, grain_active=case != "nograin")
    hal = CFG1 if case == "grain_cfg1" else None
    with engine.open(img, delta) as s:
        if hal:
            s.set_halation(*hal)
        a, _ = s.render("full")
        neg, counts = s.develop_debug("full", FIRST_SEED, w, h)
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    o = oracle.Oracle(f64, seed=FIRST_SEED, halation=hal)
    out, neg64 = o.render(img, counts=counts)
    st = lsb_stats(a, out)
    # binary32 device arithmetic against binary64: at most 1 LSB16 on every channel but two (measured: one
    # channel at 2 LSB16 in 786,432 without grain and with the cfg1 halation, none with the preset)
    assert st["n_gt1"] <= 2 and st["max"] <= 2, st
    np.testing.assert_allclose(neg, neg64, rtol=0, atol=5e-5)


@pytest.mark.parametrize("amount", [0.5, 1.0])
def test_couplers_within_one_lsb_of_reference(engine, lib, resources, ref, ref_engine, amount):
    """DIR couplers (reference src/film/develop.cpp:203-226) on the device against the reference engine,
    without grain: render and reprint within 1 LSB16 on every pixel whose negative the pre-inverted curve
    does not reach through its fold, the negatives within 2e-5 there (coupler_steep_mask)."""
    import ctypes
    w, h = 200, 136
    img = sc.synthetic_image(w, h, 3)
    delta = dict(BASE, grain_active=False, dir_couplers_active=True, dir_couplers_amount=amount)
    a, b = render_pair(engine, img, delta)
    with engine.open(img, delta) as s:
        neg_dev, _ = s.develop_debug("full", FIRST_SEED, w, h)
    out = np.zeros((2, h, w, 4), np.uint16)
    neg = np.zeros((h, w, 3), np.float32)
    ex = (ctypes.c_double * 2)(1.0, 1.2)
    z = (ctypes.c_double * 3)(0, 0, 0)
    ref.check(ref.lib.spkref_render(ref_engine.h, img.ctypes.data_as(sc.FP), w, h, json.dumps(delta).encode(), 0, z,
                                    z, z, ex, 2, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                    neg.ctypes.data_as(sc.FP)))
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    steep, _ = coupler_steep_mask(f64, neg)
    assert steep.mean() < 0.01
    assert np.abs(neg_dev - neg)[~steep].max() <= 2e-5
    flat = ~steep.any(-1)
    assert lsb_stats(a[flat][None], out[0][flat][None])["max"] <= 1
    assert lsb_stats(b[flat][None], out[1][flat][None])["max"] <= 1


def test_couplers_fp64_gate_fixed_noise(engine, lib, resources):
    """DIR couplers with grain against the float64 oracle, the device's own Poisson counts as fixed noise:
    the RGBA within 1 LSB16 on all but a handful of pixels away from the pre-inverted curve's fold (the
    developed density, before the grain, inside the fold's steep segment; widened by the final blur's
    radius of 2 pixels, which spreads the fold's binary32 differences to the neighbours)."""
    from scipy.ndimage import binary_dilation
    w, h = 384, 256
    img = sc.synthetic_image(w, h, 0)
    delta = dict(BASE, grain_active=True, dir_couplers_active=True, dir_couplers_amount=1.0)
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
        neg, counts = s.develop_debug("full", FIRST_SEED, w, h)
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    out, neg64 = oracle.Oracle(f64, seed=FIRST_SEED).render(img, counts=counts)
    plain = setup_f64(lib, resources, dict(delta, grain_active=False), 35000.0 / max(w, h))["f64"]
    fold = coupler_steep_mask(plain, oracle.Oracle(plain).render(img)[1])[0].any(-1)
    flat = ~binary_dilation(fold, np.ones((5, 5), bool))
    st = lsb_stats(a[flat][None], out[flat][None])
    d = np.abs(a.astype(np.int64) - out.astype(np.int64))[..., :3].max(-1)
    info = dict(st, fold=float(fold.mean()), flat=float(flat.mean()), gt1_all=int((d > 1).sum()),
                gt1_fold=int((d[fold] > 1).sum()), gt1_flat=int((d[flat] > 1).sum()),
                neg_flat=float(np.abs(neg - neg64)[flat].max()))
    assert st["max"] <= 1, info
    assert fold.mean() < 0.02 and flat.mean() > 0.75, info  # the fold is a thin contour; widened, a sixth of the frame


def test_sampler_bit_exact(lib):
    import ctypes
    lam = np.repeat(np.array([0.0, 0.5, 3.0, 9.99, 10.0, 37.0, 150.0, 600.0, 2500.0, 1e5], np.float32), 4096)
    dev = np.zeros_like(lam)
    lib.check(lib.lib.spkx_sampler_poisson(lam.ctypes.data_as(sc.FP), dev.ctypes.data_as(sc.FP), lam.size, 7, 1))
    host = oracle.poisson(lam, 7, 1)
    assert np.array_equal(dev, host)
    ln = np.zeros(50000, np.float32)
    lib.check(lib.lib.spkx_sampler_lognormal(ln.ctypes.data_as(sc.FP), ln.size, 1.0, 0.2, 100, 9))
    assert np.array_equal(ln, oracle.lognormal(ln.size, 1.0, 0.2, 100, 9))


def film_format_for(lib, resources, grains, long_edge):
    """film_format_mm giving a mean of `grains` grains per sub-layer and pixel (counts scale with the
    square of the pixel pitch)."""
    import ctypes
    p0 = 10.0
    out = ctypes.c_char_p()
    lib.check(lib.lib.spkx_setup_json(resources.encode(), json.dumps(BASE).encode(), p0, ctypes.byref(out)))
    counts = lib.take_json(out)["f64"]["grain_count"]
    return p0 * (grains / float(np.mean(counts))) ** 0.5 * long_edge / 1000.0


# (the film format stays within the schema's 4..200 mm: a wide frame for the fine pitch of 40 grains, which
# still stays above the pitch where dye clouds begin)
@pytest.mark.parametrize("w,h,seed,grains", [(300, 200, FIRST_SEED, 600.0), (401, 73, 12345, 600.0),
                                             (800, 48, 99, 40.0)])
def test_develop_draws_match_sampler(engine, lib, resources, w, h, seed, grains):
    """Every grain draw of the develop kernel (its first attempts run in lockstep, the rest deferred and
    finished apart) equals the shared sampler's count for the same lambda, pixel, stream and seed; at 40
    grains per pixel the low densities take the product method (lambda < 10)."""
    img = sc.synthetic_image(w, h, 5)
    delta = dict(BASE, grain_active=True, film_format_mm=film_format_for(lib, resources, grains, max(w, h)))
    with engine.open(img, delta) as s:
        s.set_halation(*CFG1)
        counts, lam = s.develop_draws("full", seed, w, h)
    assert (lam >= 10).any()
    if grains < 100:
        assert (lam < 10).any()
    for c in range(3):
        for l in range(3):
            want = oracle.poisson(lam[..., c * 3 + l].ravel(), c + 10 * l, seed)
            assert np.array_equal(counts[..., c * 3 + l].ravel(), want), (c, l)


def test_philox_on_device(lib):
    rng = np.random.default_rng(0)
    ctr = rng.integers(0, 2 ** 32, (1024, 4), dtype=np.uint64).astype(np.uint32)
    key = rng.integers(0, 2 ** 32, (1024, 2), dtype=np.uint64).astype(np.uint32)
    ctr[0] = (0, 0, 0, 0)
    key[0] = (0, 0)
    ctr[1] = (0, 200, 0, 0)
    key[1] = (0x5EED, 0)
    out = np.zeros_like(ctr)
    U = sc.UP
    lib.check(lib.lib.spkx_philox(ctr.ctypes.data_as(U), key.ctypes.data_as(U), out.ctypes.data_as(U), 1024))
    assert np.array_equal(out, oracle.philox(ctr, key))
    assert tuple(out[0]) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert tuple(out[1]) == (0x15CECB3F, 0xF63DFA39, 0x3EC2DC0E, 0xF78F6C18)


@pytest.mark.parametrize("shape", [(61, 97), (1, 40), (40, 1), (2, 3), (300, 257)])
@pytest.mark.parametrize("sigma", [(0.65, 0.65, 0.65), (1.5, 2.9, 0.3), (3.0, 8.0, 40.0), (20.0, 120.0, 0.0),
                                   (2.5, 3.5, 1.0)])
def test_gaussian_against_fp64(lib, shape, sigma):
    import ctypes
    h, w = shape
    rng = np.random.default_rng(h * 1000 + w)
    plane = rng.random((h, w, 3), dtype=np.float32) + 0.1
    out = np.zeros_like(plane)
    s3 = (ctypes.c_double * 3)(*sigma)
    lib.check(lib.lib.spkx_gaussian(plane.ctypes.data_as(sc.FP), out.ctypes.data_as(sc.FP), w, h, s3))
    want = oracle.gaussian(plane, sigma)
    rel = np.abs(out - want) / np.abs(want)
    for c in range(3):
        tol = 1e-5 if sigma[c] >= 3 else 2e-6  # the reference's tolerances (tests/test_fx.cpp:200)
        assert rel[..., c].max() <= tol, (c, rel[..., c].max())


def test_gaussian_golden(lib):
    import ctypes
    g = golden("golden_gaussian.npz")
    plane = g["plane"]
    h, w, _ = plane.shape
    for k in range(3):
        sig = g[f"s{k}_sigma"]
        out = np.zeros_like(plane)
        lib.check(lib.lib.spkx_gaussian(plane.ctypes.data_as(sc.FP), out.ctypes.data_as(sc.FP), w, h,
                                        (ctypes.c_double * 3)(*sig)))
        ref = g[f"s{k}_mode1"]  # the reference's same-order binary64-state copy
        rel = np.abs(out - ref) / np.maximum(np.abs(ref), 1e-6)
        assert rel.max() <= 4e-6, (k, rel.max())
