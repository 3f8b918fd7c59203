"""The steps before the film path, on the CPU: the tier downscale, the input transfer decode and the
geometry, in the float64 oracle against the reference engine built for the CPU (oracle/_ref).

  * the downscale is specified in binary32 with fused multiply-adds in a fixed order (reference
    src/session/tiers.cpp:1-10): the oracle's restatement gives the reference's bits;
  * decode + geometry + the whole render, through the reference's own C ABI (spk_open / spk_render on
    the live and full tiers) against the oracle: within 1 LSB16 without grain.
"""

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64


@pytest.mark.parametrize("w,h,L", [(1000, 600, 800), (640, 480, 100), (97, 61, 40), (3, 200, 17), (1, 50, 7),
                                   (513, 257, 256), (300, 300, 299)])
def test_downscale_bit_exact_with_reference(ref, w, h, L):
    img = sc.synthetic_image(w, h, 7)
    got = oracle.downscale(img, L)
    want = sc.reference_downscale(ref, img, L)
    assert got.shape == want.shape == (*oracle.downscale_size(w, h, L)[::-1], 3)
    assert np.array_equal(got, want)


def test_downscale_size_rules():
    # floor of each side, the long edge may land one short (reference src/session/tiers.hpp:42-44)
    assert oracle.downscale_size(2156, 1000, 1600) == (1599, 742)
    assert oracle.downscale_size(800, 600, 800) == (800, 600)
    assert oracle.downscale_size(5000, 2, 1000) == (1000, 1)


def ref_render(ref_engine, img, delta, tier):
    with ref_engine.open(img, delta) as s:
        out, _ = s.render(tier)
    return out


def oracle_render(lib, resources, img, delta, long_edge, seed=0, counts=None):
    """decode + geometry + render in the oracle at the tier's long edge (0: the frame)."""
    h, w, _ = img.shape
    tier = oracle.downscale(img, long_edge)
    th, tw, _ = tier.shape
    rho = max(tw, th) / max(w, h)
    f64 = setup_f64(lib, resources, delta, 1000.0 * delta.get("film_format_mm", 35.0) / max(tw, th))["f64"]
    prepared = oracle.prepare(tier, delta, f64["input_cctf_mode"])
    return oracle.Oracle(f64, seed=seed, rho_tier=rho).render64(prepared, counts)


GEOMETRIES = {
    "crop": {"geometry_crop_x": 0.1, "geometry_crop_y": 0.2, "geometry_crop_w": 0.7, "geometry_crop_h": 0.5},
    "rotate": {"geometry_rotation_deg": 7.5},
    "turn_flip": {"geometry_quarter_turns": 1, "geometry_flip_h": True},
    "all": {"geometry_crop_x": 0.05, "geometry_crop_w": 0.9, "geometry_crop_h": 0.8, "geometry_rotation_deg": -12.0,
            "geometry_quarter_turns": 3, "geometry_flip_v": True},
}


def encoded(img, gamma=1 / 1.8):
    """An encoded-looking input in [0, 1] for the decode tests."""
    return np.ascontiguousarray(np.clip(img, 0.0, 1.0) ** gamma, np.float32)


@pytest.mark.parametrize("geo", sorted(GEOMETRIES))
@pytest.mark.parametrize("decode", [False, True])
def test_decode_geometry_against_reference(lib, resources, ref, ref_engine, geo, decode):
    w, h = 160, 112
    img = sc.synthetic_image(w, h, 11)
    if decode:
        img = encoded(img)
    delta = dict(BASE, grain_active=False, input_cctf_decoding=decode, **GEOMETRIES[geo])
    want = ref_render(ref_engine, img, delta, "full")
    got, _ = oracle_render(lib, resources, img, delta, 0)
    assert got.shape == want.shape
    st = lsb_stats(got, want)
    assert st["max"] <= 1, st


@pytest.mark.parametrize("space", ["sRGB", "Adobe RGB (1998)", "ITU-R BT.709"])
def test_decode_spaces_against_reference(lib, resources, ref, ref_engine, space):
    w, h = 96, 64
    img = encoded(sc.synthetic_image(w, h, 12), 0.45)
    delta = dict(BASE, grain_active=False, input_cctf_decoding=True, input_color_space=space)
    want = ref_render(ref_engine, img, delta, "full")
    got, _ = oracle_render(lib, resources, img, delta, 0)
    assert lsb_stats(got, want)["max"] <= 1


def test_live_tier_against_reference(lib, resources, ref, ref_engine):
    """The live tier of a 1000 x 700 frame at preview_long_edge 800 (the schema's smallest): downscale,
    pitch at the tier's long edge, the unsharp mask scaled by rho."""
    w, h = 1000, 700
    img = sc.synthetic_image(w, h, 13)
    delta = dict(BASE, grain_active=False, preview_long_edge=800)
    want = ref_render(ref_engine, img, delta, "live")
    assert want.shape == (560, 800, 4)
    got, _ = oracle_render(lib, resources, img, delta, 800)
    assert lsb_stats(got, want)["max"] <= 1
