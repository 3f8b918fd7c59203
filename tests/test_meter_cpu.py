"""The auto-exposure meter on the CPU (reference src/film/meter.cpp:45-120): the float64 oracle's meter
against the reference's own meter_values on the same images, and renders with auto exposure through the
reference's C ABI against the oracle (meter image = the frame at a 1600 px long edge, then decode and
geometry; the develop scales the RGB by f32(2^EV) of the session's method)."""

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_tiers_cpu import GEOMETRIES, encoded, ref_render

METHODS = oracle.METER_METHODS


def meter_image(w, h, seed):
    """A frame with a sky, a bright patch and some pixels below the meter's floor."""
    img = sc.synthetic_image(w, h, seed)
    img[: h // 4] *= 3.0
    img[h // 2: h // 2 + 8, w // 3: w // 3 + 16] = 20.0
    img[-3:, :5] = 0.0
    return np.ascontiguousarray(img, np.float32)


@pytest.mark.parametrize("w,h", [(1600, 900), (333, 517), (64, 1), (1, 1), (2, 2)])
def test_meter_against_reference(lib, resources, ref, w, h):
    img = meter_image(w, h, 31)
    m = setup_f64(lib, resources, BASE, 10.0)["f64"]["input_rgb_to_xyz"]
    want = sc.reference_meter(ref, img, m)
    got = oracle.meter(img, m)
    for k in METHODS:
        assert got[k] == pytest.approx(want[k], abs=1e-9), k


def oracle_render_ae(lib, resources, img, delta, long_edge=0):
    """The oracle's render with the meter: the meter image (1600 px), decode + geometry, the EV of the
    delta's method, the RGB scaled by f32(2^EV) before the develop."""
    h, w, _ = img.shape
    tier = oracle.downscale(img, long_edge)
    th, tw, _ = tier.shape
    f64 = setup_f64(lib, resources, delta, 1000.0 * delta.get("film_format_mm", 35.0) / max(tw, th))["f64"]
    mimg = oracle.prepare(oracle.downscale(img, 1600), delta, f64["input_cctf_mode"])
    ev = oracle.meter(mimg, f64["input_rgb_to_xyz"])[delta.get("auto_exposure_method", "center_weighted")]
    gain = float(np.float32(2.0 ** ev))
    prepared = oracle.prepare(tier, delta, f64["input_cctf_mode"]) * gain
    return oracle.Oracle(f64, rho_tier=max(tw, th) / max(w, h)).render64(prepared)


@pytest.mark.parametrize("method", METHODS)
def test_auto_exposure_render_against_reference(lib, resources, ref, ref_engine, method):
    img = meter_image(240, 160, 32)
    delta = dict(BASE, grain_active=False, auto_exposure=True, auto_exposure_method=method)
    want = ref_render(ref_engine, img, delta, "full")
    got, _ = oracle_render_ae(lib, resources, img, delta)
    assert lsb_stats(got, want)["max"] <= 1


def test_auto_exposure_with_downscale_decode_geometry(lib, resources, ref, ref_engine):
    """A 2000 x 1200 frame: the meter on its own 1600 px downscale, through decode and a rotation."""
    img = encoded(meter_image(2000, 1200, 33))
    delta = dict(BASE, grain_active=False, auto_exposure=True, input_cctf_decoding=True, preview_long_edge=900,
                 **GEOMETRIES["rotate"])
    want = ref_render(ref_engine, img, delta, "live")
    got, _ = oracle_render_ae(lib, resources, img, delta, 900)
    assert lsb_stats(got, want)["max"] <= 1
