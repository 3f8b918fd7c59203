"""The auto-exposure meter on the device (marked gpu): its seven EV values against the reference's own
meter_values on the same meter image (the tier downscale is bit-exact, so the image is the same), and
renders with auto exposure through the C ABI against the reference engine, within 1 LSB16 without grain."""

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_meter_cpu import METHODS, meter_image, oracle_render_ae
from test_tiers_cpu import GEOMETRIES, encoded, ref_render

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("w,h", [(1600, 900), (2400, 1350), (333, 517), (3, 1)])
def test_meter_values_against_reference(engine, lib, resources, ref, w, h):
    img = meter_image(w, h, 41)
    delta = dict(BASE, auto_exposure=True)
    with engine.open(img, delta) as s:
        got = s.meter()
    m = setup_f64(lib, resources, delta, 10.0)["f64"]["input_rgb_to_xyz"]
    want = sc.reference_meter(ref, oracle.downscale(img, 1600), m)
    for k in METHODS:
        assert got[k] == pytest.approx(want[k], abs=1e-9), (k, got[k], want[k])


def test_meter_with_decode_and_geometry(engine, lib, resources):
    img = encoded(meter_image(1800, 1000, 42))
    delta = dict(BASE, auto_exposure=True, input_cctf_decoding=True, **GEOMETRIES["all"])
    with engine.open(img, delta) as s:
        got = s.meter()
    f64 = setup_f64(lib, resources, delta, 10.0)["f64"]
    want = oracle.meter(oracle.prepare(oracle.downscale(img, 1600), delta, f64["input_cctf_mode"]),
                        f64["input_rgb_to_xyz"])
    for k in METHODS:
        assert got[k] == pytest.approx(want[k], abs=1e-5), k


@pytest.mark.parametrize("method", METHODS)
def test_auto_exposure_render_within_one_lsb(engine, ref, ref_engine, method):
    img = meter_image(240, 160, 43)
    delta = dict(BASE, grain_active=False, auto_exposure=True, auto_exposure_method=method)
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
    assert lsb_stats(a, ref_render(ref_engine, img, delta, "full"))["max"] <= 1


def test_auto_exposure_live_tier_within_one_lsb(engine, lib, resources, ref, ref_engine):
    """A 2000 x 1200 frame on the live tier at 1600 px (the meter reads the live tier's image) and at 900 px
    (its own downscale), with decode and a rotation: within 1 LSB16 of the reference; the float64 oracle's
    gate as elsewhere."""
    img = encoded(meter_image(2000, 1200, 44))
    for L in (1600, 900):
        delta = dict(BASE, grain_active=False, auto_exposure=True, input_cctf_decoding=True, preview_long_edge=L,
                     **GEOMETRIES["rotate"])
        with engine.open(img, delta) as s:
            a, _ = s.render("live")
        assert lsb_stats(a, ref_render(ref_engine, img, delta, "live"))["max"] <= 1
        # binary32 against the float64 oracle (decode and a rotation before the develop): the FP64 gate
        st = lsb_stats(a, oracle_render_ae(lib, resources, img, delta, L)[0])
        assert st["n_gt1"] <= 4 and st["max"] <= 2, st  # measured: three channels at 2 LSB16 in 12 M


def test_meter_rearms_on_its_key(engine):
    img = meter_image(800, 600, 45)
    with engine.open(img, dict(BASE, grain_active=False, auto_exposure=True)) as s:
        m1 = s.meter()
        s.set_params({"print_exposure": 1.3})  # not in the meter's key
        assert s.meter() == m1
        s.set_params({"geometry_crop_w": 0.5})  # in the key: metered again, on the cropped image
        m2 = s.meter()
        assert m2["average"] != m1["average"]
        s.set_params({"geometry_crop_w": 1.0})
        assert s.meter() == m1
    with engine.open(img, dict(BASE, auto_exposure=False)) as s:
        with pytest.raises(sc.SpkError):
            s.meter()
