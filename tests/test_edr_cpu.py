"""The EDR tone map on the CPU (reference kernels/print.metal:319-347, src/print/build.cpp:83-85, :210-222):
the float64 oracle against the reference's own spk_render, and the refusal of a paper without a tone map."""

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_tiers_cpu import ref_render


@pytest.mark.parametrize("extra", [{}, {"print_exposure": 2.5}, {"output_color_space": "sRGB"}])
def test_edr_against_reference(lib, resources, ref, ref_engine, extra):
    w, h = 192, 128
    img = sc.synthetic_image(w, h, 111)
    img[40:60, 50:90] = 40.0  # highlights above the shoulder
    img = np.ascontiguousarray(img, np.float32)
    delta = dict(BASE, grain_active=False, extended_dynamic_range=True, **extra)
    want = ref_render(ref_engine, img, delta, "full")
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert f64["edr"]["active"]
    got, _ = oracle.Oracle(f64).render(img)
    # within 1 LSB16 where the reference's channels are all away from the ends of the encode range; in
    # saturated colours the tone map's y' / y amplifies the rounding of a small luminance y
    d = np.abs(got.astype(np.int64) - want.astype(np.int64))[..., :3].max(-1)
    inside = ((want[..., :3] >= 4096) & (want[..., :3] <= 61439)).all(-1)
    assert d[inside].max(initial=0) <= 1
    assert (d > 1).mean() <= 2e-3
    plain = ref_render(ref_engine, img, dict(delta, extended_dynamic_range=False), "full")
    assert lsb_stats(plain, want)["max"] > 1  # the tone map shows
