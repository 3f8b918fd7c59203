"""The EDR tone map on the device (marked gpu): against the reference's own spk_render within 1 LSB16
(both binary32, the same operations in the same order), on the tiled scanner and on the separate
encode (a large unsharp radius), and the refusal of a profile without a tone map."""

import numpy as np
import pytest

from conftest import BASE, lsb_stats, sc
from test_tiers_cpu import ref_render

pytestmark = pytest.mark.gpu


def edr_image(w, h, seed):
    img = sc.synthetic_image(w, h, seed)
    img[h // 3: h // 3 + 20, w // 4: w // 4 + 40] = 40.0
    return np.ascontiguousarray(img, np.float32)


@pytest.mark.parametrize("extra", [{}, {"print_exposure": 2.5}, {"output_color_space": "sRGB"},
                                   {"preview_long_edge": 800}])
def test_edr_within_one_lsb(engine, ref, ref_engine, extra):
    img = edr_image(1000, 640, 112)
    delta = dict(BASE, grain_active=False, extended_dynamic_range=True, **extra)
    tier = "live" if "preview_long_edge" in extra else "full"
    with engine.open(img, delta) as s:
        a, _ = s.render(tier)
    assert lsb_stats(a, ref_render(ref_engine, img, delta, tier))["max"] <= 1


def test_edr_on_a_scanned_negative_is_off(engine, ref, ref_engine):
    img = edr_image(160, 100, 113)
    delta = dict(BASE, grain_active=False, extended_dynamic_range=True, scan_film=True)
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
    assert lsb_stats(a, ref_render(ref_engine, img, delta, "full"))["max"] <= 1
