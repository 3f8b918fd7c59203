"""The film side's highlight stages on the CPU: the highlight boost (reference src/film/develop.cpp:32-62)
and the back-reflection halation with its headroom (src/fx/halation.cpp:64-86, used when the
anti-halation layer is removed), in the float64 oracle against the reference's own spk_render."""

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_tiers_cpu import ref_render

CASES = {
    "boost_1.5": {"halation_boost_ev": 1.5},
    "boost_4": {"halation_boost_ev": 4.0},
    "backref_headroom_4": {"antihalation_removed": True},
    "backref_headroom_2": {"antihalation_removed": True, "halation_headroom_ev": 2.0},
    "backref_no_headroom": {"antihalation_removed": True, "halation_headroom_ev": 0.0},
    "boost_and_headroom": {"antihalation_removed": True, "halation_boost_ev": 2.0},
}


def bright_image(w, h, seed):
    img = sc.synthetic_image(w, h, seed)
    img[h // 3: h // 3 + 12, w // 4: w // 4 + 20] = 60.0  # a highlight to lift and to halate
    return np.ascontiguousarray(img, np.float32)


@pytest.mark.parametrize("case", sorted(CASES))
def test_highlights_against_reference(lib, resources, ref, ref_engine, case):
    w, h = 192, 128
    img = bright_image(w, h, 91)
    delta = dict(BASE, grain_active=False, **CASES[case])
    want = ref_render(ref_engine, img, delta, "full")
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    got, _ = oracle.Oracle(f64).render(img)
    st = lsb_stats(got, want)
    assert st["max"] <= 1, st
