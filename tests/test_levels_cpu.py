"""Scanner levels on the CPU (reference src/print/setup.cpp:262-390, kernels/print.metal:234-246): the
black and white corrections, alone and together, in the float64 oracle against the reference's own
spk_render; the correction changes the print's gain (kappa) to keep mid grey."""

import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_tiers_cpu import ref_render

LEVELS = {"black": {"scanner_black_correction": True}, "white": {"scanner_white_correction": True},
          "both": {"scanner_black_correction": True, "scanner_white_correction": True}}


@pytest.mark.parametrize("case", sorted(LEVELS))
def test_levels_against_reference(lib, resources, ref, ref_engine, case):
    w, h = 192, 128
    img = sc.synthetic_image(w, h, 101)
    delta = dict(BASE, grain_active=False, **LEVELS[case])
    want = ref_render(ref_engine, img, delta, "full")
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert f64["levels"]["active"]
    got, _ = oracle.Oracle(f64).render(img)
    assert lsb_stats(got, want)["max"] <= 1
    plain = ref_render(ref_engine, img, dict(delta, scanner_black_correction=False, scanner_white_correction=False),
                       "full")
    assert lsb_stats(plain, want)["max"] > 1  # the levels show


def test_levels_pass_through_a_scanned_negative(lib, resources, ref, ref_engine):
    w, h = 96, 64
    img = sc.synthetic_image(w, h, 102)
    delta = dict(BASE, grain_active=False, scan_film=True, **LEVELS["both"])
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert not f64["levels"]["active"]
    got, _ = oracle.Oracle(f64).render(img)
    assert lsb_stats(got, ref_render(ref_engine, img, delta, "full"))["max"] <= 1
