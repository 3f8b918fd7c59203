"""The highlight boost and the back-reflection halation with its headroom on the device (marked gpu),
against the reference's own spk_render within 1 LSB16 without grain, and the float64 oracle's gate with
the device's grain counts as fixed noise."""

import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_highlights_cpu import CASES, bright_image
from test_tiers_cpu import ref_render

pytestmark = pytest.mark.gpu
FIRST_SEED = 0x4ABEA221


@pytest.mark.parametrize("case", sorted(CASES))
def test_highlights_within_one_lsb(engine, ref, ref_engine, case):
    img = bright_image(256, 176, 92)
    delta = dict(BASE, grain_active=False, **CASES[case])
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
    assert lsb_stats(a, ref_render(ref_engine, img, delta, "full"))["max"] <= 1


def test_highlights_fp64_gate_with_grain(engine, lib, resources):
    w, h = 512, 384
    img = bright_image(w, h, 93)
    delta = dict(BASE, grain_active=True, **CASES["boost_and_headroom"])
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
        _, counts = s.develop_debug("full", FIRST_SEED, w, h)
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    out, _ = oracle.Oracle(f64, seed=FIRST_SEED).render(img, counts=counts)
    st = lsb_stats(a, out)
    assert st["max"] <= 1, st


def test_boost_of_a_black_frame(engine, ref, ref_engine):
    """A frame whose maximum is 0: the boost scales it by 0 (the reference's M = 0 case)."""
    img = sc.synthetic_image(64, 48, 94) * 0.0
    delta = dict(BASE, grain_active=False, halation_boost_ev=2.0)
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
    assert lsb_stats(a, ref_render(ref_engine, img, delta, "full"))["max"] <= 1
