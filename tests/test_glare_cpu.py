"""Print glare on the CPU (reference src/fx/glare.cpp:27-50, kernels/fx_glare.metal): the float64 oracle
against the reference engine's own spk_render. The glare draws the print seed, the first draw of a fresh
seed sequence when the grain is off; its lognormal field comes from the sampler shared with the device."""

import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64
from test_tiers_cpu import ref_render

FIRST_SEED = 0x4ABEA221  # the first draw of a pipeline's seed sequence


@pytest.mark.parametrize("amount", [1.0, 4.0, 30.0])
def test_glare_against_reference(lib, resources, ref, ref_engine, amount):
    w, h = 192, 128
    img = sc.synthetic_image(w, h, 51)
    delta = dict(BASE, grain_active=False, glare_active=True, glare_amount=amount)
    want = ref_render(ref_engine, img, delta, "full")
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert f64["glare"]["draws"]
    got, _ = oracle.Oracle(f64, print_seed=FIRST_SEED).render(img)
    assert lsb_stats(got, want)["max"] <= 1
    plain, _ = oracle.Oracle(setup_f64(lib, resources, dict(delta, glare_active=False), 35000.0 / max(w, h))["f64"]
                             ).render(img)
    assert lsb_stats(plain, want)["max"] > 1  # the glare shows


def test_glare_off_on_a_scanned_negative(lib, resources, ref, ref_engine):
    """scan_film: the print seed is drawn but no glare is added."""
    w, h = 96, 64
    img = sc.synthetic_image(w, h, 52)
    delta = dict(BASE, grain_active=False, glare_active=True, scan_film=True)
    want = ref_render(ref_engine, img, delta, "full")
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    assert not f64["glare"]["draws"]
    got, _ = oracle.Oracle(f64).render(img)
    assert lsb_stats(got, want)["max"] <= 1
