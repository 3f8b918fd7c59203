"""Parity at the benchmark's own workload (marked gpu: needs a B200).

The 4K render + reprint that the benchmark times, through the C ABI, checked pixel for pixel:

  * 3840 x 2160 linear ProPhoto frame (sc.synthetic_image(3840, 2160, 0)), the synthetic stocks;
  * halation as a 2-Gaussian mixture of sigma 20 and 120 px at weight 0.03 (the block-parallel recursive
    blur at 4K line lengths), scanner lens blur 1.5 px (the fused 5-tap scanner kernel), and grain at a
    film format giving 600 grains per pixel and sub-layer;
  * the render at print_exposure 1.0 and a reprint of the cached negative at 1.2.

Reference call chain: src/session/session.cpp:405-450 -> src/film/develop.cpp:101-236 ->
src/print/run.cpp:101-188, scanner src/fx/scanner.cpp:16-31.

Without grain the device is held to the reference engine itself (oracle/_ref) and to the float64 oracle:
every channel of both images within 1 LSB16. With grain, the float64 oracle takes the device's own Poisson
counts as fixed noise (a binary64 lambda flips counts against a binary32 one) and the same 1 LSB16 gate
applies to the render and to the reprint.
"""

import ctypes
import json

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_gate, sc, setup_f64

pytestmark = pytest.mark.gpu

W, H = 3840, 2160
HEADLINE = dict(BASE, scanner_lens_blur=1.5)
HALATION = ([((1, 1, 1), (20, 20, 20)), ((1, 1, 1), (120, 120, 120))], (0.03, 0.03, 0.03))
GRAINS = 600.0
FIRST_SEED = 0x4ABEA221  # the first draw of a pipeline's seed sequence
EXPOSURES = (1.0, 1.2)


@pytest.fixture(scope="module")
def frame():
    return sc.synthetic_image(W, H, 0)


@pytest.fixture(scope="module")
def film_format(lib, resources):
    """film_format_mm giving a mean of 600 grains per sub-layer and pixel at 3840 px (counts scale with the
    square of the pixel pitch)."""
    p0 = 10.0
    counts = setup_f64(lib, resources, HEADLINE, p0)["f64"]["grain_count"]
    return p0 * (GRAINS / float(np.mean(counts))) ** 0.5 * W / 1000.0


def device_pair(engine, img, delta):
    with engine.open(img, delta) as s:
        s.set_halation(*HALATION)
        a, meta = s.render("full")
        s.set_params({"print_exposure": EXPOSURES[1]})
        b, meta2 = s.reprint("full")
        assert meta["reprint"] == 0 and meta2["reprint"] == 1 and meta2["negative_was_cached"] == 1
        neg, counts = s.develop_debug("full", FIRST_SEED, W, H, counts=bool(delta.get("grain_active", True)))
    return a, b, neg, counts


def oracle_pair(lib, resources, delta, img, counts):
    pitch = delta["film_format_mm"] * 1000.0 / W
    f64 = setup_f64(lib, resources, delta, pitch)["f64"]
    k_reprint = setup_f64(lib, resources, dict(delta, print_exposure=EXPOSURES[1]), pitch)["f64"]["k_gain"]
    o = oracle.Oracle(f64, seed=FIRST_SEED, halation=HALATION)
    a, neg = o.render(img, counts=counts)
    b, _ = o.print(neg, print_exposure=k_reprint)
    return a, b, neg


def test_4k_no_grain(engine, lib, resources, ref, ref_engine, frame, film_format):
    delta = dict(HEADLINE, grain_active=False, film_format_mm=film_format)
    a, b, neg, _ = device_pair(engine, frame, delta)
    # the reference engine itself, same override of the halation mixture
    comps, strength = HALATION
    out = np.zeros((2, H, W, 4), np.uint16)
    neg_ref = np.zeros((H, W, 3), np.float32)
    ref.check(ref.lib.spkref_render(ref_engine.h, frame.ctypes.data_as(sc.FP), W, H, json.dumps(delta).encode(), 2,
                                    (ctypes.c_double * 6)(*[float(v) for c in comps for v in c[0]]),
                                    (ctypes.c_double * 6)(*[float(v) for c in comps for v in c[1]]),
                                    (ctypes.c_double * 3)(*strength), (ctypes.c_double * 2)(*EXPOSURES), 2,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), neg_ref.ctypes.data_as(sc.FP)))
    lsb_gate(a, out[0], "4k nograin render vs reference")
    lsb_gate(b, out[1], "4k nograin reprint vs reference")
    dn = float(np.abs(neg - neg_ref).max())
    assert dn <= 2e-5, dn
    oa, ob, neg64 = oracle_pair(lib, resources, delta, frame, None)
    lsb_gate(a, oa, "4k nograin render vs fp64")
    lsb_gate(b, ob, "4k nograin reprint vs fp64")
    assert float(np.abs(neg - neg64).max()) <= 2e-5


def test_4k_grain_fixed_noise(engine, lib, resources, frame, film_format):
    delta = dict(HEADLINE, grain_active=True, film_format_mm=film_format)
    a, b, neg, counts = device_pair(engine, frame, delta)
    assert float(counts.mean()) > 10.0 and float(counts.max()) > GRAINS  # the grain path ran at this pitch
    oa, ob, neg64 = oracle_pair(lib, resources, delta, frame, counts)
    lsb_gate(a, oa, "4k grain render vs fp64 (fixed noise)")
    lsb_gate(b, ob, "4k grain reprint vs fp64 (fixed noise)")
    assert float(np.abs(neg - neg64).max()) <= 5e-5
