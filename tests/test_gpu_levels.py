"""Scanner levels on the device (marked gpu): renders and a reprint at a new print exposure against the
reference's own spk_render / spk_reprint within 1 LSB16, on the binary32 kernel and the spectral-mode
kernels, and in a batch."""

import numpy as np
import pytest

from conftest import BASE, lsb_stats, sc
from test_levels_cpu import LEVELS

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(LEVELS))
def test_levels_render_and_reprint(engine, ref, ref_engine, case):
    img = sc.synthetic_image(256, 176, 103)
    delta = dict(BASE, grain_active=False, **LEVELS[case])
    out = []
    for eng in (engine, ref_engine):
        with eng.open(img, delta) as s:
            a, _ = s.render("full")
            s.set_params({"print_exposure": 1.25})
            b, _ = s.reprint("full")
        out.append((a, b))
    assert lsb_stats(out[0][0], out[1][0])["max"] <= 1
    assert lsb_stats(out[0][1], out[1][1])["max"] <= 1


def test_levels_on_the_spectral_kernel(engine):
    img = sc.synthetic_image(200, 136, 104)
    delta = dict(BASE, grain_active=False, **LEVELS["both"])
    with engine.open(img, delta) as s:
        a, _ = s.render("full")
        s.set_print_mode("fp64")
        b, _ = s.reprint("full")
    assert lsb_stats(a, b)["max"] <= 1


def test_levels_in_a_batch(engine):
    delta = dict(BASE, grain_active=False, **LEVELS["white"])
    imgs = [sc.synthetic_image(320, 200, 105 + k) for k in range(3)]
    singles = []
    for img in imgs:
        with engine.open(img, delta) as s:
            singles.append(s.render("full")[0])
    sessions = [engine.open(img, delta) for img in imgs]
    try:
        outs, _ = engine.render_batch(sessions, "full")
        for r, b in zip(outs, singles):
            assert np.array_equal(r.pixels, b)
            r.free()
    finally:
        for s in sessions:
            s.close()
