"""Print glare on the device (marked gpu), through the C ABI: renders and reprints against the reference
engine's own spk_render / spk_reprint (each draws the next print seed), on the full and live tiers and
in batches, within 1 LSB16 without grain; with grain, the film seed and the print seed come from the
same sequence in the reference's order."""

import numpy as np
import pytest

from conftest import BASE, lsb_stats, sc

pytestmark = pytest.mark.gpu


def render_reprints(session, tier, exposures):
    out = [session.render(tier)[0]]
    for e in exposures:
        session.set_params({"print_exposure": e})
        out.append(session.reprint(tier)[0])
    return out


@pytest.mark.parametrize("amount", [1.0, 6.0])
def test_glare_render_and_reprints_within_one_lsb(engine, ref, ref_engine, amount):
    w, h = 256, 176
    img = sc.synthetic_image(w, h, 53)
    delta = dict(BASE, grain_active=False, glare_active=True, glare_amount=amount)
    with engine.open(img, delta) as s:
        got = render_reprints(s, "full", [1.2, 0.9])
    with ref_engine.open(img, delta) as r:
        want = render_reprints(r, "full", [1.2, 0.9])
    for a, b in zip(got, want):
        assert lsb_stats(a, b)["max"] <= 1
    assert not np.array_equal(got[0], got[2])  # a new print seed each call


def test_glare_live_tier_and_grain(engine, ref, ref_engine):
    """The live tier (the glare blur scales with rho) with grain: film seed, then print seed."""
    w, h = 1200, 800
    img = sc.synthetic_image(w, h, 54)
    delta = dict(BASE, grain_active=True, glare_active=True, preview_long_edge=800)
    with engine.open(img, delta) as s:
        a, _ = s.render("live")
    with ref_engine.open(img, delta) as r:
        b, _ = r.render("live")
    st = lsb_stats(a, b)
    # the grain's draws near a count boundary differ from the reference's own (its sampler's host log and
    # exp differ from this build's in the last bit), as in the golden renders; measured 3.4 % of the channels
    assert st["frac_gt1"] < 0.05, st
    nograin = dict(delta, grain_active=False)
    with engine.open(img, nograin) as s:
        a, _ = s.render("live")
    with ref_engine.open(img, nograin) as r:
        b, _ = r.render("live")
    assert lsb_stats(a, b)["max"] <= 1


def test_glare_in_a_batch(engine):
    """A batch gives each frame the glare of its own session's print seed, as single renders do."""
    w, h = 320, 200
    delta = dict(BASE, grain_active=False, glare_active=True)
    imgs = [sc.synthetic_image(w, h, 60 + k) for k in range(3)]
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


def test_batch_on_the_live_tier_with_meter_and_glare(engine):
    """A batch on the live tier (frames of different sizes and geometries) with the meter and glare on
    gives each frame its single render's bits: tier images, EVs and print seeds per session."""
    frames = [(1200, 800, {}), (900, 1300, {"geometry_quarter_turns": 1}),
              (1000, 700, {"geometry_crop_w": 0.6, "geometry_rotation_deg": 4.0})]
    delta0 = dict(BASE, grain_active=True, glare_active=True, auto_exposure=True, preview_long_edge=800)
    singles = []
    for k, (w, h, extra) in enumerate(frames):
        with engine.open(sc.synthetic_image(w, h, 70 + k), dict(delta0, **extra)) as s:
            singles.append(s.render("live")[0])
    sessions = [engine.open(sc.synthetic_image(w, h, 70 + k), dict(delta0, **extra))
                for k, (w, h, extra) in enumerate(frames)]
    try:
        outs, _ = engine.render_batch(sessions, "live")
        for r, b in zip(outs, singles):
            assert r.pixels.shape == b.shape
            assert np.array_equal(r.pixels, b)
            r.free()
    finally:
        for s in sessions:
            s.close()
