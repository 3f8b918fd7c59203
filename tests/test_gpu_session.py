"""Session behaviour through the C ABI on the device (marked gpu): render / reprint flags and the cached
negative, live print parameters, determinism and the seed sequence, refusals, the 4K workload's
size-independent properties (reference src/session/session.cpp:216-259, :327-450;
include/spektralab.h:287-308)."""

import ctypes
import json

import numpy as np
import pytest

from conftest import BASE, lsb_stats, sc

pytestmark = pytest.mark.gpu


def test_reprint_reuses_negative_and_live_exposure(engine):
    img = sc.synthetic_image(160, 120, 1)
    with engine.open(img, BASE) as s:
        a1, m1 = s.reprint("full")  # no cached negative: develops, reprint flag 0
        assert m1["reprint"] == 0 and m1["negative_was_cached"] == 0
        n1 = s.negative("full", 160, 120)
        a2, m2 = s.reprint("full")
        assert m2["reprint"] == 1
        assert np.array_equal(a1, a2)  # same negative, same print parameters
        reply = s.set_params({"print_exposure": 1.4})
        assert reply["invalidated"] == "print"
        a3, m3 = s.reprint("full")
        assert m3["reprint"] == 1 and not np.array_equal(a2, a3)
        assert np.array_equal(n1, s.negative("full", 160, 120))
        # brighter print exposure gives a denser print (darker)
        assert a3[..., :3].astype(np.float64).mean() < a2[..., :3].astype(np.float64).mean()
        reply = s.set_params({"grain_amount": 0.5})
        assert reply["invalidated"] == "shoot"
        with pytest.raises(sc.SpkError):
            s.negative("full", 160, 120)


def test_seed_sequence_and_determinism(engine):
    img = sc.synthetic_image(96, 64, 2)
    with engine.open(img, BASE) as s1, engine.open(img, BASE) as s2:
        a, _ = s1.render("full")
        b, _ = s2.render("full")
        assert np.array_equal(a, b)  # two fresh pipelines draw the same film seed
        c, _ = s1.render("full")
        assert not np.array_equal(a, c)  # the next render draws the next seed
    nograin = dict(BASE, grain_active=False)
    with engine.open(img, nograin) as s:
        a, _ = s.render("full")
        b, _ = s.render("full")
        r, _ = s.reprint("full")
        assert np.array_equal(a, b) and np.array_equal(a, r)


def test_unknown_tier_and_result_zeroed(engine, lib):
    img = sc.synthetic_image(8, 8, 0)
    with engine.open(img, BASE) as s:
        r = sc.SpkResult()
        st = lib.lib.spk_render(s.h, b"huge", ctypes.byref(r))
        # the tier is checked before the result is touched (reference src/abi/abi.cpp:293-300)
        assert st == sc.SPK_ERR_INVALID_ARG and "unknown tier" in lib.last_error()
    wide = sc.synthetic_image(3500, 4, 0)
    with engine.open(wide, BASE) as s:
        # the preview tier of a frame wider than 3400 px: its downscaled image, floor(4 * 3400 / 3500) rows
        a, meta = s.render("preview")
        assert a.shape == (3, 3400, 4) and meta["row_stride_px"] % 32 == 0


def test_every_parameter_renders(engine):
    """No parameter of the schema is refused at open: every stage of the reference's render path is here."""
    img = sc.synthetic_image(32, 24, 0)
    for extra in ({"auto_exposure": True}, {"glare_active": True}, {"halation_boost_ev": 1.0},
                  {"scanner_white_correction": True}, {"extended_dynamic_range": True},
                  {"antihalation_removed": True}, {"geometry_flip_h": True}, {"input_cctf_decoding": True}):
        with engine.open(img, dict(BASE, **extra)) as s:
            a, _ = s.render("full")
            assert (a[..., 3] == 65535).all()


def test_couplers_have_no_adjoint(engine):
    """The DIR couplers render; the adjoint (spk_render_vjp) refuses them as outside its parameters."""
    img = sc.synthetic_image(16, 12, 0)
    with engine.open(img, dict(BASE, grain_active=False, dir_couplers_active=True)) as s:
        a, _ = s.render("full")
        assert (a[..., 3] == 65535).all()
        with pytest.raises(sc.SpkError) as e:
            s.render_vjp(np.ones((12, 16, 3), np.float32), 1)
        assert e.value.status == sc.SPK_ERR_UNSUPPORTED and "DIR couplers" in str(e.value)


def test_geometry_and_decode_have_no_adjoint(engine):
    img = sc.synthetic_image(16, 12, 0)
    for extra in ({"geometry_flip_h": True}, {"input_cctf_decoding": True}, {"auto_exposure": True},
                  {"glare_active": True}, {"halation_boost_ev": 1.0}, {"extended_dynamic_range": True}):
        with engine.open(img, dict(BASE, grain_active=False, **extra)) as s:
            with pytest.raises(sc.SpkError) as e:
                s.render_vjp(np.ones((12, 16, 3), np.float32), 1)
            assert e.value.status == sc.SPK_ERR_UNSUPPORTED


def test_channels_and_nonfinite_inputs(engine):
    img3 = sc.synthetic_image(33, 21, 4)
    img4 = np.concatenate([img3, np.full((21, 33, 1), 123.0, np.float32)], axis=2)
    bad = img3.copy()
    bad[0, 0, 0] = np.nan
    bad[1, 1, 1] = np.inf
    delta = dict(BASE, grain_active=False)
    with engine.open(img3, delta) as s:
        a, _ = s.render("full")
    with engine.open(img4, delta) as s:
        b, _ = s.render("full")
    assert np.array_equal(a, b)
    with engine.open(bad, delta) as s:
        c, _ = s.render("full")
    fixed = img3.copy()
    fixed[0, 0, 0] = 0.0
    fixed[1, 1, 1] = 0.0
    with engine.open(fixed, delta) as s:
        d, _ = s.render("full")
    assert np.array_equal(c, d)


def test_4k_properties(engine):
    w, h = 3840, 2160
    img = sc.synthetic_image(w, h, 0)
    with engine.open(img, BASE) as s:
        s.set_halation([((1, 1, 1), (20, 20, 20)), ((1, 1, 1), (120, 120, 120))], (0.03, 0.03, 0.03))
        a, meta = s.render("full")
        assert meta["row_stride_px"] % 32 == 0 and meta["row_stride_px"] >= w
        assert (a[..., 3] == 65535).all()
        neg = s.negative("full", w, h)
        assert np.isfinite(neg).all()
        s.set_params({"print_exposure": 1.2})
        b, m2 = s.reprint("full")
        assert m2["reprint"] == 1
        assert np.array_equal(neg, s.negative("full", w, h))
        # a reprint at the first exposure gives the render's image back bit for bit
        s.set_params({"print_exposure": 1.0})
        c, _ = s.reprint("full")
        assert np.array_equal(a, c)
        prof = s.profile("full", True, 2)
        assert set(prof["stages"]) >= {"print", "scanner"}
