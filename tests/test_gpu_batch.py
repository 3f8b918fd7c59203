"""Batched renders through spkx_render_batch (marked gpu): every plan gives, pixel for pixel, what
spk_render / spk_reprint give the same sessions one at a time (frames of mixed sizes, per-frame print
exposure and halation, frames that stay on the scanner's separate passes), the timed choice of plan, and the
refusals."""

import ctypes

import numpy as np
import pytest

from conftest import BASE, sc

pytestmark = pytest.mark.gpu

# (width, height, extra parameters): 5 x 6 is narrower than the scanner's halo and 320 x 200 with a lens
# blur of 4 px takes the recursive branch; both stay on the separate passes inside a batch
FRAMES = [
    (256, 256, {}),
    (640, 360, {"print_exposure": 1.3}),
    (97, 131, {"print_exposure": 0.8}),
    (1024, 768, {}),
    (300, 1000, {"print_exposure": 1.1}),
    (33, 35, {}),
    (5, 6, {}),
    (320, 200, {"scanner_lens_blur": 4.0}),
]
HALATION = {0: ([(0.2, 0.1, 0.05), (3.0, 3.0, 3.0)], (0.3, 0.2, 0.1)),
            3: ([(0.1, 0.1, 0.1), (8.0, 8.0, 8.0)], (0.25, 0.25, 0.25))}
PLANS = ["frames:1", "frames:4", "frames:16", "persistent:2048:592", "persistent:8192:1184", "persistent:2:148",
         "persistent:8192:1184:4", "persistent:2048:592:3", "persistent:8192:1184:64"]


def open_all(engine):
    out = []
    for i, (w, h, extra) in enumerate(FRAMES):
        s = engine.open(sc.synthetic_image(w, h, 10 + i), dict(BASE, **extra))
        if i in HALATION:
            comps, strength = HALATION[i]
            s.set_halation([(comps[0], comps[1])], strength)
        out.append(s)
    return out


def take(results):
    arrs = [r.pixels.copy() for r in results]
    metas = [(r.r.reprint, r.r.negative_was_cached) for r in results]
    for r in results:
        r.free()
    return arrs, metas


def singles(engine, n_renders):
    """Per session: n_renders spk_render calls, then print_exposure +0.2 and one spk_reprint."""
    ss = open_all(engine)
    try:
        renders = [[s.render("full")[0] for s in ss] for _ in range(n_renders)]
        for s, (_, _, extra) in zip(ss, FRAMES):
            s.set_params({"print_exposure": extra.get("print_exposure", 1.0) + 0.2})
        reprints = [s.reprint("full")[0] for s in ss]
    finally:
        for s in ss:
            s.close()
    return renders, reprints


@pytest.fixture(scope="module")
def expected(engine):
    return singles(engine, 2)


@pytest.mark.parametrize("plan", PLANS)
def test_pinned_plan_matches_singles(engine, expected, plan):
    renders, reprints = expected
    engine.batch_plan(plan)
    ss = open_all(engine)
    try:
        for k in range(2):
            res, info = engine.render_batch(ss, "full")
            assert info["plan"] == plan and info["tuning_ms"] == 0
            arrs, metas = take(res)
            for i, a in enumerate(arrs):
                assert a.shape == renders[k][i].shape
                assert np.array_equal(a, renders[k][i]), (plan, k, FRAMES[i][:2])
                assert metas[i] == (0, 0)
        for s, (_, _, extra) in zip(ss, FRAMES):
            s.set_params({"print_exposure": extra.get("print_exposure", 1.0) + 0.2})
        res, info = engine.render_batch(ss, "full", reprint=True)
        arrs, metas = take(res)
        for i, a in enumerate(arrs):
            assert np.array_equal(a, reprints[i]), (plan, "reprint", FRAMES[i][:2])
            assert metas[i] == (1, 1)
    finally:
        engine.batch_plan(None)
        for s in ss:
            s.close()


def test_timed_choice_then_reuse(engine, expected):
    renders, _ = expected
    engine.batch_plan(None)
    ss = open_all(engine)
    try:
        res, info1 = engine.render_batch(ss, "full")
        a1, _ = take(res)
        res, info2 = engine.render_batch(ss, "full")
        a2, _ = take(res)
    finally:
        for s in ss:
            s.close()
    assert info1["tuning_ms"] > 0 and info2["tuning_ms"] == 0
    assert info1["plan"] == info2["plan"]
    assert len(info2["frame_done_ms"]) == len(FRAMES) and all(t > 0 for t in info2["frame_done_ms"])
    for i in range(len(FRAMES)):
        assert np.array_equal(a1[i], renders[0][i]) and np.array_equal(a2[i], renders[1][i])


def test_batch_refusals(engine, lib):
    s1 = engine.open(sc.synthetic_image(16, 16, 1), BASE)
    s2 = engine.open(sc.synthetic_image(16, 16, 2), BASE)
    try:
        with pytest.raises(sc.SpkError) as e:
            engine.render_batch([s1, s1], "full")
        assert e.value.status == sc.SPK_ERR_INVALID_ARG and "twice" in str(e.value)
        with pytest.raises(sc.SpkError) as e:
            engine.render_batch([s1, s2], "huge")
        assert e.value.status == sc.SPK_ERR_INVALID_ARG and "unknown tier" in str(e.value)
        with pytest.raises(sc.SpkError) as e:
            engine.render_batch([], "full")
        assert e.value.status == sc.SPK_ERR_INVALID_ARG
        for bad in ("frames:0", "frames:17", "persistent:3:10", "persistent:2048", "persistent:2048:0", "fast",
                    "persistent:2048:592:0", "persistent:2048:592:1025", "persistent:2048:592:", "persistent:2048:592:x"):
            with pytest.raises(sc.SpkError) as e:
                engine.batch_plan(bad)
            assert e.value.status == sc.SPK_ERR_INVALID_ARG
        # a failed batch leaves every result zeroed
        rs = (sc.SpkResult * 2)()
        rs[0].width = 77
        hs = (sc.P * 2)(s1.h, s1.h)
        st = lib.lib.spkx_render_batch(hs, 2, b"full", 0, rs, None)
        assert st == sc.SPK_ERR_INVALID_ARG and rs[0].width == 0 and not rs[0].texture
        res, info = engine.render_batch([s1, s2], "full")
        take(res)
    finally:
        s1.close()
        s2.close()


@pytest.mark.parametrize("plan", ["persistent:2048:592", "persistent:8192:2368", "persistent:2048:592:2"])
def test_persistent_plan_with_per_frame_filters(engine, plan):
    """Frames whose enlarger filters differ do not share spectral tables: the persistent print then stages
    every frame's tables itself (the frames above share theirs, which the kernel takes once). Each frame
    still equals its single render."""
    specs = [(300, 200, {"m_filter_shift": 0.2}), (256, 128, {"y_filter_shift": -0.3}), (512, 288, {})]
    imgs = [sc.synthetic_image(w, h, 40 + i) for i, (w, h, _) in enumerate(specs)]
    singles_out = []
    for img, (w, h, extra) in zip(imgs, specs):
        with engine.open(img, dict(BASE, **extra)) as s:
            singles_out.append(s.render("full")[0])
    engine.batch_plan(plan)
    ss = [engine.open(img, dict(BASE, **extra)) for img, (w, h, extra) in zip(imgs, specs)]
    try:
        res, info = engine.render_batch(ss, "full")
        arrs, _ = take(res)
        assert info["plan"] == plan
        for a, want in zip(arrs, singles_out):
            assert np.array_equal(a, want), plan
    finally:
        engine.batch_plan(None)
        for s in ss:
            s.close()
