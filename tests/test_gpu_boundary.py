"""The ABI's control surface under load (marked gpu: needs a B200): cancellation from a second thread,
the progress record, the memory report, and the failure paths of the tensor-core kernel's and the
recursive blur's bounded mbarrier waits.

Reference behaviour:
  * cancel: tests/session_check.py:287-306 -- a render polled with spk_cancel returns SPK_ERR_CANCELLED,
    its result zeroed, the progress record cancelled and not done, and the next reprint re-develops
    (src/session/session.cpp:405-450, src/core/render.hpp:78-81);
  * progress: src/session/progress.cpp:46-72 (the snapshot's nine keys, pct, unknown ids);
  * memory report: src/session/engine.cpp:246-319 and the invariants tests/session_check.py:157-168 and
    tests/abi_smoke.py:114-120 check.
"""

import ctypes
import json
import subprocess
import sys
import threading

import numpy as np
import pytest

from conftest import BASE, PKG, sc

pytestmark = pytest.mark.gpu

SNAPSHOT_KEYS = ["auto_exposure_ev", "cancelled", "done", "effect_versions", "memory_pressure_critical",
                 "node_times", "pct", "progress_id", "stage"]
LABELS = {"preprocess.decode", "preprocess.geometry", "filming.auto_exposure", "filming.upsample",
          "filming.exposure_compensation", "filming.boost", "filming.headroom", "filming.lens_blur",
          "filming.halation", "filming.log", "filming.curves", "filming.couplers", "filming.grain",
          "printing.enlarger", "printing.gain", "printing.paper", "scanning.scan", "scanning.levels",
          "scanning.glare", "scanning.to_rgb", "scanning.gamut", "scanning.scanner", "scanning.edr",
          "scanning.encode", "queued"}


def progress(lib, s, pid=None):
    out = ctypes.c_char_p()
    st = lib.lib.spk_progress(s.h, pid.encode() if pid else None, ctypes.byref(out))
    return st, (lib.take_json(out) if st == sc.SPK_OK else None)


def render_in_thread(lib, s, box, tier=b"full"):
    r = sc.SpkResult()
    box["st"] = lib.lib.spk_render(s.h, tier, ctypes.byref(r))
    box["texture"] = r.texture
    box["rgba16"] = bool(r.rgba16)
    box["width"] = r.width
    if r.texture:
        lib.lib.spk_result_free(ctypes.byref(r))


def test_cancel_from_a_second_thread(engine, lib):
    img = sc.synthetic_image(2048, 1536, 2)
    cancelled = 0
    for attempt in range(6):
        with engine.open(img, BASE) as s:
            box = {}
            th = threading.Thread(target=render_in_thread, args=(lib, s, box))
            th.start()
            while th.is_alive():
                lib.lib.spk_cancel(s.h, None)
            th.join()
            st, pr = progress(lib, s)
            assert st == sc.SPK_OK and sorted(pr) == SNAPSHOT_KEYS
            if box["st"] == sc.SPK_ERR_CANCELLED:
                cancelled += 1
                assert not box["texture"] and not box["rgba16"] and box["width"] == 0  # the result is zeroed
                assert pr["cancelled"] and not pr["done"] and pr["pct"] < 100.0
                _, meta = s.reprint("full")
                assert meta["reprint"] == 0 and meta["negative_was_cached"] == 0  # the negative was dropped
                _, meta = s.reprint("full")
                assert meta["reprint"] == 1
            else:
                assert box["st"] == sc.SPK_OK and pr["done"]
    assert cancelled >= 1, "no cancel landed in six renders"


def test_cancel_of_another_progress_id_is_ignored(engine, lib):
    img = sc.synthetic_image(1024, 768, 2)
    with engine.open(img, BASE) as s:
        box = {}
        th = threading.Thread(target=render_in_thread, args=(lib, s, box))
        th.start()
        while th.is_alive():
            lib.lib.spk_cancel(s.h, b"p0")  # not the current render's id
        th.join()
        assert box["st"] == sc.SPK_OK
        st, pr = progress(lib, s)
        assert not pr["cancelled"] and pr["done"]


def test_progress_record(engine, lib):
    img = sc.synthetic_image(640, 480, 2)
    with engine.open(img, BASE) as s:
        st, pr = progress(lib, s)
        assert st == sc.SPK_OK and pr["stage"] == "queued" and not pr["done"] and pr["pct"] == 0.0
        seen = []
        box = {}
        th = threading.Thread(target=render_in_thread, args=(lib, s, box))
        th.start()
        while th.is_alive():
            st, p = progress(lib, s)
            if st == sc.SPK_OK:
                seen.append((p["pct"], p["stage"], p["progress_id"]))
        th.join()
        assert box["st"] == sc.SPK_OK
        st, pr = progress(lib, s)
        assert sorted(pr) == SNAPSHOT_KEYS
        assert pr["done"] and pr["pct"] == 100.0 and pr["stage"] == "scanning.encode" and not pr["cancelled"]
        assert pr["auto_exposure_ev"] is None and pr["node_times"] == {} and not pr["memory_pressure_critical"]
        assert pr["effect_versions"] == ("halation=reference;grain=reference;glare=reference;"
                                         "print_spatial=reference;dir_couplers=reference")
        assert {stage for _, stage, _ in seen} <= LABELS
        for pid in {p for _, _, p in seen}:
            pcts = [pct for pct, _, q in seen if q == pid]
            assert pcts == sorted(pcts)  # pct never goes back within one render
        _, meta = s.reprint("full")
        st, pr2 = progress(lib, s, meta["progress_id"])
        assert st == sc.SPK_OK and pr2["progress_id"] == meta["progress_id"] != pr["progress_id"]
        assert progress(lib, s, pr["progress_id"])[0] == sc.SPK_ERR_USER  # an id that is not current
        assert "unknown progress id" in lib.last_error()
    with engine.open(img, dict(BASE, auto_exposure=True)) as s:
        s.render("full")
        _, pr = progress(lib, s)
        assert isinstance(pr["auto_exposure_ev"], float) and np.isfinite(pr["auto_exposure_ev"])


MEMORY_SCRIPT = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import spk_ctypes as sc, synth_resources
lib = sc.load()
res = synth_resources.ensure(sc.RESOURCES)
eng = lib.engine(res, device=0)
def mem():
    return json.loads(lib.lib.spk_memory_report(eng.h).decode())
m0 = mem()
base = {"film_stock": "synthetic_negative_400", "print_stock": "synthetic_paper", "auto_exposure": False,
        "dir_couplers_active": False, "glare_active": False, "preview_long_edge": 800}
img = sc.synthetic_image(1200, 900, 1)
s = eng.open(img, base)
s.render("live")
s.render("full")
m1 = mem()
s.close()
lib.lib.spk_engine_trim(eng.h)
m2 = mem()
print(json.dumps([m0, m1, m2]))
"""


def test_memory_report(lib):
    """In a fresh process (the device pool is process-wide): the reference's keys and invariants while two
    negatives are cached, and after the session is released and the engine trimmed."""
    r = subprocess.run([sys.executable, "-c", MEMORY_SCRIPT, PKG], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    m0, m1, m2 = json.loads(r.stdout.strip().splitlines()[-1])
    for m in (m0, m1, m2):
        assert sorted(m) == ["persistent", "pool", "pressure", "total_bytes"]
        assert m["total_bytes"] == m["pool"]["total_bytes"] + m["persistent"]["bytes"]
        assert all(m["pool"]["audit"][k] == 0 for k in ("live_underflows", "over_releases", "reclaim_while_encoding"))
        assert sorted(m["pressure"]) == ["critical_events", "critical_pending", "idle_trim_seconds", "idle_trims",
                                         "monitor", "warn_events"]
        assert sorted(m["pool"]) == ["audit", "buffers", "frame_high_water_bytes", "free_buffers", "free_bytes",
                                     "live_buffers", "live_bytes", "pending_buffers", "pending_bytes", "total_bytes"]
    pr = m1["persistent"]
    assert pr["source_bytes"] == 1200 * 900 * 12
    assert pr["source_bytes"] + pr["cached_negative_bytes"] <= pr["bytes"]
    assert len(pr["sessions"]) == 1 and pr["sessions"][0]["negatives"] == 2 and pr["negatives"] == 2
    assert pr["cached_negative_bytes"] == 1200 * 900 * 12 + 800 * 600 * 12  # the full and live negatives
    assert m1["pool"]["frame_high_water_bytes"] > 0
    assert m2["pool"]["total_bytes"] == 0 and m2["persistent"]["source_bytes"] == 0
    assert m2["persistent"]["sessions"] == [] and m2["persistent"]["negatives"] == 0


def test_tensor_core_wait_runs_out(engine, lib):
    """The spectral-mode kernel's stage waits cut to one SM clock: a wait runs out, the kernel drains the MMAs
    it issued, frees its tensor memory and flags the failure; the reprint returns SPK_ERR_GPU without a hang,
    and with the limit restored the same session renders the same image as before."""
    img = sc.synthetic_image(512, 384, 6)
    with engine.open(img, dict(BASE, grain_active=False)) as s:
        s.set_print_mode("bf16x3", 81)
        want, _ = s.render("full")
        lib.check(lib.lib.spkx_test_set_tc_wait_limit(1))
        try:
            with pytest.raises(sc.SpkError) as e:
                s.reprint("full")
            assert e.value.status == sc.SPK_ERR_GPU and "tensor-core wait" in str(e.value)
        finally:
            lib.check(lib.lib.spkx_test_set_tc_wait_limit(0))
        got, meta = s.reprint("full")
        assert meta["reprint"] == 1 and np.array_equal(got, want)
    assert lib.lib.spkx_test_set_tc_wait_limit(-1) == sc.SPK_ERR_INVALID_ARG


HALATION = ([((1, 1, 1), (8, 8, 8)), ((1, 1, 1), (40, 40, 40))], (0.03, 0.03, 0.03))


def test_iir_column_wait_runs_out(engine, lib):
    """The recursive blur's column pass loads its strips by TMA and waits on an mbarrier. With the wait cut
    to one SM clock the strip waits give up at once: each CTA counts the event, waits again under the full
    limit for the copies in flight and goes on, so the render (width a multiple of 4: the TMA path) is the
    image a fresh session renders under the normal limit, and no wait gives up under that limit."""
    img = sc.synthetic_image(512, 384, 6)
    n = ctypes.c_uint32(0)
    lib.check(lib.lib.spkx_test_take_iir_waits_given_up(ctypes.byref(n)))
    with engine.open(img, BASE) as s:
        s.set_halation(*HALATION)
        want, _ = s.render("full")
    lib.check(lib.lib.spkx_test_take_iir_waits_given_up(ctypes.byref(n)))
    assert n.value == 0
    lib.check(lib.lib.spkx_test_set_iir_wait_limit(1))
    try:
        with engine.open(img, BASE) as s:
            s.set_halation(*HALATION)
            got, _ = s.render("full")
        lib.check(lib.lib.spkx_test_take_iir_waits_given_up(ctypes.byref(n)))
    finally:
        lib.check(lib.lib.spkx_test_set_iir_wait_limit(0))
    assert n.value > 0
    assert np.array_equal(got, want)
    assert lib.lib.spkx_test_set_iir_wait_limit(-1) == sc.SPK_ERR_INVALID_ARG
    assert lib.lib.spkx_test_take_iir_waits_given_up(None) == sc.SPK_ERR_INVALID_ARG
