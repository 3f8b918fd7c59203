"""The print-preview tables on the device (marked gpu), through the C ABI: the catalog and the tables
against the reference's, and spk_preview_stock_lut against the reference engine's and the oracle's
trilinear lookup of the device's own negative."""

import json

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc
from test_lut_cpu import PAPER, table_of

pytestmark = pytest.mark.gpu


def test_catalog_and_tables_match_reference(lib, engine, ref, ref_engine):
    mine = json.loads(lib.lib.spk_print_lut_catalog(engine.h).decode())
    theirs = json.loads(ref.lib.spk_print_lut_catalog(ref_engine.h).decode())
    assert mine == theirs and PAPER in mine
    st, a = table_of(lib, engine, PAPER)
    st2, b = table_of(ref, ref_engine, PAPER)
    assert st == st2 == 0 and np.array_equal(a, b)
    assert table_of(lib, engine, "no_such_paper")[0] == sc.SPK_ERR_USER


@pytest.mark.parametrize("tier,w,h", [("full", 200, 136), ("live", 1000, 700)])
def test_preview_within_one_lsb_of_reference(lib, engine, ref, ref_engine, tier, w, h):
    img = sc.synthetic_image(w, h, 72)
    delta = dict(BASE, grain_active=False, preview_long_edge=800)
    with engine.open(img, delta) as s:
        got, meta, reply = s.preview_lut(None, tier)
        assert meta == {"reprint": 1, "negative_was_cached": 1}
        neg = s.negative(tier, got.shape[1], got.shape[0])  # the preview cached the negative it developed
        _, m2 = s.reprint(tier)
        assert m2["reprint"] == 1
    with ref_engine.open(img, delta) as r:
        want, _, reply2 = r.preview_lut(None, tier)
    assert lsb_stats(got, want)["max"] <= 1
    skip = ("apply_ms", "apply_backend")
    assert {k: v for k, v in reply.items() if k not in skip} == {k: v for k, v in reply2.items() if k not in skip}
    _, table = table_of(lib, engine, PAPER)
    lut = oracle.print_lut(neg, table, 17, np.float32([0, 0, 0]), np.float32([3.2, 3.2 * 1.05, 3.2 * 0.95]))
    assert lsb_stats(got, lut)["max"] <= 1


def test_preview_refuses_a_missing_table(engine):
    with engine.open(sc.synthetic_image(32, 24, 73), BASE) as s:
        with pytest.raises(sc.SpkError) as e:
            s.preview_lut("no_such_paper", "full")
        assert e.value.status == sc.SPK_ERR_USER
