"""The print-preview tables on the CPU (reference include/spektralab.h:323-346, src/res/tables.cpp,
src/session/session.cpp:503-572): the reference's tables, and its own preview render against the oracle's
trilinear restatement (the device's entry points are compared with the reference's in test_gpu_lut.py)."""

import ctypes
import json

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc

PAPER = "synthetic_paper"


def table_of(lib, eng, stock):
    t = ctypes.POINTER(ctypes.c_float)()
    size = ctypes.c_uint32()
    st = lib.lib.spk_print_lut_table(eng.h, stock.encode(), ctypes.byref(t), ctypes.byref(size))
    if st != 0:
        return st, None
    S = size.value
    return st, np.ctypeslib.as_array(t, shape=(S, S, S, 3)).copy()


def test_reference_tables(ref, ref_engine):
    st, t = table_of(ref, ref_engine, PAPER)
    assert st == 0 and t.shape == (17, 17, 17, 3)
    assert table_of(ref, ref_engine, "no_such_paper")[0] == sc.SPK_ERR_USER
    assert PAPER in json.loads(ref.lib.spk_print_lut_catalog(ref_engine.h).decode())


def test_reference_preview_against_oracle(resources, ref, ref_engine):
    """The reference's preview of a frame equals the oracle's trilinear lookup of the reference's own
    negative (the same develop, through spkref_render)."""
    w, h = 160, 120
    img = sc.synthetic_image(w, h, 71)
    delta = dict(BASE, grain_active=False)
    with ref_engine.open(img, delta) as s:
        got, meta, reply = s.preview_lut(None, "full")
    assert meta == {"reprint": 1, "negative_was_cached": 1}
    assert reply["print_stock"] == PAPER and reply["paired_film"] == BASE["film_stock"] and "warning" not in reply
    out = np.zeros((1, h, w, 4), np.uint16)
    neg = np.zeros((h, w, 3), np.float32)
    z = (ctypes.c_double * 3)(0, 0, 0)
    ref.check(ref.lib.spkref_render(ref_engine.h, img.ctypes.data_as(sc.FP), w, h, json.dumps(delta).encode(), 0, z,
                                    z, z, (ctypes.c_double * 1)(1.0), 1,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), neg.ctypes.data_as(sc.FP)))
    _, table = table_of(ref, ref_engine, PAPER)
    lo = [0.0, 0.0, 0.0]
    hi = [3.2, 3.2 * 1.05, 3.2 * 0.95]
    want = oracle.print_lut(neg, table, 17, np.float32(lo), np.float32(hi))
    assert lsb_stats(got, want)["max"] <= 1
