"""The rest of the reference's C ABI through this build (marked gpu: the engine needs a device), each
against the reference engine's own entry point on the same resources: spk_output_transform (matrix,
gamut constants, the C_max table), spk_solve and spk_warm_up (include/spektralab.h:217-360)."""

import ctypes
import json

import numpy as np
import pytest

from conftest import BASE, sc

pytestmark = pytest.mark.gpu


def output_transform(L, eng, src, dst, gamut):
    out = ctypes.c_char_p()
    cmax = ctypes.POINTER(ctypes.c_float)()
    n = ctypes.c_uint32()
    st = L.lib.spk_output_transform(eng.h, src.encode(), dst.encode(), gamut.encode() if gamut else None,
                                    ctypes.byref(out), ctypes.byref(cmax), ctypes.byref(n))
    if st != 0:
        return st, None, None
    return st, L.take_json(out), np.ctypeslib.as_array(cmax, shape=(n.value,)).copy()


def close(a, b, path=""):
    if isinstance(a, dict):
        assert set(a) == set(b), path
        for k in a:
            close(a[k], b[k], path + "/" + k)
    elif isinstance(a, list):
        assert len(a) == len(b), path
        for i, (x, y) in enumerate(zip(a, b)):
            close(x, y, f"{path}[{i}]")
    elif isinstance(a, float):
        assert a == pytest.approx(b, rel=1e-12, abs=1e-14), path
    else:
        assert a == b, path


@pytest.mark.parametrize("src,dst", [("ProPhoto RGB", "sRGB"), ("sRGB", "ProPhoto RGB"), ("sRGB", "sRGB"),
                                     ("Adobe RGB (1998)", "ITU-R BT.709")])
@pytest.mark.parametrize("gamut", [None, '{"algorithm": "off"}',
                                   '{"knee": [0, 1, 5], "lightness_compression_active": false}',
                                   '{"lightness_compression": [0.5, 1.0, 2.0], "knee": [1, 2]}'])
def test_output_transform_matches_reference(lib, engine, ref, ref_engine, src, dst, gamut):
    st, mine, cm = output_transform(lib, engine, src, dst, gamut)
    st2, theirs, cm2 = output_transform(ref, ref_engine, src, dst, gamut)
    assert st == st2 == 0
    close(mine, theirs)
    assert cm.shape == cm2.shape == (64 * 720,)
    np.testing.assert_allclose(cm, cm2, rtol=2e-7, atol=0)


@pytest.mark.parametrize("args,status", [(("Nope", "sRGB", None), sc.SPK_ERR_USER),
                                         (("sRGB", "sRGB", '{"algorithm": "aces"}'), sc.SPK_ERR_USER),
                                         (("sRGB", "sRGB", "[1, 2]"), sc.SPK_ERR_INVALID_ARG)])
def test_output_transform_refusals(lib, engine, ref, ref_engine, args, status):
    assert output_transform(lib, engine, *args)[0] == output_transform(ref, ref_engine, *args)[0] == status


def solve(L, sess, target):
    out = ctypes.c_char_p()
    st = L.lib.spk_solve(sess.h, target.encode() if target is not None else None, ctypes.byref(out))
    return st, (L.take_json(out) if st == 0 else None)


@pytest.mark.parametrize("target", [None, "both", "exposure", "filter_pack"])
@pytest.mark.parametrize("ae", [False, True])
def test_solve_matches_reference(engine, ref, ref_engine, target, ae):
    img = sc.synthetic_image(900, 600, 81)
    delta = dict(BASE, auto_exposure=ae, auto_exposure_method="balanced")
    with engine.open(img, delta) as s, ref_engine.open(img, delta) as r:
        st, mine = solve(engine.L, s, target)
        st2, theirs = solve(ref_engine.L, r, target)
        assert st == st2 == 0
        close(mine, theirs)
        assert solve(engine.L, s, "nonsense")[0] == solve(ref_engine.L, r, "nonsense")[0] == sc.SPK_ERR_USER


def warm_up(L, eng, film, paper):
    out = ctypes.c_char_p()
    st = L.lib.spk_warm_up(eng.h, film.encode() if film else None, paper.encode() if paper else None,
                           ctypes.byref(out))
    return st, L.take_json(out)


def test_warm_up_matches_reference(engine, ref, ref_engine):
    st, mine = warm_up(engine.L, engine, BASE["film_stock"], BASE["print_stock"])
    st2, theirs = warm_up(ref_engine.L, ref_engine, BASE["film_stock"], BASE["print_stock"])
    assert st == st2 == 0
    names = lambda r: [(x["name"], x["ok"]) for x in r["steps"]]
    assert names(mine) == names(theirs) == [("profiles", True), ("pipeline", True), ("kernels", True)]
    # the default stocks are not in these resources: the first step fails and ends the sequence
    st, mine = warm_up(engine.L, engine, None, None)
    st2, theirs = warm_up(ref_engine.L, ref_engine, None, None)
    assert st == st2 == 0 and names(mine) == names(theirs) == [("profiles", False)]
    assert mine["film_stock"] == theirs["film_stock"] == "kodak_portra_400"
