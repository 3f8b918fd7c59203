"""The C ABI boundary without a GPU: exported symbols, struct layouts, NULL-argument statuses,
parameter validation (reference src/abi/abi.cpp:40-65, src/params/delta.cpp:41-96,
tests/abi_smoke.py)."""

import ctypes
import json
import os
import re

import pytest

from conftest import BASE, REPO, sc

HEADERS = [os.path.join(REPO, "include", "spektralab.h"), os.path.join(REPO, "include", "spektralab_b200.h")]


def declared():
    names = []
    for h in HEADERS:
        text = open(h).read()
        names += re.findall(r"SPK_API[^;(]*?\b(sp[kx]\w*)\s*\(", text)
    return names


def test_headers_declare_the_reference_entry_points():
    names = set(declared())
    for n in sc.ABI:
        assert n in names, n
    # the reference's 26, plus the render's adjoint (spk_render_vjp) in the extension header
    assert {n for n in names if n.startswith("spk_")} == set(sc.ABI) | {"spk_render_vjp"}


def test_library_exports_every_declared_symbol(lib):
    for name in declared():
        assert hasattr(lib.lib, name), name


def test_struct_layouts():
    assert ctypes.sizeof(sc.SpkImage) == 24 and ctypes.alignment(sc.SpkImage) == 8
    assert ctypes.sizeof(sc.SpkDeviceImage) == 24
    assert ctypes.sizeof(sc.SpkResult) == 88
    assert sc.SpkResult.elapsed_ms.offset == 32 and sc.SpkResult.progress_id.offset == 48
    assert sc.SpkResult.row_stride_px.offset == 24 and sc.SpkResult.reprint.offset == 40


def test_null_arguments(lib):
    L = lib.lib
    r = sc.SpkResult()
    assert L.spk_render(None, b"full", ctypes.byref(r)) == sc.SPK_ERR_INVALID_ARG
    assert "session is NULL" in lib.last_error()
    assert L.spk_reprint(None, b"full", ctypes.byref(r)) == sc.SPK_ERR_INVALID_ARG
    assert L.spk_set_params(None, b"{}", None) == sc.SPK_ERR_INVALID_ARG
    assert L.spk_get_params(None, None) == sc.SPK_ERR_INVALID_ARG
    assert L.spk_progress(None, None, None) == sc.SPK_ERR_INVALID_ARG
    assert L.spk_open(None, None, None, None) is None
    assert L.spk_engine_create(None, None) is None
    L.spk_result_free(None)
    L.spk_result_free(ctypes.byref(r))
    L.spk_string_free(None)
    L.spk_engine_destroy(None)
    L.spk_session_release(None)
    L.spk_cancel(None, None)
    assert L.spk_capabilities(None) == b""
    assert L.spk_params_schema(None) == b""
    assert L.spk_memory_report(None) == b""
    assert L.spk_engine_trim(None) == 0
    assert L.spk_last_error(None) is not None


def test_build_info(lib):
    info = lib.lib.spk_build_info().decode()
    assert info.startswith("spektralab-native 1.0.0") and "math=safe" in info


def test_missing_resources_is_io_error(lib):
    e = lib.lib.spk_engine_create(b"/nonexistent/resources", None)
    assert e is None
    msg = lib.last_error()
    assert "does not exist" in msg or "no CUDA device" in msg


def _setup(lib, resources, delta):
    out = ctypes.c_char_p()
    st = lib.lib.spkx_setup_json(resources.encode(), delta.encode() if isinstance(delta, str) else json.dumps(delta).encode(),
                                 9.0, ctypes.byref(out))
    if st == 0:
        lib.take_json(out)
    return st, lib.last_error()


@pytest.mark.parametrize("delta,needle", [
    ('{"no_such_field": 1}', "unknown parameter"),
    ('{"print_exposure": 100}', "outside"),
    ('{"print_exposure": "1"}', "expects float"),
    ('{"grain_active": 1}', "expects bool"),
    ('{"auto_exposure_method": "bogus"}', "is not one of"),
    ('[1, 2]', "must be an object"),
    ('{"print_exposure": 1.0', "JSON"),
    ('{"film_stock": "../x"}', "invalid stock id"),
    ('{"film_stock": "missing_stock"}', "cannot read"),
])
def test_delta_validation(lib, resources, delta, needle):
    st, msg = _setup(lib, resources, delta)
    assert st == sc.SPK_ERR_USER, (st, msg)
    assert needle in msg, msg


def test_valid_delta_builds(lib, resources):
    st, msg = _setup(lib, resources, BASE)
    assert st == sc.SPK_OK, msg


def test_wait_limit_hooks_check_their_arguments(lib):
    """The failure-path test hooks refuse bad arguments before any CUDA call (so here, with no GPU)."""
    L = lib.lib
    assert L.spkx_test_set_tc_wait_limit(-1) == sc.SPK_ERR_INVALID_ARG
    assert L.spkx_test_set_iir_wait_limit(-1) == sc.SPK_ERR_INVALID_ARG
    assert "SM clocks" in lib.last_error()
    assert L.spkx_test_take_iir_waits_given_up(None) == sc.SPK_ERR_INVALID_ARG
    assert "count is NULL" in lib.last_error()
    assert L.spkx_test_set_iir_wait_limit(0) == sc.SPK_OK
