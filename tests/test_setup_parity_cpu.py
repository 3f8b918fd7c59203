"""The binary64 set-up, narrowed to the kernels' binary32 constants, is bit-identical to the reference
engine's: against the golden hashes (reference output stored in tests/golden) and, where the CPU build
of the reference is present, against it directly for more parameter sets."""

import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import BASE, GOLDEN, sc


def mine(lib, resources, delta, pitch):
    out = ctypes.c_char_p()
    lib.check(lib.lib.spkx_setup_json(resources.encode(), json.dumps(delta).encode(), float(pitch), ctypes.byref(out)))
    return lib.take_json(out)


def theirs(ref, ref_engine, delta, pitch):
    out = ctypes.c_char_p()
    ref.check(ref.lib.spkref_setup_json(ref_engine.h, json.dumps(delta).encode(), float(pitch), ctypes.byref(out)))
    return json.loads(out.value.decode())


def test_setup_matches_golden_hashes(lib, resources):
    g = json.load(open(os.path.join(GOLDEN, "golden_setup.json")))
    for name, delta in g["deltas"].items():
        d = mine(lib, resources, delta, g["pitch_um"])
        want = g["sha256"][name]
        for key, h in want.items():
            got = hashlib.sha256(np.asarray(d[key], np.float32).tobytes()).hexdigest()
            assert got == h, (name, key)


@pytest.mark.parametrize("extra", [
    {},
    {"print_exposure": 0.7, "m_filter_shift": -0.3, "y_filter_shift": 0.4, "filter_shift_scale": 5.0},
    {"preflash_exposure": 0.2, "c_filter_neutral": 5.0, "m_filter_neutral": 30.0, "y_filter_neutral": 20.0},
    {"exposure_compensation_ev": -1.5, "density_curve_gamma": 0.8, "grain_sublayers_active": True},
    {"scan_film": True},
    {"enlarger_illuminant": "BB3200"},
    {"product_defaults": True},
])
def test_setup_matches_reference(lib, ref, ref_engine, resources, extra):
    delta = dict(BASE, **extra)
    a = mine(lib, resources, delta, 9.1)
    b = theirs(ref, ref_engine, delta, 9.1)
    for key, v in b.items():
        if key == "f64":
            continue
        x = np.asarray(a[key], np.float32)
        y = np.asarray(v, np.float32)
        assert x.shape == y.shape, key
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), key


@pytest.mark.parametrize("extra", [
    {},
    {"print_exposure": 0.7, "m_filter_shift": -0.3, "y_filter_shift": 0.4, "filter_shift_scale": 5.0},
    {"preflash_exposure": 0.2, "c_filter_neutral": 5.0, "m_filter_neutral": 30.0, "y_filter_neutral": 20.0},
    {"scan_film": True},
    {"output_color_space": "sRGB", "enlarger_illuminant": "BB3200"},
])
def test_binary64_setup_matches_reference(lib, ref, ref_engine, resources, extra):
    """The binary64 values the float64 oracle is fed (this build's set-up) are the reference's own binary64
    values bit for bit, where the reference keeps them: the spectral table, the input matrix, the enlarger
    and scan tables with the exposure factor and preflash, the C_max table and the output matrices. So the
    oracle's inputs are the reference's, not only their narrowed copies."""
    delta = dict(BASE, **extra)
    a = mine(lib, resources, delta, 9.1)["f64"]
    b = theirs(ref, ref_engine, delta, 9.1)["f64"]
    for key, v in b.items():
        x = np.asarray(a[key], np.float64).ravel()
        y = np.asarray(v, np.float64).ravel()
        assert x.shape == y.shape, key
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), (key, float(np.abs(x - y).max()))
