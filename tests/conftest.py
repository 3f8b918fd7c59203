"""Shared fixtures. Tests marked `gpu` need a CUDA device (they run on a B200 box); all others run
on any CPU machine. The checkers (the float64 oracle and the CPU build of the reference engine) are
loaded only here and in the tests."""

import json
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "spektralab-engine_b200")
ORACLE = os.path.join(REPO, "oracle")
GOLDEN = os.path.join(REPO, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

import spk_ctypes as sc  # noqa: E402
import synth_resources  # noqa: E402

BASE = {"film_stock": "synthetic_negative_400", "print_stock": "synthetic_paper", "auto_exposure": False,
        "dir_couplers_active": False, "glare_active": False}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def resources():
    return synth_resources.ensure(sc.RESOURCES)


@pytest.fixture(scope="session")
def lib():
    return sc.load()


@pytest.fixture(scope="session")
def ref(resources):
    if not os.path.exists(sc.REF_PATH):
        pytest.skip("the CPU build of the reference engine (oracle/_ref) is not built here")
    return sc.load_reference()


@pytest.fixture(scope="session")
def ref_engine(ref, resources):
    e = ref.engine(resources)
    yield e
    e.close()


@pytest.fixture(scope="session")
def engine(lib, resources):
    e = lib.engine(resources)
    yield e
    e.close()


def setup_f64(lib, resources, delta, pitch):
    import ctypes
    out = ctypes.c_char_p()
    lib.check(lib.lib.spkx_setup_json(resources.encode(), json.dumps(delta).encode(), float(pitch), ctypes.byref(out)))
    return lib.take_json(out)


def lsb_stats(a, b, label=None):
    """|a - b| of the colour channels of two RGBA16 images in LSB16: max, mean, share and count above 1
    (recorded under the label, or the running test's id, when SPK_TEST_STATS is set)."""
    d = np.abs(a.astype(np.int64) - b.astype(np.int64))[..., :3]
    st = {"max": int(d.max()), "mean": float(d.mean()), "frac_gt1": float((d > 1).mean()),
          "n_gt1": int((d > 1).sum()), "n": int(d.size)}
    record(label or os.environ.get("PYTEST_CURRENT_TEST", "?").split(" ")[0], st)
    return st


def record(label, stats):
    """Append a gate's measured figures to the JSON-lines file named by SPK_TEST_STATS (when set), so that a
    run of the suite leaves the maxima behind, not only a pass."""
    path = os.environ.get("SPK_TEST_STATS")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"gate": label, **stats}) + "\n")


def lsb_gate(got, want, label, max_lsb=1, max_over=0):
    """RGBA16 agreement: alpha equal, and every colour channel within max_lsb LSB16 of want except at most
    max_over of them (which stay within 64). The message carries the maximum and the count above 1."""
    st = lsb_stats(got, want, label)
    d = np.abs(got.astype(np.int64) - want.astype(np.int64))[..., :3]
    st["n_over"] = int((d > max_lsb).sum())
    assert (got[..., 3] == want[..., 3]).all(), (label, "alpha differs")
    assert st["n_over"] <= max_over and (st["n_over"] == 0 or st["max"] <= 64), (label, st)
    return st


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def coupler_steep_mask(f64, D, slope=50.0, margin=1e-5):
    """Values of the negative D (h, w, 3) that the couplers' pre-inverted curve y0 reaches inside a
    segment steeper than `slope` (density per log10 exposure), away from its two ends by `margin`. Where
    the forward development folds, y0 climbs by up to two densities within one knot spacing (and is flat
    on either side), so a binary32 rounding of L - chi (about 1e-7) moves D by slope x 1e-7: the
    reference's binary32 arithmetic and the binary64 oracle part there by up to a few 1e-4."""
    x = np.asarray(f64["curve_x"])
    y0 = np.asarray(f64["couplers"]["y0"]).reshape(3, -1)
    mask = np.zeros(D.shape, bool)
    for c in range(3):
        s = np.diff(y0[c]) / np.diff(x)
        for k in np.where(s > slope)[0]:
            mask[..., c] |= (D[..., c] > y0[c][k] + margin) & (D[..., c] < y0[c][k + 1] - margin)
    return mask, float(max((np.diff(y0[c]) / np.diff(x)).max() for c in range(3)))
