"""Generate the golden fixtures of tests/golden from the reference engine itself.

The reference engine (JamesQiu2005/spektralab-engine) is compiled for the CPU from its own sources by
oracle/Makefile (oracle/_ref/libspektralab_ref.so: its src/ stage code unmodified, its Metal kernels
compiled as C++). This script runs it on the seeded synthetic resources and stores what it returns:

  golden_renders.npz   RGBA16 renders and negatives of a 64 x 48 frame for five parameter sets (the last
                       with the 4K workload's halation and scanner lens blur)
                       (render at print_exposure 1.0 and a reprint at 1.2 of the same negative)
  golden_sampler.npz   the reference's Poisson counts and lognormal values for a lambda grid
  golden_gaussian.npz  the reference's blur of a 97 x 61 plane (kernel path and same-order CPU copy)
  golden_setup.json    SHA-256 of every narrowed kernel constant of two set-ups

Run here (where the reference sources are) with: python tests/golden/make_golden.py
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "spektralab-engine_b200"))

import spk_ctypes as sc  # noqa: E402
import synth_resources  # noqa: E402

BASE = {"film_stock": "synthetic_negative_400", "print_stock": "synthetic_paper", "auto_exposure": False,
        "dir_couplers_active": False, "glare_active": False}
CFG1_HALATION = ([((1, 1, 1), (8, 8, 8)), ((1, 1, 1), (40, 40, 40))], (0.02, 0.02, 0.02))
# the 4K workload's halation (sigma 20 and 120 px, weight 0.03) and scanner lens blur (1.5 px)
CFG2_HALATION = ([((1, 1, 1), (20, 20, 20)), ((1, 1, 1), (120, 120, 120))], (0.03, 0.03, 0.03))

CASES = {
    "nograin_nohalation": (dict(BASE, grain_active=False, halation_active=False), None),
    "nograin_preset": (dict(BASE, grain_active=False), None),
    "grain_preset": (dict(BASE), None),
    "grain_cfg1": (dict(BASE), CFG1_HALATION),
    "nograin_lens_cfg2": (dict(BASE, grain_active=False, scanner_lens_blur=1.5), CFG2_HALATION),
}
W, H = 64, 48
EXPOSURES = (1.0, 1.2)
LAMBDAS = np.array([0.0, 0.5, 3.0, 9.99, 10.0, 37.0, 150.0, 600.0, 2500.0], np.float32)
SETUP_DELTAS = {
    "base": dict(BASE),
    "live": dict(BASE, print_exposure=1.3, m_filter_shift=0.2, y_filter_shift=-0.1, preflash_exposure=0.05,
                 exposure_compensation_ev=0.5, density_curve_gamma=1.1),
}
SETUP_PITCH = 9.114583333333334  # 35 mm over 3840 px


def ref_render(ref, eng, img, delta, halation):
    h, w, _ = img.shape
    comps, strength = halation if halation else ([], (0, 0, 0))
    n = len(comps)
    wts = (ctypes.c_double * max(3 * n, 1))(*[float(v) for c in comps for v in c[0]])
    sig = (ctypes.c_double * max(3 * n, 1))(*[float(v) for c in comps for v in c[1]])
    st = (ctypes.c_double * 3)(*strength)
    ex = (ctypes.c_double * len(EXPOSURES))(*EXPOSURES)
    out = np.zeros((len(EXPOSURES), h, w, 4), np.uint16)
    neg = np.zeros((h, w, 3), np.float32)
    x = np.ascontiguousarray(img, np.float32)
    ref.check(ref.lib.spkref_render(eng.h, x.ctypes.data_as(sc.FP), w, h, json.dumps(delta).encode(), n, wts, sig,
                                    st, ex, len(EXPOSURES), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                                    neg.ctypes.data_as(sc.FP)))
    return out, neg


def setup_hashes(ref, eng, delta):
    out = ctypes.c_char_p()
    ref.check(ref.lib.spkref_setup_json(eng.h, json.dumps(delta).encode(), SETUP_PITCH, ctypes.byref(out)))
    d = json.loads(out.value.decode())
    return {k: hashlib.sha256(np.asarray(v, np.float32).tobytes()).hexdigest() for k, v in sorted(d.items())
            if k != "f64"}


def main():
    synth_resources.ensure(sc.RESOURCES)
    ref = sc.load_reference()
    eng = ref.engine(sc.RESOURCES)
    img = sc.synthetic_image(W, H, 0)
    arrays = {"image": img}
    for name, (delta, hal) in CASES.items():
        out, neg = ref_render(ref, eng, img, delta, hal)
        arrays[f"{name}_rgba"] = out
        arrays[f"{name}_negative"] = neg
    np.savez_compressed(os.path.join(HERE, "golden_renders.npz"), **arrays)
    with open(os.path.join(HERE, "golden_renders.json"), "w") as f:
        json.dump({"cases": {k: {"delta": v[0], "halation": v[1]} for k, v in CASES.items()},
                   "exposures": EXPOSURES, "width": W, "height": H, "seed": 0}, f, indent=1)

    lam = np.repeat(LAMBDAS, 2000)
    counts = np.zeros_like(lam)
    logn = np.zeros_like(lam)
    ref.check(ref.lib.spkref_sampler(eng.h, lam.ctypes.data_as(sc.FP), counts.ctypes.data_as(sc.FP),
                                     logn.ctypes.data_as(sc.FP), lam.size, 7, 1, 1.0, 0.2))
    np.savez_compressed(os.path.join(HERE, "golden_sampler.npz"), lam=lam, counts=counts, lognormal=logn,
                        stream=7, seed=1, mean=1.0, sd=0.2)

    rng = np.random.default_rng(5)
    plane = rng.random((61, 97, 3), dtype=np.float32)
    g = {"plane": plane}
    for k, s3 in enumerate([(0.65, 2.9, 0.0), (1.5, 3.0, 40.0), (0.3, 12.0, 120.0)]):
        sg = (ctypes.c_double * 3)(*s3)
        for mode in (0, 1):
            out = np.zeros_like(plane)
            ref.check(ref.lib.spkref_gaussian(eng.h, plane.ctypes.data_as(sc.FP), out.ctypes.data_as(sc.FP), 97, 61,
                                              sg, mode))
            g[f"s{k}_mode{mode}"] = out
        g[f"s{k}_sigma"] = np.array(s3)
    np.savez_compressed(os.path.join(HERE, "golden_gaussian.npz"), **g)

    with open(os.path.join(HERE, "golden_setup.json"), "w") as f:
        json.dump({"pitch_um": SETUP_PITCH, "deltas": SETUP_DELTAS,
                   "sha256": {k: setup_hashes(ref, eng, d) for k, d in SETUP_DELTAS.items()}}, f, indent=1)
    eng.close()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
