"""Seeded synthetic resources in the spektralab resources-folder layout.

The engine reads one directory (docs/RESOURCE_FORMAT.md of the reference engine):

    <dir>/spektralab_constants.bin     the SPKR constants blob (header 16 B, entries 104 B,
                                       8-aligned little-endian data; docs/RESOURCE_FORMAT.md:213-236)
    <dir>/profiles/<stock>.json        film and paper profiles (docs/RESOURCE_FORMAT.md:38-131)
    <dir>/neutral_print_filters.json   the neutral filter database (docs/RESOURCE_FORMAT.md:155-174)

No real film, paper or colour-science measurement is shipped with the reference, so every
table here is synthetic and smooth:

* CIE 1931 colour matching functions: the multi-lobe piecewise-Gaussian fit of Wyman, Sloan and
  Shirley, "Simple Analytic Approximations to the CIE XYZ Color Matching Functions", JCGT 2(2), 2013.
* Illuminants "D50", "D55", "D65": black bodies at 5003 K, 5503 K and 6504 K with a smooth
  blue-side modulation (daylight-like stand-ins, not the CIE daylight tables).
* "filters/kg3": a smooth logistic long-pass cut at 710 nm (a KG3-like heat filter stand-in).
* "hanatos/spectra_lut": for every chromaticity node, an exp-quadratic spectrum
  s(l) = exp(c0 + c1 u + c2 u^2), u = (l - 580)/200, whose chromaticity is solved to the node's
  (damped Newton; Y = 1).
* Film "synthetic_negative_400": Gaussian layer sensitivities at 650/550/450 nm (sigma 30 nm),
  Gaussian dye spectra at 650/550/450 nm (sigma 40 nm), tanh density curves (Dmin 0.1, Dmax 2.6,
  1024 points over log10 exposure [-3, 1]) centred on the film's mid-grey exposure, and three
  sub-layer curves per channel.
* Paper "synthetic_paper": the same Gaussian form; its curves are a "cdfs" model (three normal
  CDFs per channel), which the printed path requires.

Everything is a pure function of the seed, so two runs give byte-identical files.
"""

from __future__ import annotations

import json
import os
import struct
import sys

import numpy as np

FORMAT_VERSION = "synthetic-resources-v5"
LUT_SIZE = 17
FILM_STOCK = "synthetic_negative_400"
PAPER_STOCK = "synthetic_paper"
L_TABLE = 192  # the engine's spectral-upsampling table size (src/film/film_internal.hpp:19)

WL = 380.0 + 5.0 * np.arange(81)


# ---- colour science stand-ins ------------------------------------------------------------------

def _lobe(l, mu, s1, s2):
    s = np.where(l < mu, s1, s2)
    return np.exp(-0.5 * ((l - mu) / s) ** 2)


def cmfs_1931(l=WL):
    """Wyman-Sloan-Shirley 2013 multi-lobe fit of the CIE 1931 2-degree observer, (81, 3)."""
    x = 1.056 * _lobe(l, 599.8, 37.9, 31.0) + 0.362 * _lobe(l, 442.0, 16.0, 26.7) - 0.065 * _lobe(l, 501.1, 20.4, 26.2)
    y = 0.821 * _lobe(l, 568.8, 46.9, 40.5) + 0.286 * _lobe(l, 530.9, 16.3, 31.1)
    z = 1.217 * _lobe(l, 437.0, 11.8, 36.0) + 0.681 * _lobe(l, 459.0, 26.0, 13.8)
    return np.stack([x, y, z], axis=1)


def blackbody(kelvin, l=WL):
    c1, c2 = 3.741771e-16, 1.4388e-2
    lam = l * 1e-9
    return (c1 / (np.pi * lam ** 5)) / np.expm1(c2 / (lam * kelvin))


def daylight_like(kelvin):
    s = blackbody(kelvin) * (1.0 + 0.08 * np.sin((WL - 380.0) / 400.0 * 3.0 * np.pi))
    return s / s.mean()


def npm(primaries, white):
    """Normalised primary matrix: RGB -> XYZ with white Y = 1 (SMPTE RP 177 construction)."""
    P = np.zeros((3, 3))
    for k in range(3):
        x, y = primaries[2 * k], primaries[2 * k + 1]
        P[:, k] = [x / y, 1.0, (1.0 - x - y) / y]
    W = np.array([white[0] / white[1], 1.0, (1.0 - white[0] - white[1]) / white[1]])
    S = np.linalg.solve(P, W)
    return P * S[None, :]


SPACES = {
    "ProPhoto RGB": ((0.7347, 0.2653, 0.1596, 0.8404, 0.0366, 0.0001), (0.3457, 0.3585)),
    "sRGB": ((0.64, 0.33, 0.30, 0.60, 0.15, 0.06), (0.3127, 0.3290)),
    # inputs for the transfer-function decode tests (published primaries, D65 white)
    "Adobe RGB (1998)": ((0.64, 0.33, 0.21, 0.71, 0.15, 0.06), (0.3127, 0.3290)),
    "ITU-R BT.709": ((0.64, 0.33, 0.30, 0.60, 0.15, 0.06), (0.3127, 0.3290)),
}

# Published cone-response matrices (CIECAM02's CAT02; CAM16's M16, Li et al. 2017).
CAT02 = np.array([[0.7328, 0.4296, -0.1624], [-0.7036, 1.6975, 0.0061], [0.0030, 0.0136, 0.9834]])
CAT16 = np.array([[0.401288, 0.650173, -0.051461], [-0.250268, 1.204414, 0.045854], [-0.002079, 0.048952, 0.953127]])


# ---- the spectral-upsampling table --------------------------------------------------------------

def _xy_of(c, cmf):
    u = (WL - 580.0) / 200.0
    s = np.exp(c[..., 0:1] + c[..., 1:2] * u + c[..., 2:3] * u * u)
    XYZ = s @ cmf
    t = XYZ.sum(-1)
    return XYZ, np.stack([XYZ[..., 0] / t, XYZ[..., 1] / t], -1), s


def spectra_lut(L=L_TABLE):
    """(L, L, 81) float32: node (i, j) sits at chromaticity (1 - sqrt(t0), t1 sqrt(t0))."""
    cmf = cmfs_1931()
    t = np.arange(L) / (L - 1.0)
    t0, t1 = np.meshgrid(t, t, indexing="ij")
    sq = np.sqrt(t0)
    target = np.stack([1.0 - sq, t1 * sq], -1).reshape(-1, 2)
    # keep targets inside a safe region of the chromaticity plane
    target[:, 1] = np.clip(target[:, 1], 0.02, 0.85)
    target[:, 0] = np.clip(target[:, 0], 0.02, 0.75)
    c = np.zeros((target.shape[0], 3))
    for _ in range(40):
        _, xy, _ = _xy_of(c, cmf)
        r = xy - target
        J = np.zeros((c.shape[0], 2, 2))
        for k in (1, 2):
            d = np.zeros(3)
            d[k] = 1e-4
            _, xy2, _ = _xy_of(c + d, cmf)
            J[:, :, k - 1] = (xy2 - xy) / 1e-4
        det = J[:, 0, 0] * J[:, 1, 1] - J[:, 0, 1] * J[:, 1, 0]
        det = np.where(np.abs(det) < 1e-12, 1e-12, det)
        dx = (J[:, 1, 1] * r[:, 0] - J[:, 0, 1] * r[:, 1]) / det
        dy = (-J[:, 1, 0] * r[:, 0] + J[:, 0, 0] * r[:, 1]) / det
        step = np.stack([dx, dy], -1)
        n = np.linalg.norm(step, axis=-1, keepdims=True)
        step = step * np.minimum(1.0, 4.0 / np.maximum(n, 1e-30))
        c[:, 1:] -= 0.7 * step
        c[:, 1] = np.clip(c[:, 1], -40.0, 40.0)
        c[:, 2] = np.clip(c[:, 2], -60.0, 25.0)
    XYZ, _, s = _xy_of(c, cmf)
    s = s / XYZ[:, 1:2]  # Y = 1
    return s.reshape(L, L, 81).astype(np.float32)


# ---- profiles -----------------------------------------------------------------------------------

def _gauss(mu, sigma):
    return np.exp(-0.5 * ((WL - mu) / sigma) ** 2)


def _log_sens(mus, sigma=30.0):
    return np.stack([np.log10(np.maximum(_gauss(m, sigma), 1e-300)) for m in mus], 1)


def _dyes(mus, sigma=40.0):
    return np.stack([_gauss(m, sigma) for m in mus], 1)


def _tanh_curve(le, centre, dmin=0.1, dmax=2.6, gamma=1.4):
    return dmin + (dmax - dmin) * 0.5 * (np.tanh(gamma * (le - centre)) + 1.0)


def film_midgrey_log_exposure(lut, sens_log, illum_xy):
    """log10 of the film exposure of an 18.4 % grey at the reference illuminant's chromaticity,
    evaluated on the nearest table node (enough to centre the synthetic curves)."""
    L = lut.shape[0]
    x, y = illum_xy
    o = 1.0 - x
    t0, t1 = min(max(o * o, 0.0), 1.0), min(max(y / max(o, 1e-10), 0.0), 1.0)
    i, j = int(round(t0 * (L - 1))), int(round(t1 * (L - 1)))
    S = 10.0 ** sens_log
    T = lut[i, j].astype(np.float64) @ S
    b = 0.184 / max(y, 1e-6)  # X + Y + Z of a grey with Y = 0.184
    return np.log10(b * T)


def profile_film(lut, illum_xy_d55):
    le = np.linspace(-3.0, 1.0, 1024)
    mus = (650.0, 550.0, 450.0)
    sens = _log_sens(mus)
    centres = film_midgrey_log_exposure(lut, sens, illum_xy_d55)
    curves = np.stack([_tanh_curve(le, centres[c]) for c in range(3)], 1)
    # sub-layers fast / medium / slow: shifted, scaled copies of the channel curve
    layers = np.zeros((le.size, 3, 3))
    shifts, fracs = (-0.35, 0.0, 0.35), (0.30, 0.35, 0.35)
    for c in range(3):
        for l in range(3):
            layers[:, l, c] = fracs[l] * (_tanh_curve(le, centres[c] + shifts[l], 0.0, 2.5))
    base = 0.05 + 0.15 * np.exp(-(WL - 380.0) / 50.0)
    return {
        "info": {"stock": FILM_STOCK, "name": "Synthetic negative 400", "type": "negative", "support": "film",
                 "use": "still", "antihalation": "weak", "reference_illuminant": "D55",
                 "viewing_illuminant": "D50"},
        "data": {
            "wavelengths": WL.tolist(),
            "log_sensitivity": sens.tolist(),
            "channel_density": _dyes(mus).tolist(),
            "base_density": base.tolist(),
            "log_exposure": le.tolist(),
            "density_curves": curves.tolist(),
            "density_curves_layers": layers.tolist(),
            "hanatos2025_adaptation_window_params": [],
        },
    }


def profile_paper():
    le = np.linspace(-3.0, 1.0, 1024)
    mus = (650.0, 550.0, 450.0)
    centers = np.array([[-0.35, 0.0, 0.35]] * 3) + np.array([[0.05], [0.0], [-0.05]])
    amplitudes = np.array([[0.75, 0.95, 0.80]] * 3)
    sigmas = np.array([[0.22, 0.25, 0.28]] * 3)
    from math import erfc, sqrt

    curves = np.zeros((le.size, 3))
    for c in range(3):
        for l in range(3):
            z = (le - centers[c, l]) / sigmas[c, l]
            curves[:, c] += amplitudes[c, l] * 0.5 * np.array([erfc(-v / sqrt(2.0)) for v in z])
    curves += 0.06
    return {
        "info": {"stock": PAPER_STOCK, "name": "Synthetic paper", "type": "negative", "support": "paper",
                 "viewing_illuminant": "D50"},
        "data": {
            "wavelengths": WL.tolist(),
            "log_sensitivity": _log_sens(mus).tolist(),
            "channel_density": _dyes(mus).tolist(),
            "base_density": (0.03 + 0.02 * np.exp(-(WL - 380.0) / 40.0)).tolist(),
            "log_exposure": le.tolist(),
            "density_curves": curves.tolist(),
            "density_curves_model": {"model_type": "cdfs", "centers": centers.tolist(),
                                     "amplitudes": amplitudes.tolist(), "sigmas": sigmas.tolist()},
            # an EDR tone map: identity between toe (2^-8) and shoulder (2^-0.5), both on knots of the 0.5-step
            # table, shadows lifted (slope 0.8) and highlights compressed (slope 0.5) outside, in log2 Y
            "edr_tone_map": {"version": 1, "domain_log2_y": [-14.0, 3.0], "toe_y": 2.0 ** -8, "shoulder_y": 2.0 ** -0.5,
                             "target_log2_y": [x if -8.0 <= x <= -0.5 else
                                               (-8.0 + 0.8 * (x + 8.0) if x < -8.0 else -0.5 + 0.5 * (x + 0.5))
                                               for x in np.linspace(-14.0, 3.0, 35).tolist()]},
        },
    }


# ---- the SPKR blob --------------------------------------------------------------------------------

_DTYPES = {np.dtype(np.float64): 0, np.dtype(np.float32): 1, np.dtype(np.float16): 2,
           np.dtype(np.int32): 3, np.dtype(np.uint8): 4}


def write_blob(path, entries):
    """entries: list of (name, ndarray). Header, 104-byte entry table, 8-aligned C-order data."""
    count = len(entries)
    head = 16 + 104 * count
    off = (head + 7) // 8 * 8
    table = bytearray()
    datas = []
    for name, arr in entries:
        a = np.ascontiguousarray(arr)
        nb = name.encode("utf-8")
        assert len(nb) <= 63
        dims = list(a.shape) + [0] * (4 - a.ndim)
        table += nb + b"\0" * (64 - len(nb))
        table += struct.pack("<II4I", _DTYPES[a.dtype], a.ndim, *dims)
        table += struct.pack("<QQ", off, a.nbytes)
        datas.append((off, a.tobytes()))
        off = (off + a.nbytes + 7) // 8 * 8
    buf = bytearray(off)
    buf[0:16] = b"SPKR" + struct.pack("<III", 1, count, 0)
    buf[16:16 + len(table)] = table
    for o, d in datas:
        buf[o:o + len(d)] = d
    with open(path, "wb") as f:
        f.write(bytes(buf))


def generate(out_dir, seed=0):
    """Write the synthetic resources folder; returns out_dir. The seed only salts the spare
    'present, unused' entries: every table the render reads is a fixed function of this file."""
    rng = np.random.default_rng(seed)
    os.makedirs(os.path.join(out_dir, "profiles"), exist_ok=True)
    cmf = cmfs_1931()
    lut = spectra_lut()
    entries = [
        ("spectral/wavelengths", WL.astype(np.float64)),
        ("colour/cmfs_1931_2deg", cmf.astype(np.float64)),
        ("colour/cmfs_lms", rng.random((81, 3))),
        ("colour/matrix_16", CAT16.copy()),
        ("colour/mallett_srgb_basis", rng.random((81, 3))),
        ("hanatos/spectra_lut", lut),
        ("colour/cat/CAT02", CAT02.copy()),
        ("colour/cat/CAT16", CAT16.copy()),
        ("colour/sd_illuminant/D50", daylight_like(5003.0)),
        ("colour/sd_illuminant/D55", daylight_like(5503.0)),
        ("colour/sd_illuminant/D65", daylight_like(6504.0)),
        ("filters/kg3", 0.92 / (1.0 + np.exp((WL - 710.0) / 25.0))),
    ]
    for name, (prim, white) in SPACES.items():
        M = npm(prim, white)
        entries += [
            (f"colour/cs/{name}/primaries", np.array(prim, dtype=np.float64)),
            (f"colour/cs/{name}/whitepoint", np.array(white, dtype=np.float64)),
            (f"colour/cs/{name}/matrix_RGB_to_XYZ", M),
            (f"colour/cs/{name}/matrix_XYZ_to_RGB", np.linalg.inv(M)),
        ]
    # a print-preview table for the synthetic paper: densities (three axes 0..3.2) -> a smooth display RGB
    S = LUT_SIZE
    ax = np.linspace(0.0, 3.2, S)
    di, dj, dk = np.meshgrid(ax, ax, ax, indexing="ij")
    T = np.stack([10.0 ** -(0.9 * di + 0.1 * dj), 10.0 ** -(0.1 * di + 0.8 * dj + 0.1 * dk),
                  10.0 ** -(0.15 * dj + 0.85 * dk)], axis=-1) ** (1 / 2.2)
    entries += [
        (f"print_lut/{PAPER_STOCK}", T.astype(np.float32)),
        (f"print_lut_axes/{PAPER_STOCK}", np.stack([ax, ax * 1.05, ax * 0.95]).astype(np.float32)),
    ]
    write_blob(os.path.join(out_dir, "spektralab_constants.bin"), entries)

    d55 = daylight_like(5503.0)
    X = d55 @ cmf
    xy55 = (X[0] / X.sum(), X[1] / X.sum())
    with open(os.path.join(out_dir, "profiles", FILM_STOCK + ".json"), "w") as f:
        json.dump(profile_film(lut, xy55), f)
    with open(os.path.join(out_dir, "profiles", PAPER_STOCK + ".json"), "w") as f:
        json.dump(profile_paper(), f)
    with open(os.path.join(out_dir, "neutral_print_filters.json"), "w") as f:
        json.dump({PAPER_STOCK: {"TH-KG3": {FILM_STOCK: [0.0, 10.0, 10.0]}}}, f)
    with open(os.path.join(out_dir, "print_luts.json"), "w") as f:
        json.dump({PAPER_STOCK: {"paired_film": FILM_STOCK, "lut_size": LUT_SIZE, "declared_pairing": True,
                                 "output_color_space": "sRGB", "output_cctf_encoding": True}}, f)
    with open(os.path.join(out_dir, "VERSION"), "w") as f:
        f.write(FORMAT_VERSION + "\n")
    return out_dir


def ensure(out_dir):
    """Generate into out_dir unless a current copy is already there."""
    stamp = os.path.join(out_dir, "VERSION")
    try:
        with open(stamp) as f:
            if f.read().strip() == FORMAT_VERSION:
                return out_dir
    except OSError:
        pass
    return generate(out_dir)


if __name__ == "__main__":
    print(generate(sys.argv[1] if len(sys.argv) > 1 else "synthetic_resources"))
