"""Test infrastructure: ctypes front of the float64 oracle (liboracle.so, spk_oracle.c).

Only tests, the smoke check and the benchmark's CPU-baseline leg use this module. It fills the
oracle's OracleSetup from the binary64 set-up that the engine reports (spkx_setup_json, the "f64"
section), which the set-up parity tests pin bit for bit (after narrowing) against the reference
engine's own set-up.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
MAXC = 8

D = ctypes.c_double
I32 = ctypes.c_int32
PD = ctypes.POINTER(ctypes.c_double)


class OracleSetup(ctypes.Structure):
    _fields_ = [
        ("A", D * 9), ("gain", D), ("L", I32), ("table", PD),
        ("n_scatter", I32), ("n_bounce", I32),
        ("scatter_w", (D * 3) * MAXC), ("scatter_s", (D * 3) * MAXC), ("scatter_a", D * 3), ("scatter_b", D * 3),
        ("bounce_w", (D * 3) * MAXC), ("bounce_s", (D * 3) * MAXC), ("mix_a", D * 3), ("mix_b", D * 3),
        ("lens_blur_px", D),
        ("K", I32), ("cx", PD), ("cinv", PD), ("cy", PD),
        ("grain", I32), ("positive", I32), ("gK", I32), ("gaxis", PD), ("ginv", PD), ("glayers", PD),
        ("count", D * 9), ("sat_d", D * 9), ("dmin_l", D * 9), ("uniformity", D * 3), ("dmin_c", D * 3),
        ("final_blur", D), ("amount", D), ("seed", ctypes.c_uint32),
        ("printed", I32), ("enl_eps", D * 243), ("enl_beta", D * 81), ("enl_wt", D * 243), ("g", D * 3),
        ("o", D * 3), ("k_gain", D),
        ("pK", I32), ("px", PD), ("pr", PD), ("py", PD),
        ("scan_eps", D * 243), ("scan_beta", D * 81), ("scan_wt", D * 243), ("to_rgb", D * 9),
        ("cam_k", D * 22), ("m_to_xyz", D * 9), ("m_to_rgb", D * 9), ("m16", D * 9), ("m16_inv", D * 9),
        ("cmax", PD), ("lc_active", I32),
        ("scanner_lens_blur", D), ("unsharp_sigma", D), ("unsharp_amount", D),
        ("cctf_active", I32), ("cctf_mode", I32), ("m_nid", D * 9),
        ("couplers", I32), ("n_dir", I32), ("coupler_m", D * 9), ("dmax", D * 3), ("cy0", PD),
        ("dir_w", (D * 3) * MAXC), ("dir_s", (D * 3) * MAXC),
        ("glare", I32), ("glare_mean", ctypes.c_float), ("glare_sd", ctypes.c_float), ("glare_sigma", D),
        ("glare_tint", D * 3), ("print_seed", ctypes.c_uint32),
        ("boost_ev", D), ("headroom_ev", D),
        ("levels", I32), ("levels_m", D), ("levels_q", D),
        ("edr", I32), ("edr_n", I32), ("edr_r_y", D * 3), ("edr_lo", D), ("edr_hi", D), ("edr_toe", D),
        ("edr_shoulder", D), ("edr_tab", PD),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} is not built (make -C oracle)")
        L = ctypes.CDLL(LIB)
        FP = ctypes.POINTER(ctypes.c_float)
        U16 = ctypes.POINTER(ctypes.c_uint16)
        U32P = ctypes.POINTER(ctypes.c_uint32)
        L.orc_render.argtypes = [ctypes.POINTER(OracleSetup), FP, I32, I32, FP, U16, PD]
        L.orc_develop.argtypes = [ctypes.POINTER(OracleSetup), FP, I32, I32, FP, PD]
        L.orc_print.argtypes = [ctypes.POINTER(OracleSetup), PD, I32, I32, U16, PD]
        L.orc_render_linear.argtypes = [ctypes.POINTER(OracleSetup), PD, I32, I32, FP, PD]
        L.orc_gaussian.argtypes = [PD, PD, I32, I32, PD]
        L.orc_spectral.argtypes = [PD, PD, PD, I32, PD, ctypes.c_int64, PD]
        L.orc_gaussian.restype = None
        L.orc_downscale.argtypes = [FP, I32, I32, I32, I32, FP]
        L.orc_prepare.argtypes = [FP, I32, I32, I32, I32, PD, PD, ctypes.POINTER(I32), ctypes.POINTER(I32)]
        L.orc_render64.argtypes = [ctypes.POINTER(OracleSetup), PD, I32, I32, FP, U16, PD]
        L.orc_meter.argtypes = [PD, I32, I32, PD, PD]
        L.orc_poisson.argtypes = [FP, FP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_poisson.restype = None
        L.orc_lognormal.argtypes = [FP, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_uint32,
                                    ctypes.c_uint32]
        L.orc_lognormal.restype = None
        L.orc_philox.argtypes = [U32P, U32P, U32P, ctypes.c_uint32]
        L.orc_philox.restype = None
        for f in ("orc_logf", "orc_expf", "orc_cosf"):
            getattr(L, f).argtypes = [ctypes.c_float]
            getattr(L, f).restype = ctypes.c_float
        L.orc_uniform.argtypes = [ctypes.c_uint32]
        L.orc_uniform.restype = ctypes.c_float
        L.orc_splitmix_next.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        L.orc_splitmix_next.restype = ctypes.c_uint32
        _lib = L
    return _lib


class Oracle:
    """An OracleSetup plus the arrays it points into (kept alive here)."""

    def __init__(self, f64, seed=0, halation=None, print_exposure=None, rho_tier=1.0, print_seed=0):
        s = OracleSetup()
        self.keep = []

        def buf(values):
            a = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
            self.keep.append(a)
            return a.ctypes.data_as(PD)

        def put(field, values):
            arr = getattr(s, field)
            for i, v in enumerate(values):
                arr[i] = float(v)

        put("A", f64["input_matrix"])
        s.gain = f64["gain"]
        s.L = int(round(len(f64["table"]) / 3) ** 0.5 + 0.5)
        s.table = buf(f64["table"])
        hal = f64["halation"]
        sc = hal["scatter"]
        s.n_scatter = len(sc)
        for k, (w, sg) in enumerate(sc):
            for c in range(3):
                s.scatter_w[k][c] = w[c]
                s.scatter_s[k][c] = sg[c]
        put("scatter_a", hal["scatter_a"])
        put("scatter_b", hal["scatter_b"])
        if halation is not None:  # the test override: (comps, strength); the scatter stage is dropped
            comps, strength = halation
            s.n_scatter = 0
            s.n_bounce = len(comps)
            for k, (w, sg) in enumerate(comps):
                for c in range(3):
                    s.bounce_w[k][c] = w[c]
                    s.bounce_s[k][c] = sg[c]
            put("mix_a", [1.0 / (1.0 + a) for a in strength])
            put("mix_b", [a / (1.0 + a) for a in strength])
        else:
            bo = hal["bounce"]
            s.n_bounce = len(bo)
            for k, (w, sg) in enumerate(bo):
                for c in range(3):
                    s.bounce_w[k][c] = w[c]
                    s.bounce_s[k][c] = sg[c]
            put("mix_a", hal["mix_a"])
            put("mix_b", hal["mix_b"])
        s.lens_blur_px = f64["lens_blur_px"]
        s.K = len(f64["curve_x"])
        s.cx = buf(f64["curve_x"])
        s.cinv = buf(f64["curve_inv"])
        s.cy = buf(f64["curve_y"])
        s.grain = 1 if f64.get("grain_active") else 0
        s.positive = 1 if f64.get("positive") else 0
        if s.grain:
            s.gK = len(f64["grain_axis"]) // 3
            s.gaxis = buf(f64["grain_axis"])
            s.ginv = buf(f64["grain_inv"])
            s.glayers = buf(f64["grain_layers"])
            put("count", f64["grain_count"])
            put("sat_d", f64["grain_sat_d"])
            put("dmin_l", f64["grain_dmin_l"])
            put("uniformity", [0.97, 0.99, 0.97])
            put("dmin_c", [0.03, 0.03, 0.03])
            s.final_blur = f64["grain_final_blur"]
            s.amount = f64["grain_amount"]
        s.seed = seed
        s.printed = 1 if f64["printed"] else 0
        put("enl_eps", f64["enl_eps"])
        put("enl_beta", f64["enl_beta"])
        put("enl_wt", f64["enl_wt"])
        put("g", f64["enl_g"])
        put("o", f64["enl_o"])
        s.k_gain = f64["k_gain"] if print_exposure is None else print_exposure
        if "paper_x" in f64:
            s.pK = len(f64["paper_x"])
            s.px = buf(f64["paper_x"])
            s.pr = buf(f64["paper_r"])
            s.py = buf(f64["paper_y"])
        put("scan_eps", f64["scan_eps"])
        put("scan_beta", f64["scan_beta"])
        put("scan_wt", f64["scan_wt"])
        put("to_rgb", f64["to_rgb"])
        put("cam_k", f64["cam_k"])
        put("m_to_xyz", f64["cam_m_to_xyz"])
        put("m_to_rgb", f64["cam_m_to_rgb"])
        put("m16", f64["cam_m16"])
        put("m16_inv", f64["cam_m16_inv"])
        s.cmax = buf(f64["cmax"])
        s.lc_active = 1
        s.scanner_lens_blur = f64["scanner_lens_blur"]
        s.unsharp_sigma = f64["unsharp_sigma"] * rho_tier  # the unsharp mask's sigma scales with the tier
        s.unsharp_amount = f64["unsharp_amount"]
        s.cctf_active = 1 if f64["cctf_active"] else 0
        s.cctf_mode = int(f64["cctf_mode"])
        put("m_nid", f64["m_nid"])
        s.boost_ev = f64.get("boost_ev", 0.0)
        s.headroom_ev = f64.get("headroom_ev", 0.0)
        ed = f64.get("edr")
        if ed and ed["active"]:
            s.edr, s.edr_n = 1, len(ed["table"])
            put("edr_r_y", ed["r_y"])
            s.edr_lo, s.edr_hi, s.edr_toe, s.edr_shoulder = ed["lo"], ed["hi"], ed["toe"], ed["shoulder"]
            s.edr_tab = buf(ed["table"])
        lv = f64.get("levels")
        if lv and lv["active"]:
            s.levels, s.levels_m, s.levels_q = 1, lv["m"], lv["q"]
        gl = f64.get("glare")
        if gl and gl["draws"]:
            s.glare = 1
            s.glare_mean = gl["mean"]
            s.glare_sd = gl["sd"]
            s.glare_sigma = gl["sigma_full"] * rho_tier
            put("glare_tint", gl["tint"])
            s.print_seed = print_seed
        cp = f64.get("couplers")
        if cp and cp["active"]:
            s.couplers = 1
            put("coupler_m", cp["m"])
            put("dmax", cp["dmax"])
            s.cy0 = buf(cp["y0"])
            s.n_dir = len(cp["dir"])
            for k, (w, sg) in enumerate(cp["dir"]):
                for c in range(3):
                    s.dir_w[k][c] = w[c]
                    s.dir_s[k][c] = sg[c]
        self.s = s

    def render(self, rgb, counts=None):
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w, _ = rgb.shape
        out = np.zeros((h, w, 4), np.uint16)
        neg = np.zeros((h, w, 3), np.float64)
        cp = None
        if counts is not None:
            counts = np.ascontiguousarray(counts, np.float32)
            cp = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lib().orc_render(ctypes.byref(self.s), rgb.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), w, h, cp,
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), neg.ctypes.data_as(PD))
        return out, neg

    def render64(self, rgb64, counts=None):
        """render() of a binary64 frame (the output of prepare())."""
        rgb64 = np.ascontiguousarray(rgb64, np.float64)
        h, w, _ = rgb64.shape
        out = np.zeros((h, w, 4), np.uint16)
        neg = np.zeros((h, w, 3), np.float64)
        cp = None
        if counts is not None:
            counts = np.ascontiguousarray(counts, np.float32)
            cp = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        lib().orc_render64(ctypes.byref(self.s), rgb64.ctypes.data_as(PD), w, h, cp,
                           out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), neg.ctypes.data_as(PD))
        return out, neg

    def render_linear(self, rgb64, counts):
        """The scanned linear RGB of a binary64 frame (the output the render's adjoint differentiates)."""
        rgb64 = np.ascontiguousarray(rgb64, np.float64)
        h, w, _ = rgb64.shape
        counts = np.ascontiguousarray(counts, np.float32)
        lin = np.zeros((h, w, 3), np.float64)
        lib().orc_render_linear(ctypes.byref(self.s), rgb64.ctypes.data_as(PD), w, h,
                                counts.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), lin.ctypes.data_as(PD))
        return lin

    def print(self, negative, print_exposure=None):
        if print_exposure is not None:
            self.s.k_gain = print_exposure
        neg = np.ascontiguousarray(negative, np.float64)
        h, w, _ = neg.shape
        out = np.zeros((h, w, 4), np.uint16)
        lin = np.zeros((h, w, 3), np.float64)
        lib().orc_print(ctypes.byref(self.s), neg.ctypes.data_as(PD), w, h,
                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), lin.ctypes.data_as(PD))
        return out, lin


def spectral(eps, beta, wt, densities):
    """The print's spectral integral in binary64 (orc_spectral): eps (nl, 3), beta (nl,), wt (nl, 3),
    densities (..., 3) -> (..., 3)."""
    eps = np.ascontiguousarray(eps, np.float64)
    beta = np.ascontiguousarray(beta, np.float64)
    wt = np.ascontiguousarray(wt, np.float64)
    d = np.ascontiguousarray(densities, np.float64)
    out = np.zeros(d.shape, np.float64)
    lib().orc_spectral(eps.ctypes.data_as(PD), beta.ctypes.data_as(PD), wt.ctypes.data_as(PD), len(beta),
                       d.ctypes.data_as(PD), d.size // 3, out.ctypes.data_as(PD))
    return out


def downscale_size(w, h, long_edge):
    """The tier image's size (reference src/session/tiers.cpp:50-57)."""
    m = max(w, h)
    if long_edge == 0 or m <= long_edge:
        return w, h
    s = long_edge / m
    return max(1, int(np.floor(w * s))), max(1, int(np.floor(h * s)))


def downscale(rgb, long_edge):
    """The tier image of a float32 frame at a target long edge (orc_downscale; the frame itself when it
    fits)."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w, _ = rgb.shape
    ow, oh = downscale_size(w, h, long_edge)
    if (ow, oh) == (w, h):
        return rgb.copy()
    out = np.zeros((oh, ow, 3), np.float32)
    FP = ctypes.POINTER(ctypes.c_float)
    lib().orc_downscale(rgb.ctypes.data_as(FP), w, h, ow, oh, out.ctypes.data_as(FP))
    return out


GEOMETRY_KEYS = ("geometry_crop_x", "geometry_crop_y", "geometry_crop_w", "geometry_crop_h",
                 "geometry_rotation_deg", "geometry_quarter_turns", "geometry_flip_h", "geometry_flip_v")
GEOMETRY_DEFAULTS = (0.0, 0.0, 1.0, 1.0, 0.0, 0, False, False)


def prepare(rgb, delta, cctf_mode):
    """The input decode (when delta has input_cctf_decoding) and the geometry of delta's geometry_* keys,
    in binary64 (orc_prepare): float32 frame -> float64 frame of the geometry's output size."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w, _ = rgb.shape
    geo = (ctypes.c_double * 8)(*[float(delta.get(k, d)) for k, d in zip(GEOMETRY_KEYS, GEOMETRY_DEFAULTS)])
    out = np.zeros(h * w * 3, np.float64)
    ow, oh = I32(), I32()
    lib().orc_prepare(rgb.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), w, h,
                      1 if delta.get("input_cctf_decoding") else 0, int(cctf_mode), geo, out.ctypes.data_as(PD),
                      ctypes.byref(ow), ctypes.byref(oh))
    return out[: oh.value * ow.value * 3].reshape(oh.value, ow.value, 3)


def print_lut(negative, table, size, lo, hi):
    """The print-preview table render (reference kernels/print.metal:368-407) restated in numpy binary32:
    densities (h, w, 3) through the trilinear S x S x S x 3 table (along k, then j, then i), each operation
    rounded on its own, then the 16-bit encode -> (h, w, 4) uint16."""
    f32 = np.float32
    d = np.asarray(negative, f32)
    T = np.asarray(table, f32).reshape(size, size, size, 3)
    lo = np.asarray(lo, f32)
    sc = np.array([np.float32(1.0 / (float(h_) - float(l_))) for l_, h_ in zip(lo, hi)], f32)
    u = np.minimum(np.maximum((d - lo) * sc, f32(0)), f32(1)) * f32(size - 1)
    fl = np.floor(u)
    i0 = fl.astype(np.int64)
    f = (u - fl).astype(f32)
    i1 = np.minimum(i0 + 1, size - 1)
    one = f32(1)

    def lerp(a, b, t):
        return a * (one - t) + b * t

    idx = [i0, i1]
    c = [[lerp(T[idx[di][..., 0], idx[dj][..., 1], i0[..., 2]], T[idx[di][..., 0], idx[dj][..., 1], i1[..., 2]],
               f[..., 2:3]) for dj in (0, 1)] for di in (0, 1)]
    v = lerp(lerp(c[0][0], c[0][1], f[..., 1:2]), lerp(c[1][0], c[1][1], f[..., 1:2]), f[..., 0:1])
    out = np.zeros(d.shape[:2] + (4,), np.uint16)
    vc = np.minimum(np.maximum(v, f32(0)), f32(1))
    out[..., :3] = np.where(np.isnan(v), 0, np.floor(vc * f32(65535) + f32(0.5))).astype(np.uint16)
    out[..., 3] = 65535
    return out


METER_METHODS = ("center_weighted", "average", "median", "balanced", "center", "protect_highlights",
                 "protect_shadows")


def meter(rgb, rgb_to_xyz):
    """The auto-exposure meter's seven EV values of an image (orc_meter, binary64), by method name."""
    x = np.ascontiguousarray(rgb, np.float64)
    h, w, _ = x.shape
    m = np.ascontiguousarray(np.asarray(rgb_to_xyz, np.float64).reshape(9))
    out = np.zeros(7, np.float64)
    lib().orc_meter(x.ctypes.data_as(PD), w, h, m.ctypes.data_as(PD), out.ctypes.data_as(PD))
    return dict(zip(METER_METHODS, out.tolist()))


def gaussian(plane, sigma3):
    x = np.ascontiguousarray(plane, np.float64)
    h, w, _ = x.shape
    out = np.zeros_like(x)
    sg = (ctypes.c_double * 3)(*[float(v) for v in sigma3])
    lib().orc_gaussian(x.ctypes.data_as(PD), out.ctypes.data_as(PD), w, h, sg)
    return out


def poisson(lam, stream, seed):
    lam = np.ascontiguousarray(lam, np.float32)
    out = np.zeros_like(lam)
    FP = ctypes.POINTER(ctypes.c_float)
    lib().orc_poisson(lam.ctypes.data_as(FP), out.ctypes.data_as(FP), lam.size, stream, seed)
    return out


def lognormal(n, mean, sd, stream, seed):
    out = np.zeros(n, np.float32)
    lib().orc_lognormal(out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, mean, sd, stream, seed)
    return out


def philox(ctr, key):
    ctr = np.ascontiguousarray(ctr, np.uint32).reshape(-1, 4)
    key = np.ascontiguousarray(key, np.uint32).reshape(-1, 2)
    out = np.zeros_like(ctr)
    U = ctypes.POINTER(ctypes.c_uint32)
    lib().orc_philox(ctr.ctypes.data_as(U), key.ctypes.data_as(U), out.ctypes.data_as(U), ctr.shape[0])
    return out


def splitmix(n, state=0x243F6A8885A308D3):
    st = ctypes.c_uint64(state)
    return [lib().orc_splitmix_next(ctypes.byref(st)) for _ in range(n)]
