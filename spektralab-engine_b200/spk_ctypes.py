"""ctypes binding of the spektralab C ABI (include/spektralab.h) and of the B200 extensions
(include/spektralab_b200.h).

The same binding loads the B200 library (libspektralab.so beside this file) and the CPU build of the
reference engine used as the oracle (oracle/_ref/libspektralab_ref.so); both export the reference's
26 entry points with identical signatures. Mirrors the role of the reference's tests/spk_ctypes.py:
signatures bound once, RGBA16 results read through row_stride_px.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libspektralab.so")
REF_PATH = os.path.join(REPO, "oracle", "_ref", "libspektralab_ref.so")
RESOURCES = os.path.join(REPO, "_build", "resources")

SPK_OK = 0
SPK_ERR_INVALID_ARG = -1
SPK_ERR_USER = -2
SPK_ERR_UNSUPPORTED = -4
SPK_ERR_GPU = -5
SPK_ERR_IO = -6
SPK_ERR_CANCELLED = -7


class SpkImage(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(ctypes.c_float)), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("channels", ctypes.c_uint32)]


class SpkDeviceImage(ctypes.Structure):
    _fields_ = [("buffer", ctypes.c_void_p), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("channels", ctypes.c_uint32)]


class SpkResult(ctypes.Structure):
    _fields_ = [("rgba16", ctypes.POINTER(ctypes.c_uint16)), ("texture", ctypes.c_void_p),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("row_stride_px", ctypes.c_uint32),
                ("elapsed_ms", ctypes.c_double), ("reprint", ctypes.c_int32),
                ("negative_was_cached", ctypes.c_int32), ("progress_id", ctypes.c_char * 40)]


assert ctypes.sizeof(SpkImage) == 24 and ctypes.sizeof(SpkResult) == 88

P = ctypes.c_void_p
C = ctypes.c_char_p
PS = ctypes.POINTER(ctypes.c_char_p)
I32 = ctypes.c_int32
U32 = ctypes.c_uint32

# name -> (restype, argtypes); the 26 entry points of the reference ABI
ABI = {
    "spk_engine_create": (P, [C, P]),
    "spk_engine_create_for_device": (P, [C, P, I32]),
    "spk_engine_destroy": (None, [P]),
    "spk_engine_trim": (ctypes.c_size_t, [P]),
    "spk_build_info": (C, []),
    "spk_capabilities": (C, [P]),
    "spk_params_schema": (C, [P]),
    "spk_memory_report": (C, [P]),
    "spk_warm_up": (I32, [P, C, C, PS]),
    "spk_open": (P, [P, ctypes.POINTER(SpkImage), C, PS]),
    "spk_open_device": (P, [P, ctypes.POINTER(SpkDeviceImage), C, PS]),
    "spk_set_params": (I32, [P, C, PS]),
    "spk_get_params": (I32, [P, PS]),
    "spk_session_release": (None, [P]),
    "spk_render": (I32, [P, C, ctypes.POINTER(SpkResult)]),
    "spk_reprint": (I32, [P, C, ctypes.POINTER(SpkResult)]),
    "spk_result_free": (None, [ctypes.POINTER(SpkResult)]),
    "spk_solve": (I32, [P, C, PS]),
    "spk_print_lut_catalog": (C, [P]),
    "spk_print_lut_table": (I32, [P, C, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)), ctypes.POINTER(U32)]),
    "spk_preview_stock_lut": (I32, [P, C, C, ctypes.POINTER(SpkResult), PS]),
    "spk_output_transform": (I32, [P, C, C, C, PS, ctypes.POINTER(ctypes.POINTER(ctypes.c_float)),
                                   ctypes.POINTER(U32)]),
    "spk_cancel": (None, [P, C]),
    "spk_progress": (I32, [P, C, PS]),
    "spk_string_free": (None, [ctypes.c_void_p]),
    "spk_last_error": (C, [P]),
}

FP = ctypes.POINTER(ctypes.c_float)
DP = ctypes.POINTER(ctypes.c_double)
UP = ctypes.POINTER(ctypes.c_uint32)
EXT = {
    "spkx_session_set_halation": (I32, [P, U32, DP, DP, DP]),
    "spkx_session_profile": (I32, [P, C, I32, U32, PS]),
    "spkx_session_negative": (I32, [P, C, FP, ctypes.c_size_t]),
    "spkx_session_meter": (I32, [P, PS]),
    "spkx_session_tier_image": (I32, [P, C, FP, ctypes.c_size_t, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
    "spkx_session_setup_json": (I32, [P, ctypes.c_double, PS]),
    "spkx_sampler_poisson": (I32, [FP, FP, U32, U32, U32]),
    "spkx_sampler_lognormal": (I32, [FP, U32, ctypes.c_float, ctypes.c_float, U32, U32]),
    "spkx_philox": (I32, [UP, UP, UP, U32]),
    "spkx_gaussian": (I32, [FP, FP, U32, U32, DP]),
    "spkx_setup_json": (I32, [C, C, ctypes.c_double, PS]),
    "spkx_session_develop_debug": (I32, [P, C, U32, FP, FP]),
    "spkx_session_develop_draws": (I32, [P, C, U32, FP, FP]),
    "spk_render_vjp": (I32, [P, C, U32, FP, FP, DP, U32, FP]),
    "spkx_render_batch": (I32, [ctypes.POINTER(P), U32, C, I32, ctypes.POINTER(SpkResult), PS]),
    "spkx_engine_batch_plan": (I32, [P, C]),
    "spkx_session_set_print_mode": (I32, [P, C, U32]),
    "spkx_print_negative": (I32, [P, P, U32, U32, P, U32, P, ctypes.POINTER(ctypes.c_double)]),
    "spkx_test_set_tc_wait_limit": (I32, [ctypes.c_int64]),
    "spkx_test_set_iir_wait_limit": (I32, [ctypes.c_int64]),
    "spkx_test_take_iir_waits_given_up": (I32, [UP]),
}

REF_EXT = {
    "spkref_render": (I32, [P, FP, U32, U32, C, U32, DP, DP, DP, DP, U32, ctypes.POINTER(ctypes.c_uint16), FP]),
    "spkref_setup_json": (I32, [P, C, ctypes.c_double, PS]),
    "spkref_sampler": (I32, [P, FP, FP, FP, U32, U32, U32, ctypes.c_float, ctypes.c_float]),
    "spkref_gaussian": (I32, [P, FP, FP, U32, U32, DP, I32]),
    "spkref_open": (P, [P, FP, U32, U32, C, U32, DP, DP, DP]),
    "spkref_develop": (I32, [P]),
    "spkref_print": (I32, [P, ctypes.c_double, ctypes.POINTER(ctypes.c_uint16)]),
    "spkref_close": (None, [P]),
    "spkref_meter": (I32, [FP, U32, U32, DP, DP]),
    "spkref_downscale": (I32, [FP, U32, U32, U32, FP, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
}


def reference_downscale(ref, rgb, long_edge):
    """The reference engine's CPU tier downscale (spkref_downscale) of a float32 frame."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w, _ = img.shape
    out = np.zeros(h * w * 3, np.float32)
    ow, oh = U32(), U32()
    ref.check(ref.lib.spkref_downscale(img.ctypes.data_as(FP), w, h, long_edge, out.ctypes.data_as(FP),
                                       ctypes.byref(ow), ctypes.byref(oh)))
    return out[: ow.value * oh.value * 3].reshape(oh.value, ow.value, 3)


def reference_meter(ref, rgb, rgb_to_xyz):
    """The reference engine's meter statistics (spkref_meter) of a float32 image, by method name."""
    img = np.ascontiguousarray(rgb, np.float32)
    h, w, _ = img.shape
    m = np.ascontiguousarray(np.asarray(rgb_to_xyz, np.float64).reshape(9))
    out = np.zeros(7, np.float64)
    ref.check(ref.lib.spkref_meter(img.ctypes.data_as(FP), w, h, m.ctypes.data_as(DP), out.ctypes.data_as(DP)))
    names = ("center_weighted", "average", "median", "balanced", "center", "protect_highlights", "protect_shadows")
    return dict(zip(names, out.tolist()))


class SpkError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"status {status}: {message}")
        self.status = status


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


class Library:
    """One loaded library (the B200 engine or the reference oracle)."""

    def __init__(self, path, extensions=True):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built")
        self.path = path
        self.lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        _bind(self.lib, ABI)
        self.has_ext = extensions
        if extensions:
            _bind(self.lib, EXT)

    def last_error(self):
        return (self.lib.spk_last_error(None) or b"").decode()

    def check(self, status):
        if status != SPK_OK:
            raise SpkError(status, self.last_error())

    def take_json(self, out):
        if not out.value:
            return None
        text = out.value.decode()
        self.lib.spk_string_free(ctypes.cast(out, ctypes.c_void_p))
        return json.loads(text)

    def engine(self, resources=RESOURCES, device=None):
        dev = ctypes.c_int(device) if device is not None else None
        e = self.lib.spk_engine_create(resources.encode(), ctypes.byref(dev) if dev is not None else None)
        if not e:
            raise SpkError(-1, self.last_error())
        return Engine(self, e)


class Engine:
    def __init__(self, lib, handle):
        self.L = lib
        self.h = handle

    def close(self):
        if self.h:
            self.L.lib.spk_engine_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def open(self, image, delta=None):
        img = np.ascontiguousarray(image, dtype=np.float32)
        h, w, c = img.shape
        si = SpkImage(img.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), w, h, c)
        out = ctypes.c_char_p()
        d = json.dumps(delta).encode() if isinstance(delta, dict) else (delta.encode() if delta else None)
        s = self.L.lib.spk_open(self.h, ctypes.byref(si), d, ctypes.byref(out))
        if not s:
            raise SpkError(-2, self.L.last_error())
        return Session(self, s, self.L.take_json(out), (h, w))

    def batch_plan(self, plan=None):
        """Pins the plan of later render_batch calls (None: timed choice)."""
        self.L.check(self.L.lib.spkx_engine_batch_plan(self.h, plan.encode() if plan else None))

    def render_batch(self, sessions, tier="full", reprint=False):
        """spkx_render_batch over Session objects of this engine: ([Result, ...], info dict). Each Result owns
        its spk_result until .free()."""
        n = len(sessions)
        hs = (P * max(n, 1))(*[s.h for s in sessions])
        rs = (SpkResult * max(n, 1))()
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spkx_render_batch(hs, n, tier.encode() if tier is not None else None, int(reprint),
                                                  rs, ctypes.byref(out)))
        info = self.L.take_json(out)
        results = []
        for i in range(n):
            r = SpkResult()
            ctypes.memmove(ctypes.byref(r), ctypes.byref(rs[i]), ctypes.sizeof(SpkResult))
            results.append(Result(self.L, r))
        return results, info


class Result:
    """An spk_result held open: .pixels is a (height, width, 4) uint16 view of its pinned host pixels,
    valid until .free()."""

    def __init__(self, lib, r):
        self.L = lib
        self.r = r
        self.pixels = np.ctypeslib.as_array(r.rgba16, shape=(r.height, r.row_stride_px, 4))[:, : r.width]
        self.row_stride_px = r.row_stride_px

    def free(self):
        if self.r is not None:
            self.pixels = None
            self.L.lib.spk_result_free(ctypes.byref(self.r))
            self.r = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


class Session:
    def __init__(self, engine, handle, reply, shape=None):
        self.E = engine
        self.L = engine.L
        self.h = handle
        self.reply = reply
        self.shape = shape  # (height, width) of the source frame

    def close(self):
        if self.h:
            self.L.lib.spk_session_release(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_params(self, delta):
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spk_set_params(self.h, json.dumps(delta).encode(), ctypes.byref(out)))
        return self.L.take_json(out)

    def _render(self, fn, tier):
        r = SpkResult()
        self.L.check(fn(self.h, tier.encode(), ctypes.byref(r)))
        try:
            a = np.ctypeslib.as_array(r.rgba16, shape=(r.height, r.row_stride_px, 4))[:, : r.width].copy()
            meta = {"reprint": r.reprint, "negative_was_cached": r.negative_was_cached,
                    "elapsed_ms": r.elapsed_ms, "row_stride_px": r.row_stride_px,
                    "progress_id": r.progress_id.decode()}
        finally:
            self.L.lib.spk_result_free(ctypes.byref(r))
        return a, meta

    def render(self, tier="full"):
        return self._render(self.L.lib.spk_render, tier)

    def preview_lut(self, print_stock=None, tier="live"):
        """spk_preview_stock_lut: (RGBA16 (h, w, 4), meta, reply)."""
        r = SpkResult()
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spk_preview_stock_lut(self.h, print_stock.encode() if print_stock else None,
                                                      tier.encode() if tier else None, ctypes.byref(r),
                                                      ctypes.byref(out)))
        try:
            a = np.ctypeslib.as_array(r.rgba16, shape=(r.height, r.row_stride_px, 4))[:, : r.width].copy()
            meta = {"reprint": r.reprint, "negative_was_cached": r.negative_was_cached}
        finally:
            self.L.lib.spk_result_free(ctypes.byref(r))
        return a, meta, self.L.take_json(out)

    def reprint(self, tier="full"):
        return self._render(self.L.lib.spk_reprint, tier)

    def render_linear(self, film_seed, tier="full"):
        """The scanned linear RGB (the output spk_render_vjp differentiates), (h, w, 3) float32, with the
        grain counts of film_seed."""
        h, w = self.shape
        y = np.empty((h, w, 3), np.float32)
        self.L.check(self.L.lib.spk_render_vjp(self.h, tier.encode(), film_seed, None, None, None, 0,
                                                y.ctypes.data_as(FP)))
        return y

    def render_vjp(self, grad_output, film_seed, n_params=0, tier="full", want_output=False):
        """spk_render_vjp: (grad_input (h, w, 3) float32, grad_params float64[n_params][, output])."""
        h, w = self.shape
        gy = np.ascontiguousarray(grad_output, np.float32)
        gx = np.empty((h, w, 3), np.float32)
        gp = np.zeros(max(n_params, 1), np.float64)
        y = np.empty((h, w, 3), np.float32) if want_output else None
        self.L.check(self.L.lib.spk_render_vjp(self.h, tier.encode(), film_seed, gy.ctypes.data_as(FP),
                                                gx.ctypes.data_as(FP), gp.ctypes.data_as(DP), n_params,
                                                y.ctypes.data_as(FP) if want_output else None))
        return (gx, gp[:n_params], y) if want_output else (gx, gp[:n_params])

    def render_result(self, tier="full", reprint=False):
        """spk_render / spk_reprint without a copy: a Result that owns the spk_result (its pinned host
        pixels and device image) until .free()."""
        r = SpkResult()
        fn = self.L.lib.spk_reprint if reprint else self.L.lib.spk_render
        self.L.check(fn(self.h, tier.encode(), ctypes.byref(r)))
        return Result(self.L, r)

    # ---- extensions ----
    def set_halation(self, comps, strength):
        """comps: list of (weight3, sigma3_px); strength: A per channel."""
        n = len(comps)
        w = (ctypes.c_double * max(3 * n, 1))(*[float(v) for c in comps for v in c[0]])
        s = (ctypes.c_double * max(3 * n, 1))(*[float(v) for c in comps for v in c[1]])
        a = (ctypes.c_double * 3)(*[float(v) for v in strength])
        self.L.check(self.L.lib.spkx_session_set_halation(self.h, n, w, s, a))

    def profile(self, tier="full", reprint=False, steps=3):
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spkx_session_profile(self.h, tier.encode(), int(reprint), steps, ctypes.byref(out)))
        return self.L.take_json(out)

    def meter(self):
        """spkx_session_meter: the seven auto-exposure EV values."""
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spkx_session_meter(self.h, ctypes.byref(out)))
        return self.L.take_json(out)

    def tier_image(self, tier):
        """spkx_session_tier_image: the tier's image, (h, w, 3) float32."""
        w, h = U32(), U32()
        self.L.check(self.L.lib.spkx_session_tier_image(self.h, tier.encode(), None, 0, ctypes.byref(w),
                                                        ctypes.byref(h)))
        buf = np.empty((h.value, w.value, 3), np.float32)
        self.L.check(self.L.lib.spkx_session_tier_image(self.h, tier.encode(), buf.ctypes.data_as(FP), buf.size,
                                                        ctypes.byref(w), ctypes.byref(h)))
        return buf

    def negative(self, tier, w, h):
        buf = np.empty((h, w, 3), np.float32)
        self.L.check(self.L.lib.spkx_session_negative(self.h, tier.encode(), buf.ctypes.data_as(FP), buf.size))
        return buf

    def develop_debug(self, tier, seed, w, h, counts=True):
        neg = np.empty((h, w, 3), np.float32)
        cnt = np.zeros((h, w, 9), np.float32) if counts else None
        self.L.check(self.L.lib.spkx_session_develop_debug(self.h, tier.encode(), seed, neg.ctypes.data_as(FP),
                                                           cnt.ctypes.data_as(FP) if counts else None))
        return neg, cnt

    def set_print_mode(self, mode, bins=81):
        """spkx_session_set_print_mode: fp32, fp32_generic, fp64, tf32, bf16 or bf16x3 at 81 or 401 wavelengths."""
        self.L.check(self.L.lib.spkx_session_set_print_mode(self.h, mode.encode(), bins))

    def print_negative(self, negative_ptr, width, height, rgba16_ptr, row_stride_px, contraction_ptr=None):
        """spkx_print_negative on device pointers (ints); returns the print kernel's device time in ms."""
        ms = ctypes.c_double()
        self.L.check(self.L.lib.spkx_print_negative(self.h, negative_ptr, width, height, rgba16_ptr, row_stride_px,
                                                    contraction_ptr, ctypes.byref(ms)))
        return ms.value

    def develop_draws(self, tier, seed, w, h):
        """(counts, lambdas), each (h, w, 9) float32 [c][l]: the grain's draws of one develop."""
        cnt = np.zeros((h, w, 9), np.float32)
        lam = np.zeros((h, w, 9), np.float32)
        self.L.check(self.L.lib.spkx_session_develop_draws(self.h, tier.encode(), seed, cnt.ctypes.data_as(FP),
                                                           lam.ctypes.data_as(FP)))
        return cnt, lam

    def setup_json(self, pitch_um):
        out = ctypes.c_char_p()
        self.L.check(self.L.lib.spkx_session_setup_json(self.h, float(pitch_um), ctypes.byref(out)))
        return self.L.take_json(out)


def load(path=LIB_PATH):
    return Library(path)


def load_reference(path=REF_PATH):
    """The reference engine built for the CPU (oracle); its driver adds the spkref_* entry points."""
    lib = Library(path, extensions=False)
    _bind(lib.lib, REF_EXT)
    return lib


def synthetic_image(w, h, seed=0):
    """Linear ProPhoto RGB, per pixel and channel v = 2^(-8 + 10 u), u from Philox4x32-10 with
    counter (pixel, channel, 0, 0) and key (seed, 0): the same numbers in C++ and Python."""
    n = w * h
    pix = np.arange(n, dtype=np.uint64)
    out = np.empty((n, 3), np.float32)
    for c in range(3):
        words = philox_np(pix, np.full(n, c, np.uint64), seed)
        u = ((words >> np.uint64(8)).astype(np.float32) + np.float32(0.5)) * np.float32(2.0 ** -24)
        out[:, c] = np.exp2(np.float32(-8.0) + np.float32(10.0) * u).astype(np.float32)
    return out.reshape(h, w, 3)


M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox_np(c0, c1, k0, c2=None, c3=None, k1=0):
    """Philox4x32-10 (Salmon et al. 2011) vectorised in numpy; returns the x word of the block."""
    mask = np.uint64(0xFFFFFFFF)
    n = len(c0)
    x = np.asarray(c0, np.uint64) & mask
    y = np.asarray(c1, np.uint64) & mask
    z = np.zeros(n, np.uint64) if c2 is None else np.asarray(c2, np.uint64)
    w = np.zeros(n, np.uint64) if c3 is None else np.asarray(c3, np.uint64)
    ka = np.full(n, k0, np.uint64)
    kb = np.full(n, k1, np.uint64)
    for _ in range(10):
        p0 = np.uint64(M0) * x
        p1 = np.uint64(M1) * z
        x, y, z, w = ((p1 >> np.uint64(32)) ^ y ^ ka) & mask, p1 & mask, ((p0 >> np.uint64(32)) ^ w ^ kb) & mask, p0 & mask
        ka = (ka + np.uint64(W0)) & mask
        kb = (kb + np.uint64(W1)) & mask
    return x
