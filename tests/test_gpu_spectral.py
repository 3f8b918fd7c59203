"""The print's spectral integrals in the spectral-mode kernel (marked gpu): the binary32 path equals the
print kernel bit for bit; each mode's enlarger integral against the float64 oracle's (orc_spectral, at
81 and 401 wavelengths); the 16-bit output after the scan against the float64 oracle's print; the
split-BF16 tensor-core mode through the whole render against the float64 gate; refusals."""

import ctypes

import numpy as np
import pytest

import oracle
from conftest import BASE, lsb_stats, sc, setup_f64

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

NOGRAIN = dict(BASE, grain_active=False)
FIRST_SEED = 0x4ABEA221
# upper bounds of max_p max_k |R - R64| / max_k |R64| for the enlarger integral of densities in [0, 3]
BOUNDS = {"fp64": 1e-7, "fp32_generic": 2e-5, "bf16x3": 1e-4, "tf32": 5e-3, "bf16": 1e-2}


def densities(w, h, seed):
    return np.random.default_rng(seed).uniform(0.0, 3.0, (h, w, 3)).astype(np.float32)


def print_negative(s, neg, mode, bins, contraction=True):
    """(rgba16 (h, w, 4), enlarger integral (h, w, 3) float64 or None, print kernel ms)."""
    h, w, _ = neg.shape
    s.set_print_mode(mode, bins)
    d = torch.from_numpy(neg).cuda()
    stride = (w + 31) // 32 * 32
    out = torch.zeros((h, stride, 4), dtype=torch.int16, device="cuda")
    con = torch.zeros((h, w, 3), dtype=torch.float32, device="cuda") if contraction else None
    ms = s.print_negative(d.data_ptr(), w, h, out.data_ptr(), stride, con.data_ptr() if contraction else None)
    torch.cuda.synchronize()
    rgba = out.cpu().numpy().view(np.uint16)[:, :w].copy()
    return rgba, (con.cpu().numpy().astype(np.float64) if contraction else None), ms


def enlarger_tables(f64, bins):
    """The binary64 enlarger tables at 81 wavelengths, or resampled to 1 nm as the engine does: linear
    interpolation, a 1 nm bin weighing a fifth of a 5 nm bin."""
    eps = np.array(f64["enl_eps"], np.float64).reshape(81, 3)
    beta = np.array(f64["enl_beta"], np.float64)
    wt = np.array(f64["enl_wt"], np.float64).reshape(81, 3)
    if bins == 81:
        return eps, beta, wt
    step = 80.0 / (bins - 1)
    x = np.arange(bins) * step
    i = np.minimum(x.astype(np.int64), 79)
    f = x - i
    lerp = lambda a: (1.0 - f)[:, None] * a[i] + f[:, None] * a[i + 1]
    return lerp(eps), (1.0 - f) * beta[i] + f * beta[i + 1], lerp(wt) * step


def rel_error(R, R64):
    scale = np.abs(R64).max(axis=-1)
    e = np.abs(R - R64).max(axis=-1) / scale
    return float(e.max()), float(e.mean())


@pytest.fixture(scope="module")
def nograin_session(engine):
    s = engine.open(sc.synthetic_image(64, 48, 5), NOGRAIN)
    yield s
    s.close()


def test_generic_fp32_is_the_print_kernel(engine):
    img = sc.synthetic_image(200, 150, 7)
    for delta in (NOGRAIN, BASE):
        with engine.open(img, delta) as s1, engine.open(img, delta) as s2:
            s2.set_print_mode("fp32_generic", 81)
            a, _ = s1.render("full")
            b, _ = s2.render("full")
            assert np.array_equal(a, b)
            s1.set_params({"print_exposure": 1.3})
            s2.set_params({"print_exposure": 1.3})
            assert np.array_equal(s1.reprint("full")[0], s2.reprint("full")[0])
    with engine.open(img, NOGRAIN) as s:
        neg = densities(131, 67, 2)
        a, _, _ = print_negative(s, neg, "fp32", 81, contraction=False)
        b, _, _ = print_negative(s, neg, "fp32_generic", 81)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("bins", [81, 401])
def test_enlarger_integral_against_oracle(engine, lib, resources, nograin_session, bins):
    neg = densities(96, 80, 1)
    f64 = setup_f64(lib, resources, NOGRAIN, 35000.0 / 64)["f64"]
    eps, beta, wt = enlarger_tables(f64, bins)
    R64 = oracle.spectral(eps, beta, wt, neg.astype(np.float64))
    errs = {}
    for mode, bound in BOUNDS.items():
        _, R, _ = print_negative(nograin_session, neg, mode, bins)
        errs[mode] = rel_error(R, R64)
        assert errs[mode][0] <= bound, (mode, bins, errs[mode])
    # the split recovers what a single BF16 product loses
    assert errs["bf16x3"][1] * 20 < errs["bf16"][1], errs


def test_lsb16_after_scan_against_oracle(engine, lib, resources, nograin_session):
    w, h = 128, 96
    neg = densities(w, h, 3)
    f64 = setup_f64(lib, resources, NOGRAIN, 35000.0 / 64)["f64"]
    ref, _ = oracle.Oracle(f64).print(neg.astype(np.float64))
    stats = {}
    for mode in ("fp32", "fp64", "bf16x3", "tf32", "bf16"):
        a, _, _ = print_negative(nograin_session, neg, mode, 81, contraction=False)
        stats[mode] = lsb_stats(a, ref)
        assert (a[..., 3] == 65535).all()
    for mode in ("fp32", "fp64", "bf16x3"):
        assert stats[mode]["frac_gt1"] <= 1e-3 and stats[mode]["max"] <= 4, (mode, stats)
    assert stats["bf16x3"]["mean"] < stats["bf16"]["mean"], stats


@pytest.mark.parametrize("case", ["nograin", "grain_cfg1"])
def test_bf16x3_render_fp64_gate(engine, lib, resources, case):
    w, h = 256, 256
    img = sc.synthetic_image(w, h, 0)
    delta = dict(BASE, grain_active=case != "nograin")
    hal = ([((1, 1, 1), (8, 8, 8)), ((1, 1, 1), (40, 40, 40))], (0.02, 0.02, 0.02)) if case == "grain_cfg1" else None
    with engine.open(img, delta) as s:
        if hal:
            s.set_halation(*hal)
        s.set_print_mode("bf16x3", 81)
        a, _ = s.render("full")
        _, counts = s.develop_debug("full", FIRST_SEED, w, h)
    f64 = setup_f64(lib, resources, delta, 35000.0 / max(w, h))["f64"]
    out, _ = oracle.Oracle(f64, seed=FIRST_SEED, halation=hal).render(img, counts=counts)
    st = lsb_stats(a, out)
    assert st["max"] <= 1, st


def test_spectral_mode_in_a_batch(engine):
    imgs = [sc.synthetic_image(160, 90, 20 + i) for i in range(3)]
    singles = []
    for i, img in enumerate(imgs):
        with engine.open(img, BASE) as s:
            if i == 1:
                s.set_print_mode("bf16x3", 81)
            singles.append(s.render("full")[0])
    ss = [engine.open(img, BASE) for img in imgs]
    try:
        ss[1].set_print_mode("bf16x3", 81)
        res, _ = engine.render_batch(ss, "full")
        for r, want in zip(res, singles):
            assert np.array_equal(r.pixels, want)
            r.free()
    finally:
        for s in ss:
            s.close()


def test_print_mode_refusals(engine, lib, nograin_session):
    s = nograin_session
    for mode, bins in (("fp16", 81), ("bf16x3", 100), ("fp64", 0)):
        with pytest.raises(sc.SpkError) as e:
            s.set_print_mode(mode, bins)
        assert e.value.status == sc.SPK_ERR_INVALID_ARG
    s.set_print_mode("fp32", 81)
    neg = torch.zeros((8, 8, 3), dtype=torch.float32, device="cuda")
    out = torch.zeros((8, 32, 4), dtype=torch.int16, device="cuda")
    con = torch.zeros((8, 8, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(sc.SpkError) as e:
        s.print_negative(neg.data_ptr(), 8, 8, out.data_ptr(), 32, con.data_ptr())
    assert e.value.status == sc.SPK_ERR_INVALID_ARG
    with pytest.raises(sc.SpkError) as e:
        s.print_negative(neg.data_ptr(), 8, 8, out.data_ptr(), 4)
    assert e.value.status == sc.SPK_ERR_INVALID_ARG
