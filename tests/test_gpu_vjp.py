"""The render's adjoint, spk_render_vjp (gpu), against binary64 central differences of the oracle.

The differentiated output is the scanned linear RGB with the grain held as fixed noise: the device's
Poisson counts for the film seed (spkx_session_develop_debug) are fed to the float64 oracle
(orc_render_linear), whose loss is differenced along a direction of the frame and along each parameter
[print_exposure, m_filter_shift, y_filter_shift, halation weights, halation sigmas, and the 48
density-curve parameters: 16 hat functions over each layer's curve table]. The loss is the L2 distance
to a target rendered with perturbed parameters.
"""

import numpy as np
import pytest

from conftest import BASE, sc, setup_f64

import oracle

pytestmark = pytest.mark.gpu

SEED = 7
W, H = 96, 72
STRENGTH = (0.03, 0.03, 0.03)
PARAMS = np.array([1.0, 0.05, -0.04, 0.02, 0.02, 8.0, 40.0])  # pe, m, y, w0, w1, s0, s1
DELTA = dict(BASE, grain_active=True, scanner_lens_blur=1.5)
PITCH = 35000.0 / max(W, H)
TOL = 1e-4  # relative, gradient against the binary64 central difference (the adjoint's accuracy gate)
N_CURVE = 3 * 16


def halation(p):
    return ([((p[3],) * 3, (p[5],) * 3), ((p[4],) * 3, (p[6],) * 3)], STRENGTH)


def delta_of(p):
    return dict(DELTA, print_exposure=float(p[0]), m_filter_shift=float(p[1]), y_filter_shift=float(p[2]))


def oracle_linear(lib, resources, img64, counts, p, pitch=PITCH):
    f64 = setup_f64(lib, resources, delta_of(p), pitch)["f64"]
    o = oracle.Oracle(f64, seed=SEED, halation=halation(p), print_exposure=float(p[0]))
    return o.render_linear(img64, counts)


def make_case(engine, w, h, params):
    """The device's forward output, Poisson counts and adjoint for a w x h frame at the given parameters,
    the loss target rendered with perturbed parameters."""
    img = sc.synthetic_image(w, h, 3)
    with engine.open(img, delta_of(params)) as s:
        s.set_halation(*halation(params))
        _, counts = s.develop_debug("full", SEED, w, h)
        y = s.render_linear(SEED)
        # the target: the same frame with perturbed parameters
        q = params * np.array([1.1, 1.0, 1.0, 1.25, 0.8, 1.1, 0.9]) + np.array([0, 0.02, 0.03, 0, 0, 0, 0])
    with engine.open(img, delta_of(q)) as s2:
        s2.set_halation(*halation(q))
        target = s2.render_linear(SEED).astype(np.float64)
    with engine.open(img, delta_of(params)) as s:
        s.set_halation(*halation(params))
        gy = (y.astype(np.float64) - target).astype(np.float32)
        gx, gp = s.render_vjp(gy, SEED, len(params) + N_CURVE)
    return dict(img=img, counts=counts, y=y, target=target, gx=gx, gp=gp, params=params,
                pitch=35000.0 / max(w, h))


@pytest.fixture(scope="module")
def case(engine):
    return make_case(engine, W, H, PARAMS)


def loss(lib, resources, case, img64, p):
    y = oracle_linear(lib, resources, img64, case["counts"], p, case["pitch"])
    return 0.5 * float(np.sum((y - case["target"]) ** 2))


def test_forward_matches_oracle(lib, resources, case):
    y64 = oracle_linear(lib, resources, case["img"].astype(np.float64), case["counts"], PARAMS)
    err = np.abs(case["y"] - y64) / np.maximum(np.abs(y64), 1e-3)
    assert err.max() < 1e-3, err.max()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_image_gradient(lib, resources, case, seed):
    rng = np.random.default_rng(seed)
    x = case["img"].astype(np.float64)
    v = rng.standard_normal(x.shape) * x
    # the curve tables are piecewise linear: a step small enough that few pixels cross a table node
    eps = 1e-7
    fd = (loss(lib, resources, case, x + eps * v, PARAMS) - loss(lib, resources, case, x - eps * v, PARAMS)) / (2 * eps)
    got = float(np.sum(case["gx"].astype(np.float64) * v))
    assert abs(got - fd) <= TOL * abs(fd), (got, fd)


@pytest.mark.parametrize("j,step", [(0, 1e-4), (1, 1e-4), (2, 1e-4), (3, 1e-5), (4, 1e-5), (5, 1e-3), (6, 1e-2)])
def test_parameter_gradient(lib, resources, case, j, step):
    x = case["img"].astype(np.float64)
    pp, pm = PARAMS.copy(), PARAMS.copy()
    pp[j] += step
    pm[j] -= step
    fd = (loss(lib, resources, case, x, pp) - loss(lib, resources, case, x, pm)) / (2 * step)
    got = float(case["gp"][j])
    assert abs(got - fd) <= TOL * abs(fd) + 1e-9, (j, got, fd)


@pytest.mark.parametrize("c,j", [(0, 4), (1, 7), (2, 10), (0, 12), (2, 2)])
def test_curve_parameter_gradient(lib, resources, case, c, j):
    x = case["img"].astype(np.float64)
    f64 = setup_f64(lib, resources, delta_of(PARAMS), PITCH)["f64"]
    K = len(f64["curve_x"])
    phi = np.maximum(0.0, 1.0 - np.abs(np.arange(K) * 15.0 / (K - 1) - j))
    step = 1e-4

    def loss_at(sign):
        y = np.array(f64["curve_y"], np.float64)
        y[c * K:(c + 1) * K] += sign * step * phi
        o = oracle.Oracle(dict(f64, curve_y=y), seed=SEED, halation=halation(PARAMS), print_exposure=float(PARAMS[0]))
        return 0.5 * float(np.sum((o.render_linear(x, case["counts"]) - case["target"]) ** 2))

    fd = (loss_at(1.0) - loss_at(-1.0)) / (2 * step)
    got = float(case["gp"][len(PARAMS) + 16 * c + j])
    # a node whose hat functions no pixel's lookup reaches has both at 0
    assert abs(got - fd) <= TOL * abs(fd) + 1e-9, (c, j, got, fd)


def test_autograd_function(engine, case):
    import torch

    import spk_torch

    img = torch.from_numpy(case["img"].copy()).requires_grad_(True)
    params = torch.tensor(PARAMS, dtype=torch.float64, requires_grad=True)
    y = spk_torch.render_linear(img, params, engine, DELTA, STRENGTH, SEED)
    loss_t = 0.5 * ((y.double() - torch.from_numpy(case["target"])) ** 2).sum()
    loss_t.backward()
    np.testing.assert_allclose(img.grad.numpy(), case["gx"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(params.grad.numpy(), case["gp"][:len(PARAMS)], rtol=1e-5, atol=1e-9)


# sigma 2 px takes the FIR branch (the derivative of its normalised taps), 12 px the recursive one (the
# tangent of the Young-van Vliet recurrences)
FIR_PARAMS = np.array([1.0, 0.05, -0.04, 0.02, 0.02, 2.0, 12.0])


@pytest.fixture(scope="module")
def case_fir(engine):
    return make_case(engine, W, H, FIR_PARAMS)


@pytest.mark.parametrize("j,step", [(5, 1e-3), (6, 1e-3)])
def test_sigma_gradient_both_branches(lib, resources, case_fir, j, step):
    x = case_fir["img"].astype(np.float64)
    pp, pm = FIR_PARAMS.copy(), FIR_PARAMS.copy()
    pp[j] += step
    pm[j] -= step
    fd = (loss(lib, resources, case_fir, x, pp) - loss(lib, resources, case_fir, x, pm)) / (2 * step)
    got = float(case_fir["gp"][j])
    assert abs(got - fd) <= TOL * abs(fd) + 1e-9, (j, got, fd)


# the differentiation workload's size: 1024 x 1024, grain as fixed noise (seed 7), halation sigma 8 and 40 px
@pytest.fixture(scope="module")
def case_1024(engine):
    return make_case(engine, 1024, 1024, PARAMS)


@pytest.mark.parametrize("window", ["centre", "corner", "frame"])
def test_1024_image_direction(lib, resources, case_1024, window):
    """A random direction of the frame: on a 128 x 128 window (the centre, and a corner where the blurs' edge
    terms act) and over the whole frame. The directional derivative sums 49 K (3.1 M) terms of both signs,
    so the bound is 1e-4 relative plus the per-pixel binary32 accuracy of the adjoint (1e-5) times
    sum |g v|, the most that per-pixel rounding can move the sum."""
    rng = np.random.default_rng(11)
    x = case_1024["img"].astype(np.float64)
    v = rng.standard_normal(x.shape) * x
    if window != "frame":
        mask = np.zeros(x.shape[:2], bool)
        if window == "centre":
            mask[448:576, 448:576] = True
        else:
            mask[:128, -128:] = True
        v *= mask[..., None]
    eps = 1e-7
    fd = (loss(lib, resources, case_1024, x + eps * v, PARAMS) -
          loss(lib, resources, case_1024, x - eps * v, PARAMS)) / (2 * eps)
    terms = case_1024["gx"].astype(np.float64) * v
    got = float(np.sum(terms))
    bound = TOL * abs(fd) + 1e-5 * float(np.abs(terms).sum())
    assert abs(got - fd) <= bound, (got, fd, float(np.abs(terms).sum()))


@pytest.mark.parametrize("j,step", [(0, 1e-4), (3, 1e-5), (5, 1e-3), (6, 1e-2)])
def test_1024_parameter_gradient(lib, resources, case_1024, j, step):
    x = case_1024["img"].astype(np.float64)
    pp, pm = PARAMS.copy(), PARAMS.copy()
    pp[j] += step
    pm[j] -= step
    fd = (loss(lib, resources, case_1024, x, pp) - loss(lib, resources, case_1024, x, pm)) / (2 * step)
    got = float(case_1024["gp"][j])
    assert abs(got - fd) <= TOL * abs(fd) + 1e-9, (j, got, fd)
