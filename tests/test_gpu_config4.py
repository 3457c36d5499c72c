"""Differentiable reconstruction at the sparse-view workload's full size.

60 angles over [0, pi) x 2048 detector pixels of a seeded 12-ellipse
phantom (seed 4000), Gaussian noise of 1 % of the sinogram's maximum, true
centre 1023.7, start 1021.0, 200 iterations of least squares + TV (weight
1e-3).  Checked here:

* the projector (``atb_radon_adjoint``) against the FP64 transpose of the
  reference back-projector (``algotom/rec/reconstruction.py:156-190``,
  restated in the oracle), element by element and through the dot-product
  identity;
* finite differences with step 1e-3 of the sinogram gradient and of three
  centre gradients (back-projection, projection loss, and the
  cross-validated reprojection objective the centre refinement descends),
  to 1e-3;
* the whole run: the refined centre, the falling data misfit and the image
  error.
"""
import numpy as np
import pytest
import scipy.ndimage as ndi
import torch

from algotom_b200 import phantom
from algotom_b200.rec import autograd as AG
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu

N, NROW, SEED = 2048, 60, 4000
C_TRUE, C_START = 1023.7, 1021.0
H = 1e-3      # finite-difference step (sinogram units and pixels)
FD_TOL = 1e-3


@pytest.fixture(scope="module")
def problem(cuda):
    sino, ang, params = phantom.gaussian_noise_sinogram(
        SEED, NROW, N, C_TRUE, noise=0.01, device=cuda)
    return sino, ang, params


def _smooth(seed, shape, sigma=16.0):
    g = np.random.default_rng(seed).standard_normal(shape)
    g = ndi.gaussian_filter(g, sigma)
    return g / np.abs(g).max()


def _disc(n, frac=0.95):
    """1 inside the circle of radius frac * n / 2 about the image centre.
    Pixels outside it are the only ones whose detector position can reach
    an edge bin, where the interpolant ends with a step; an image or weight
    that vanishes there keeps the centre derivative free of those steps
    (which the slope mode spreads over one bin and a difference quotient
    sees only where pixels happen to cross)."""
    ic = 0.5 * (n - 1)
    yy, xx = np.mgrid[0:n, 0:n] - ic
    return (xx * xx + yy * yy <= (frac * 0.5 * n) ** 2).astype(np.float64)


def test_projection_matches_reference_transpose(cuda, problem):
    """Every projected bin against the FP64 transpose of the reference
    back-projector, on a random image."""
    _, ang, _ = problem
    img = np.random.default_rng(2).standard_normal((N, N)).astype(np.float32)
    got = AG.forward_projection(torch.from_numpy(img).to(cuda), C_START, ang)
    ref = O.forward_projection(img, ang, C_START)
    assert O.rel_l2(got.cpu().numpy(), ref) < 2e-6


def test_adjoint_identity_full_size(cuda, problem):
    """<B_ref s, g> = <s, B^T g> with B_ref the FP64 reference
    back-projector, and <B s, g> = <s, B^T g> for this project's pair."""
    sino, ang, _ = problem
    a32 = np.float32(ang).astype(np.float64)
    c32 = float(np.float32(C_START))
    s = sino.cpu().numpy().astype(np.float64)
    g = np.random.default_rng(3).standard_normal((N, N)).astype(np.float32)
    rt = AG.forward_projection(torch.from_numpy(g).to(cuda), c32,
                               a32).double().cpu().numpy()
    rhs = float((rt * s).sum())
    bs_ref = O.back_projection(s, a32, c32, round_inputs=False)
    lhs_ref = float((bs_ref * g).sum())
    scale = float(np.linalg.norm(s) * np.linalg.norm(rt))
    assert abs(lhs_ref - rhs) <= 5e-6 * scale, (lhs_ref, rhs, scale)
    bs = AG.back_projection(sino, c32, a32).double().cpu().numpy()
    lhs = float((bs * g).sum())
    assert abs(lhs - rhs) <= 5e-6 * scale, (lhs, rhs, scale)
    assert O.rel_l2(bs, bs_ref) < 2e-6


def test_sinogram_gradient_fd(cuda, problem):
    """L(s) = ||B s - t||^2 / 2: autograd (the projector) against central
    differences along a smooth direction, step 1e-3."""
    sino, ang, _ = problem
    t = torch.from_numpy(_smooth(5, (N, N)).astype(np.float32)).to(cuda) * \
        float(AG.back_projection(sino, C_START, ang).abs().max())
    v = torch.from_numpy(_smooth(6, (NROW, N), 4.0).astype(np.float32)
                         ).to(cuda)

    def loss(s):
        r = AG.back_projection(s, C_START, ang).double() - t.double()
        return 0.5 * (r * r).sum()

    s = sino.clone().requires_grad_(True)
    (gs,) = torch.autograd.grad(loss(s), [s])
    analytic = float((gs.double() * v.double()).sum())
    with torch.no_grad():
        fd = (float(loss(sino + H * v)) - float(loss(sino - H * v))) / (2 * H)
    assert abs(analytic - fd) <= FD_TOL * abs(fd), (analytic, fd)


def test_center_gradient_backprojection_fd(cuda, problem):
    """d<B_c s, w>/dc (slope mode) against FP64 central differences of the
    reference back-projector, step 1e-3, with s the clean sinogram smoothed
    along the detector (sigma 2 bins) and a smooth weight.  The
    back-projection of a linear interpolant has slope kinks wherever a
    position crosses a bin; the ellipses' sharp edges and white noise put
    enough of them inside the step to move the difference quotient by
    percents, smooth inputs keep them below 1e-3.  The weight vanishes
    outside the inscribed disc (see _disc)."""
    _, ang, params = problem
    s = ndi.gaussian_filter1d(phantom.analytic_sinogram(params, ang, N,
                                                        C_TRUE), 2.0, axis=1
                              ).astype(np.float32)
    w = (_smooth(7, (N, N)) * _disc(N)).astype(np.float32)
    c = torch.tensor(C_START, dtype=torch.float64, requires_grad=True)
    loss = (AG.back_projection(torch.from_numpy(s).to(cuda), c, ang).double()
            * torch.from_numpy(w).to(cuda).double()).sum()
    (gc,) = torch.autograd.grad(loss, [c])

    def L(cv):
        return float((O.back_projection(s, ang, cv, round_inputs=False)
                      * w).sum())
    fd = (L(C_START + H) - L(C_START - H)) / (2 * H)
    assert abs(float(gc) - fd) <= FD_TOL * abs(fd), (float(gc), fd)


def _mean_derivative(fn, c0, h, n=81):
    """Mean of the derivative ``fn(c)`` (autograd) at ``n`` midpoints of
    [c0 - h, c0 + h]: what a central difference with step h measures."""
    cs = c0 - h + (np.arange(n) + 0.5) * (2 * h / n)
    vals = []
    for cv in cs:
        c = torch.tensor(float(cv), dtype=torch.float64, requires_grad=True)
        (g,) = torch.autograd.grad(fn(c), [c])
        vals.append(float(g))
    return float(np.mean(vals)), float(vals[n // 2])


def test_center_gradient_projection_fd(cuda, problem):
    """d||A_c x - b||^2/2 / dc against FP64 central differences (step 1e-3)
    of the reference back-projector's transpose, with x the phantom cut to
    a disc and then smoothed by four pixels (so that it vanishes smoothly
    before any pixel can reach a detector edge) and b the clean sinogram at
    the true centre smoothed along the detector (two bins).

    At 45 and 135 degrees every pixel of a diagonal line x - y = m has the
    same detector position 0.7071 m + c, so whole lines of pixels cross a
    bin together, about four thousand times per pixel of centre; each such
    crossing moves the derivative of the projection, however smooth the
    image.  A step-1e-3 quotient straddles several of them.  So the
    quotient is held to the derivative averaged over the step (which is
    what a difference quotient measures), and, on the other 58 angles, to
    the derivative at the point itself."""
    _, ang, params = problem
    x = ndi.gaussian_filter(phantom.phantom_image(params, N) * _disc(N, 0.92),
                            4.0).astype(np.float32)
    b = ndi.gaussian_filter1d(phantom.analytic_sinogram(params, ang, N,
                                                        C_TRUE), 2.0, axis=1
                              ).astype(np.float32)
    xt = torch.from_numpy(x).to(cuda)
    for sel in (np.arange(NROW), np.setdiff1d(np.arange(NROW), [15, 45])):
        bt = torch.from_numpy(np.ascontiguousarray(b[sel])).to(cuda)

        def loss(c):
            r = AG.forward_projection(xt, c, ang[sel]) - bt
            return 0.5 * (r.double() ** 2).sum()

        def L(cv):
            rr = O.forward_projection(x, ang[sel], cv) - b[sel]
            return float(0.5 * (rr ** 2).sum())
        fd = (L(C_START + H) - L(C_START - H)) / (2 * H)
        mean, point = _mean_derivative(loss, C_START, H)
        assert abs(mean - fd) <= FD_TOL * abs(fd), (len(sel), mean, fd)
        if len(sel) < NROW:
            assert abs(point - fd) <= FD_TOL * abs(fd), (point, fd)


def test_center_objective_gradient_fd(cuda, problem):
    """The objective the centre refinement descends (AG.CenterObjective)
    at the start centre, against its central difference with step 1e-3.

    The objective's derivative is exact but scatters from point to point
    (whole diagonal lines of pixels cross bins together at 45 and 135
    degrees, thousands of times per pixel of centre), so the quotient is
    held to the mean of the derivative at 128 centres placed at random in
    128 equal cells of the step, within three standard errors of that mean
    (plus 1e-3 of the quotient).  The mean over [c0, c0 + 0.25] must point
    towards the true centre."""
    sino, ang, _ = problem
    obj = AG.CenterObjective(sino, ang)
    rng = np.random.default_rng(11)

    def derivatives(lo, hi, n):
        out = []
        for cv in AG._jittered(lo, hi, n, rng):
            c = torch.tensor(float(cv), dtype=torch.float64,
                             requires_grad=True)
            (g,) = torch.autograd.grad(obj(c), [c])
            out.append(float(g))
        return np.array(out)
    with torch.no_grad():
        fd = (float(obj(C_START + H)) - float(obj(C_START - H))) / (2 * H)
    g = derivatives(C_START - H, C_START + H, 128)
    se = g.std(ddof=1) / np.sqrt(len(g))
    assert abs(g.mean() - fd) <= 3 * se + FD_TOL * abs(fd), (g.mean(), se, fd)
    assert derivatives(C_START, C_START + 0.25, 64).mean() < 0.0


def test_sparse_view_reconstruction_200_iterations(cuda, problem):
    """The full workload: centre refined from 1021.0 towards 1023.7 by
    descending the reprojection objective, then 200 iterations of least
    squares + TV (1e-3) on the device."""
    sino, ang, params = problem
    x, c, hist = AG.iterative_reconstruction(sino, ang, C_START, n_iter=200,
                                             tv_weight=1e-3)
    truth = phantom.phantom_image(params, N)
    err = O.rel_l2(x.cpu().numpy(), truth)
    print("centre %.4f  loss %.4e -> %.4e  image rel L2 %.4f"
          % (c, hist[0], hist[-1], err))
    assert abs(c - C_TRUE) < 0.25, c
    assert hist[-1] < 0.05 * hist[0]
    assert all(b <= a * (1 + 1e-6) for a, b in zip(hist, hist[1:]))
    assert err < 0.5
