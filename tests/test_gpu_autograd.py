"""Differentiable back-projection: adjoint identity, finite differences,
and model-based reconstruction with centre refinement (on the device)."""
import numpy as np
import pytest
import torch

from algotom_b200 import phantom
from algotom_b200.rec import autograd as AG
from oracle import fbp_oracle as O

pytestmark = pytest.mark.gpu


def _dot(a, b):
    return float((a.double() * b.double()).sum())


@pytest.mark.parametrize("ncol,nrow,cen", [(96, 60, 47.5), (129, 37, 61.3),
                                           (64, 180, 31.0)])
def test_adjoint_identity_against_reference_backprojector(cuda, ncol, nrow,
                                                          cen):
    """<B_ref s, g> = <s, B^T g> with B_ref the FP64 restatement of the
    reference back-projector and B^T this project's adjoint."""
    rng = np.random.default_rng(ncol + nrow)
    ang = np.concatenate([[0.0, np.pi / 2], rng.uniform(0, np.pi, nrow - 2)])
    s = rng.standard_normal((nrow, ncol))
    g = rng.standard_normal((ncol, ncol))
    lhs = float((O.back_projection(s, np.float32(ang), np.float32(cen)) * g)
                .sum())
    gt = torch.from_numpy(g.astype(np.float32)).cuda()
    rt = AG.forward_projection(gt, float(np.float32(cen)),
                               np.float32(ang).astype(np.float64))
    rhs = float((rt.double().cpu().numpy() * s).sum())
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + np.abs(s).sum() * 1e-3)


@pytest.mark.parametrize("ncol,nrow,cen", [(128, 90, 63.7), (257, 45, 130.2)])
def test_adjoint_identity_device_pair(cuda, ncol, nrow, cen):
    rng = np.random.default_rng(7)
    ang = rng.uniform(0, np.pi, nrow)
    s = torch.from_numpy(rng.standard_normal((nrow, ncol)).astype(np.float32)
                         ).cuda()
    g = torch.from_numpy(rng.standard_normal((ncol, ncol)).astype(np.float32)
                         ).cuda()
    bs = AG.back_projection(s, cen, ang)
    rg = AG.forward_projection(g, cen, ang)
    lhs, rhs = _dot(bs, g), _dot(s, rg)
    assert abs(lhs - rhs) <= 2e-6 * float(bs.double().norm() * g.double().norm())


BLOBS = [(20.0, -10.0, 12.0, 1.0), (-30.0, 25.0, 8.0, 0.7),
         (5.0, 40.0, 15.0, 0.5)]


def _blob_sino(ang, n, center):
    """Exact projections of Gaussian blobs (x0, y0, sigma, amplitude)."""
    u = np.arange(n)[None, :] - center
    s = np.zeros((len(ang), n))
    for x0, y0, sg, amp in BLOBS:
        u0 = x0 * np.cos(ang) - y0 * np.sin(ang)
        s += amp * np.sqrt(2 * np.pi) * sg * np.exp(-(u - u0[:, None]) ** 2
                                                    / (2 * sg * sg))
    return s


def _blob_image(n):
    ic = 0.5 * (n - 1)
    yy, xx = np.mgrid[0:n, 0:n] - ic
    img = np.zeros((n, n))
    for x0, y0, sg, amp in BLOBS:
        img += amp * np.exp(-((xx - x0) ** 2 + (yy - y0) ** 2) / (2 * sg * sg))
    return img


def _smooth_weight(n, seed=1):
    import scipy.ndimage as ndi
    return ndi.gaussian_filter(np.random.default_rng(seed).standard_normal(
        (n, n)), 8) * 50


def test_center_gradient_backprojection_fd(cuda):
    """dL/dc of L = <B_c s, w> against FP64 central differences (step 1e-3)
    of the reference back-projector, for a smooth object and weight (the
    back-projection of a linear interpolant has slope kinks wherever a
    position crosses a bin; smooth inputs keep their effect inside the step
    well below 1e-3 of the derivative)."""
    n, ang = 256, np.linspace(0, np.pi, 60, endpoint=False)
    s = _blob_sino(ang, n, 127.7).astype(np.float32)
    w = _smooth_weight(n).astype(np.float32)
    c = torch.tensor(127.7, dtype=torch.float64, requires_grad=True)
    loss = (AG.back_projection(torch.from_numpy(s).cuda(), c, ang).double()
            * torch.from_numpy(w).cuda().double()).sum()
    (gc,) = torch.autograd.grad(loss, [c])

    def L(cv):
        return float((O.back_projection(s, ang, cv, round_inputs=False)
                      * w).sum())
    h = 1e-3
    fd = (L(127.7 + h) - L(127.7 - h)) / (2 * h)
    assert abs(float(gc) - fd) <= 1e-3 * abs(fd), (float(gc), fd)


def test_center_gradient_projection_fd(cuda):
    """dL/dc of L = ||A_c x - b||^2 / 2 against FP64 central differences of
    the adjoint of the reference back-projector."""
    n = 256
    ang = np.linspace(0, np.pi, 60, endpoint=False)
    x = _blob_image(n).astype(np.float32)
    b = _blob_sino(ang, n, 128.6).astype(np.float32)
    c = torch.tensor(127.4, dtype=torch.float64, requires_grad=True)
    r = AG.forward_projection(torch.from_numpy(x).cuda(), c, ang) - \
        torch.from_numpy(b).cuda()
    loss = 0.5 * (r.double() ** 2).sum()
    (gc,) = torch.autograd.grad(loss, [c])

    def L(cv):
        rr = O.forward_projection(x, ang, cv) - b
        return float(0.5 * (rr ** 2).sum())
    h = 1e-3
    fd = (L(127.4 + h) - L(127.4 - h)) / (2 * h)
    assert abs(float(gc) - fd) <= 1e-3 * abs(fd), (float(gc), fd)


def _slope_model(s, ang, c):
    """NumPy model of the slope mode: per bin d (f = p - d) the derivative
    of the interpolant, plus +s[0] and -s[n-1] edge steps smoothed by a
    one-bin hat."""
    nrow, n = s.shape
    ic = 0.5 * (n - 1)
    xc = np.arange(n) - ic
    out = np.zeros((n, n))
    for i in range(nrow):
        p = xc[None, :] * np.cos(-ang[i]) + xc[:, None] * np.sin(-ang[i]) + c
        d = np.floor(p).astype(int)
        f = p - d
        row = s[i]
        A = np.where((d >= 0) & (d < n - 1),
                     row[np.clip(d + 1, 0, n - 1)] - row[np.clip(d, 0, n - 1)],
                     0.0)
        B = np.zeros_like(p)
        A += np.where(d == 0, row[0], 0)
        B += np.where(d == -1, row[0], 0) - np.where(d == 0, row[0], 0)
        B -= np.where(d == n - 2, row[n - 1], 0)
        A -= np.where(d == n - 1, row[n - 1], 0)
        B += np.where(d == n - 1, row[n - 1], 0)
        out += A + B * f
    return out


@pytest.mark.parametrize("n,cen", [(96, 47.3), (130, 60.9)])
def test_slope_mode_matches_model(cuda, n, cen):
    """Slope mode with non-zero detector edges (the smoothed edge steps)."""
    # smooth rows with non-zero edges: the slope is piecewise constant in p,
    # so FP32 and FP64 positions may pick neighbouring bins; smooth data
    # keeps those neighbours' slopes close
    rng = np.random.default_rng(n)
    ang = rng.uniform(0, np.pi, 40)
    u = np.arange(n)[None, :]
    s = 1.0 + 0.5 * np.sin(0.05 * u + rng.uniform(0, 6, (40, 1)))
    got = AG._bp(torch.from_numpy(s.astype(np.float32)).cuda()[:, None],
                 AG._trig(ang, torch.device("cuda")), cen, slope=True)
    ref = _slope_model(s.astype(np.float32).astype(np.float64), ang, cen)
    assert O.rel_l2(got[:, 0].cpu().numpy(), ref) < 1e-5


def test_sinogram_gradient_is_adjoint(cuda):
    """Autograd of the back-projection w.r.t. the sinogram = projection."""
    rng = np.random.default_rng(2)
    s = torch.from_numpy(rng.standard_normal((40, 80)).astype(np.float32)
                         ).cuda().requires_grad_(True)
    w = torch.from_numpy(rng.standard_normal((80, 80)).astype(np.float32)
                         ).cuda()
    ang = rng.uniform(0, np.pi, 40)
    (AG.back_projection(s, 39.2, ang) * w).sum().backward()
    ref = AG.forward_projection(w, 39.2, ang)
    assert torch.allclose(s.grad, ref, rtol=1e-6, atol=1e-6)


def test_iterative_reconstruction_with_center_refinement(cuda):
    """Sparse-view least squares + TV descent on the device after centre
    refinement through the differentiable FBP: the centre lands near the
    truth and the data misfit drops."""
    n, nrow, c_true = 256, 60, 127.7
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    b = _blob_sino(ang, n, c_true)
    b = b + np.random.default_rng(0).normal(0, 0.01 * b.max(), b.shape)
    bt = torch.from_numpy(b.astype(np.float32)).cuda()
    x, c, hist = AG.iterative_reconstruction(bt, ang, 125.5, n_iter=150,
                                             tv_weight=1e-3)
    assert hist[-1] < 0.05 * hist[0]
    assert abs(c - c_true) < 0.25, c
    truth = _blob_image(n)
    assert O.rel_l2(x.cpu().numpy(), truth) < 0.25



def test_total_variation_matches_tensor_form(cuda):
    """The fused TV value and gradient (atb_tv_value / atb_tv_grad) against
    the same formula as FP64 tensor operations through autograd, with a
    non-unit upstream gradient; odd shapes and a strided view."""
    rng = np.random.default_rng(11)
    for ny, nx in ((257, 130), (1, 9), (5, 1), (64, 64)):
        base = torch.from_numpy(rng.standard_normal((ny, nx + 3))
                                .astype(np.float32)).cuda()
        x = base[:, 1:nx + 1].clone().requires_grad_(True)
        view = base[:, 1:nx + 1]  # strided rows
        x64 = x.detach().double().requires_grad_(True)
        dx = x64[:, 1:] - x64[:, :-1]
        dy = x64[1:, :] - x64[:-1, :]
        ref = torch.sqrt(dx[:-1, :] ** 2 + dy[:, :-1] ** 2 + 1e-8).sum()
        (2.5 * ref).backward()
        got = AG.total_variation(x)
        (2.5 * got).backward()
        assert abs(got.item() - ref.item()) <= 1e-6 * max(1.0, ref.item())
        g_ref = x64.grad.float()
        assert torch.allclose(x.grad, g_ref, rtol=1e-5, atol=1e-5)
        v = AG.total_variation(view)
        assert abs(v.item() - ref.item()) <= 1e-6 * max(1.0, ref.item())
