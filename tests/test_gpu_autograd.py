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


def test_center_gradient_backprojection_fd(cuda):
    """dL/dc of L = <B_c s, w> against central differences, step 1e-3."""
    s, ang, _ = phantom.ellipse_sinogram(5, 60, 256, 127.7, photons=None)
    st = torch.from_numpy(s).cuda()
    w = torch.from_numpy(np.random.default_rng(1).standard_normal(
        (256, 256)).astype(np.float32)).cuda()
    c = torch.tensor(127.7, dtype=torch.float64, requires_grad=True)
    loss = (AG.back_projection(st, c, ang).double() * w.double()).sum()
    (gc,) = torch.autograd.grad(loss, [c])
    h = 1e-3
    lp = _dot(AG.back_projection(st, 127.7 + h, ang), w)
    lm = _dot(AG.back_projection(st, 127.7 - h, ang), w)
    fd = (lp - lm) / (2 * h)
    assert abs(float(gc) - fd) <= 1e-3 * max(abs(fd), 1e-12), (float(gc), fd)


def test_center_gradient_projection_fd(cuda):
    """dL/dc of L = ||A_c x - b||^2 / 2 against central differences."""
    n = 192
    params = phantom.ellipse_params(3, n)
    x = torch.from_numpy(phantom.phantom_image(params, n).astype(np.float32)
                         ).cuda()
    ang = np.linspace(0, np.pi, 60, endpoint=False)
    b = torch.from_numpy(phantom.analytic_sinogram(params, ang, n, 96.3)
                         .astype(np.float32)).cuda()
    c = torch.tensor(95.4, dtype=torch.float64, requires_grad=True)
    r = AG.forward_projection(x, c, ang) - b
    loss = 0.5 * (r.double() ** 2).sum()
    (gc,) = torch.autograd.grad(loss, [c])

    def L(cv):
        rr = AG.forward_projection(x, cv, ang).double() - b.double()
        return float(0.5 * (rr ** 2).sum())
    h = 1e-3
    fd = (L(95.4 + h) - L(95.4 - h)) / (2 * h)
    assert abs(float(gc) - fd) <= 1e-3 * abs(fd), (float(gc), fd)


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
    """Sparse-view least squares + TV descent recovers the image and moves
    the centre toward the truth."""
    n, nrow, c_true = 256, 60, 127.7
    params = phantom.ellipse_params(11, n)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    b = phantom.analytic_sinogram(params, ang, n, c_true)
    b = b + np.random.default_rng(0).normal(0, 0.01 * b.max(), b.shape)
    bt = torch.from_numpy(b.astype(np.float32)).cuda()
    x, c, hist = AG.iterative_reconstruction(bt, ang, 125.5, n_iter=150,
                                             tv_weight=1e-3)
    assert hist[-1] < 0.05 * hist[0]
    assert abs(c - c_true) < 0.25 * abs(125.5 - c_true), c
