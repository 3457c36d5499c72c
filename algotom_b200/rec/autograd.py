"""Differentiable back-projection and its adjoint (torch.autograd).

The back-projector B of ``algotom/rec/reconstruction.py:156-190`` is linear
in the sinogram; its adjoint is the forward (Radon) projection with the same
hat weights (``atb_radon_adjoint``).  Both depend on the rotation centre
through the detector position ``p = (x-ic) cos(-a) + (y-ic) sin(-a) + c``,
and ``dp/dc = 1``, so

* d(B s)/dc at a pixel = sum over angles of the slope of the linear
  interpolant of s at p (``atb_backproject`` slope mode), and
* for the projector, dL/dc = <x, B_slope(dL/d(Ax))>.

:class:`BackProjection` and :class:`RadonProjection` wrap these as
``torch.autograd.Function`` so that model-based iterative reconstruction and
centre refinement run on the device.  The centre is kept in float64 here
(the drop-in FBP rounds it to float32 as the reference does); finite
differences in the centre then resolve steps far below a float32 ulp.
"""
import numpy as np
import torch

from .. import _native as nat
from . import reconstruction as R


def _trig(angles, device):
    a = np.asarray(angles, dtype=np.float64)
    tab = np.stack([np.cos(-a), np.sin(-a)], axis=1)
    return torch.from_numpy(np.ascontiguousarray(tab)).to(device)


def _bp(sino3, trig, center, slope=False, mask_r2=-1.0, scale=1.0):
    nrow, nslice, ncol = sino3.shape
    sino3 = sino3.contiguous() if sino3.stride(-1) != 1 else sino3
    out = torch.empty((ncol, nslice, ncol), dtype=torch.float32,
                      device=sino3.device)
    nat.call("atb_backproject", sino3.data_ptr(), nat.F32, sino3.stride(0),
             sino3.stride(1), nrow, nslice, ncol, trig.data_ptr(),
             float(center), 0, float(mask_r2), float(scale), out.data_ptr(),
             out.stride(0), out.stride(1), 2 if slope else 0,
             R._stream_ptr(sino3.device))
    return out


def _radon(img3, trig, center, nrow):
    ncol, nslice, _ = img3.shape
    img3 = img3.contiguous()
    out = torch.empty((nrow, nslice, ncol), dtype=torch.float32,
                      device=img3.device)
    nat.call("atb_radon_adjoint", img3.data_ptr(), img3.stride(0),
             img3.stride(1), nrow, nslice, ncol, trig.data_ptr(),
             float(center), out.data_ptr(), out.stride(0), out.stride(1),
             R._stream_ptr(img3.device))
    return out


def _as3_sino(s):
    return s.unsqueeze(1) if s.dim() == 2 else s


def _as3_img(x):
    return x.unsqueeze(1) if x.dim() == 2 else x


def _from3_img(x3, two_d):
    return x3[:, 0, :] if two_d else x3


def _from3_sino(s3, two_d):
    return s3[:, 0, :] if two_d else s3


class BackProjection(torch.autograd.Function):
    """image = B(sinogram; centre), no edge padding, no mask, no scale.

    ``sino``: float32 CUDA [nrow, ncol] or [nrow, nslice, ncol];
    ``center``: 0-dim float64 tensor (may require grad); ``angles``: radians.
    """

    @staticmethod
    def forward(ctx, sino, center, angles):
        two_d = sino.dim() == 2
        trig = _trig(angles, sino.device)
        c = float(center.detach().cpu())
        out = _bp(_as3_sino(sino.detach()), trig, c)
        ctx.save_for_backward(sino)
        ctx.trig, ctx.c, ctx.two_d = trig, c, two_d
        return _from3_img(out, two_d)

    @staticmethod
    def backward(ctx, g):
        (sino,) = ctx.saved_tensors
        g3 = _as3_img(g.detach().to(torch.float32))
        gs = gc = None
        if ctx.needs_input_grad[0]:
            gs = _from3_sino(_radon(g3, ctx.trig, ctx.c, sino.shape[0]),
                             ctx.two_d)
        if ctx.needs_input_grad[1]:
            slope = _bp(_as3_sino(sino.detach()), ctx.trig, ctx.c, slope=True)
            gc = (slope.double() * g3.double()).sum().reshape(())
        return gs, gc, None


class RadonProjection(torch.autograd.Function):
    """sinogram = B^T(image; centre): the adjoint of :class:`BackProjection`.

    ``img``: float32 CUDA [ncol, ncol] or [ncol, nslice, ncol].
    """

    @staticmethod
    def forward(ctx, img, center, angles):
        two_d = img.dim() == 2
        trig = _trig(angles, img.device)
        c = float(center.detach().cpu())
        nrow = len(angles)
        out = _radon(_as3_img(img.detach()), trig, c, nrow)
        ctx.save_for_backward(img)
        ctx.trig, ctx.c, ctx.two_d = trig, c, two_d
        return _from3_sino(out, two_d)

    @staticmethod
    def backward(ctx, g):
        (img,) = ctx.saved_tensors
        g3 = _as3_sino(g.detach().to(torch.float32))
        gi = gc = None
        if ctx.needs_input_grad[0]:
            gi = _from3_img(_bp(g3, ctx.trig, ctx.c), ctx.two_d)
        if ctx.needs_input_grad[1]:
            slope = _bp(g3, ctx.trig, ctx.c, slope=True)
            gc = (slope.double() * _as3_img(img.detach()).double()).sum() \
                .reshape(())
        return gi, gc, None


def back_projection(sino, center, angles):
    """Differentiable back-projection; ``center`` a float or 0-dim tensor."""
    if not isinstance(center, torch.Tensor):
        center = torch.tensor(float(center), dtype=torch.float64)
    return BackProjection.apply(sino, center, np.asarray(angles, np.float64))


def forward_projection(img, center, angles):
    """Differentiable forward projection (adjoint of back-projection)."""
    if not isinstance(center, torch.Tensor):
        center = torch.tensor(float(center), dtype=torch.float64)
    return RadonProjection.apply(img, center, np.asarray(angles, np.float64))


def total_variation(img, eps=1e-8):
    """Smoothed isotropic total variation of a 2-D image (torch ops)."""
    dx = img[:, 1:] - img[:, :-1]
    dy = img[1:, :] - img[:-1, :]
    return torch.sqrt(dx[:-1, :] ** 2 + dy[:, :-1] ** 2 + eps).sum()


def fbp_differentiable(sino, center, angles, filter_name="hann", pad=None):
    """FBP (no mask) whose output is differentiable in the centre.

    The ramp filter does not depend on the centre, so it runs once without
    autograd (``atb_filter_rows``); the back-projection carries the centre
    gradient.  ``sino``: float32 CUDA [nrow, ncol].
    """
    nrow, ncol = sino.shape
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    f = R.filter_sinograms(sino.detach()[:, None, :], pad, "edge", False,
                           None, filter_name)[:, 0, :]
    return back_projection(f, center, angles) * (np.pi / (nrow - 1))


def estimate_center(sino, angles, center, n_steps=30, step=1.0,
                    filter_name="hann"):
    """Refine the rotation centre by minimising the reprojection error
    ||A_c FBP_c(b) - b||^2 with the exact total derivative in c (through
    both the back-projection and the projector).  Sign search: move by
    ``step`` against the gradient, halve the step whenever its sign flips.
    Returns (centre, history of (centre, loss)).
    """
    ang = np.asarray(angles, np.float64)
    c_val, last, hist = float(center), 0.0, []
    for _ in range(n_steps):
        c = torch.tensor(c_val, dtype=torch.float64, requires_grad=True)
        x = fbp_differentiable(sino, c, ang, filter_name)
        r = forward_projection(x, c, ang) - sino
        loss = (r.double() ** 2).sum()
        (gc,) = torch.autograd.grad(loss, [c])
        hist.append((c_val, float(loss.detach())))
        g = float(gc)
        if g == 0.0:
            break
        sgn = 1.0 if g > 0 else -1.0
        if last and sgn != last:
            step *= 0.5
        c_val -= sgn * step
        last = sgn
    return c_val, hist


def iterative_reconstruction(sino, angles, center, n_iter=200, tv_weight=1e-3,
                             step=None, refine_center=True, center_steps=30,
                             x0=None):
    """Gradient descent on ||A x - b||^2 / 2 + tv_weight TV(x), A = B^T.

    With ``refine_center`` the centre is first refined from ``center`` with
    :func:`estimate_center` (gradient of the reprojection error through the
    differentiable FBP and projector; with the image free, a joint descent
    lets the image absorb a centre error).  The image descent starts from
    zero (or ``x0``) with step 1 / ||A||^2 (power iteration).
    ``sino``: float32 CUDA [nrow, ncol].  Returns (image, centre, loss
    history of the image descent).
    """
    dev = sino.device
    nrow, ncol = sino.shape
    ang = np.asarray(angles, np.float64)
    c = float(center)
    if refine_center:
        c, _ = estimate_center(sino, ang, c, n_steps=center_steps)
    x = (torch.zeros((ncol, ncol), dtype=torch.float32, device=dev)
         if x0 is None else x0.clone()).requires_grad_(True)
    trig = _trig(ang, dev)
    if step is None:
        v = torch.rand((ncol, ncol), device=dev)
        for _ in range(20):
            v = _from3_img(_bp(_radon(_as3_img(v), trig, c, nrow), trig, c),
                           True)
            v = v / v.norm()
        Av = _radon(_as3_img(v), trig, c, nrow)
        step = 1.0 / max(float((Av.double() ** 2).sum()), 1e-12)
    ct = torch.tensor(c, dtype=torch.float64)
    hist = []
    for _ in range(n_iter):
        r = forward_projection(x, ct, ang) - sino
        loss = 0.5 * (r * r).sum() + tv_weight * total_variation(x)
        (gx,) = torch.autograd.grad(loss, [x])
        with torch.no_grad():
            x -= step * gx
        hist.append(float(loss.detach()))
    return x.detach(), c, hist
