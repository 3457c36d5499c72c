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


_TRIG_CACHE = {}
_WS_CACHE = {}


def _trig(angles, device):
    """float64 [nrow, 2] (cos(-a), sin(-a)) on ``device``; cached per angle
    set, so that an iteration makes no host-to-device copy."""
    a = np.ascontiguousarray(angles, dtype=np.float64)
    key = (a.tobytes(), str(device))
    tab = _TRIG_CACHE.get(key)
    if tab is None:
        t = np.stack([np.cos(-a), np.sin(-a)], axis=1)
        tab = torch.from_numpy(np.ascontiguousarray(t)).to(device)
        if len(_TRIG_CACHE) > 64:
            _TRIG_CACHE.clear()
        _TRIG_CACHE[key] = tab
    return tab


def _workspace(nbytes, device):
    """Projector scratch, kept per device and grown on demand (calls on one
    device run in stream order, so they can share it)."""
    key = str(device)
    ws = _WS_CACHE.get(key)
    if ws is None or ws.numel() * 4 < nbytes:
        ws = torch.empty((nbytes + 3) // 4, dtype=torch.float32,
                         device=device)
        _WS_CACHE[key] = ws
    return ws


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


def _radon(img3, trig, center, nrow, out=None, workspace=None):
    ncol, nslice, _ = img3.shape
    img3 = img3.contiguous() if img3.stride(-1) != 1 else img3
    if out is None:
        out = torch.empty((nrow, nslice, ncol), dtype=torch.float32,
                          device=img3.device)
    need = nat.call("atb_radon_workspace", nslice, ncol)
    if workspace is None or workspace.numel() * workspace.element_size() \
            < need:
        workspace = _workspace(need, img3.device)
    nat.call("atb_radon_adjoint", img3.data_ptr(), img3.stride(0),
             img3.stride(1), nrow, nslice, ncol, trig.data_ptr(),
             float(center), out.data_ptr(), out.stride(0), out.stride(1),
             workspace.data_ptr(), need, R._stream_ptr(img3.device))
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


class TotalVariation(torch.autograd.Function):
    """Smoothed isotropic total variation of a float32 CUDA [ny, nx] image:
    one launch for the value (``atb_tv_value``, FP64 fixed-order sum), one
    for the gradient (``atb_tv_grad``, scaled on the device by the upstream
    gradient: no host synchronisation)."""

    @staticmethod
    def forward(ctx, img, eps):
        x = img.detach()
        if x.stride(-1) != 1:
            x = x.contiguous()
        ny, nx = x.shape
        dev = x.device
        ws = _tv_workspace(dev)
        out = torch.empty((), dtype=torch.float32, device=dev)
        nat.call("atb_tv_value", x.data_ptr(), x.stride(0), ny, nx,
                 float(eps), ws.data_ptr(), ws.numel() * 8, out.data_ptr(),
                 R._stream_ptr(dev))
        ctx.save_for_backward(x)
        ctx.eps = float(eps)
        return out

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        ny, nx = x.shape
        gs = g.detach().to(device=x.device, dtype=torch.float32).reshape(())
        gx = torch.empty_like(x)
        nat.call("atb_tv_grad", x.data_ptr(), x.stride(0), ny, nx, ctx.eps,
                 gs.data_ptr(), 1.0, gx.data_ptr(), gx.stride(0), 0,
                 R._stream_ptr(x.device))
        return gx, None


_TV_WS = {}


def _tv_workspace(device):
    key = str(device)
    ws = _TV_WS.get(key)
    if ws is None:
        ws = _TV_WS[key] = torch.empty(
            (nat.call("atb_tv_workspace") + 7) // 8, dtype=torch.float64,
            device=device)
    return ws


def total_variation(img, eps=1e-8):
    """Smoothed isotropic total variation of a 2-D float32 CUDA image,
    sum over i < ny-1, j < nx-1 of sqrt(dx^2 + dy^2 + eps) (differentiable;
    :class:`TotalVariation`)."""
    return TotalVariation.apply(img, eps)


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


class CenterObjective:
    """Cross-validated reprojection misfit of a sinogram, as a differentiable
    function of the rotation centre.

    The angles are split into two interleaved folds.  Each fold is
    reconstructed by FBP at centre ``c`` (quadrature weight pi / n for the
    fold's n angles) and projected, at the same centre, onto the other
    fold's angles; the objective is the summed squared misfit of those
    predictions.  A
    centre error shifts every projection by the same amount, which no image
    reproduces across angles that span 180 degrees, so the held-out views
    expose it.  (Reprojecting onto the views an image was built from does
    not: each view largely reproduces itself, and with sparse views that
    self term hides the centre.)

    Linear interpolation makes any such misfit piecewise quadratic in the
    centre, with a ripple of period one pixel (the smoothing of a
    projection depends on the sub-pixel phase of the centre) and dense
    kinks where positions cross bins, in step at lattice angles such as 0
    and 90 degrees.  Three measures keep the trend that leads to the true
    centre:

    * the sinogram is smoothed along the detector with a Gaussian of
      ``sigma`` bins (scipy's ``gaussian_filter1d``, as algotom's own
      centre search does, ``algotom/rec/reconstruction.py:1317-1318``);
    * the misfit is averaged over ``phases`` centres spread evenly over one
      pixel around ``c`` (offsets (k - (phases-1)/2) / phases), which
      cancels the ripple's first ``phases - 1`` harmonics;
    * the filtered fold sinograms are tapered to zero over the ``taper``
      bins next to each detector edge (raised cosine), and the held-out
      misfit is weighted with the same taper: an image pixel whose position
      crosses an edge then meets no step of the interpolant (a step that
      the back-projection's centre derivative could only spread over one
      bin), so the objective is continuous in the centre and its derivative
      has no edge terms.  Nothing is cut from the image, so every held-out
      bin is predicted at every centre (cutting the image to a disc leaves
      unpredicted bins at the detector ends whose share shifts with the
      centre, which moves the minimum).

    The ramp filter does not depend on the centre and runs once per fold;
    the centre enters through the back-projection (slope mode) and the
    projector, so ``torch.autograd`` gives the exact derivative.

    ``sino``: float32 CUDA [nrow, ncol], nrow >= 4, ncol > 4 ``taper``.
    """

    def __init__(self, sino, angles, filter_name="hann", sigma=2.0,
                 pad=None, phases=8, taper=32):
        from .center import gaussian_filter_rows
        ang = np.asarray(angles, np.float64)
        nrow, ncol = sino.shape
        if nrow < 4:
            raise ValueError("the centre objective needs at least 4 angles")
        if pad is None:
            pad = min(int(0.15 * ncol), 150)
        s = sino.detach().to(torch.float32).contiguous()
        if sigma and sigma > 0:
            s = gaussian_filter_rows(s, float(sigma))
        if ncol <= 4 * taper:
            raise ValueError("the centre objective needs ncol > 4 * taper")
        u = torch.arange(ncol, dtype=torch.float64, device=s.device)
        e = torch.minimum(u, ncol - 1 - u) / float(taper)
        win = (0.5 - 0.5 * torch.cos(np.pi * e.clamp(0.0, 1.0))).to(
            torch.float32)
        self.weight = (win * win)[None, :].double()
        self.folds = []
        for idx in (np.arange(0, nrow, 2), np.arange(1, nrow, 2)):
            sf = s[torch.from_numpy(idx).to(s.device)].contiguous()
            f = R.filter_sinograms(sf[:, None, :], pad, "edge", False, None,
                                   filter_name)[:, 0, :] * win
            self.folds.append((sf, f.contiguous(), ang[idx],
                               np.pi / len(idx)))
        self.offsets = [(k - 0.5 * (phases - 1)) / phases
                        for k in range(max(1, int(phases)))]

    def __call__(self, center):
        """Averaged misfit (float64 0-dim tensor) at ``center`` (float or
        0-dim float64 tensor, may require grad)."""
        if not isinstance(center, torch.Tensor):
            center = torch.tensor(float(center), dtype=torch.float64)
        total = 0.0
        for off in self.offsets:
            c = center + off
            for k, (_, f, ang, w) in enumerate(self.folds):
                held, _, ang_h, _ = self.folds[1 - k]
                x = back_projection(f, c, ang) * w
                r = forward_projection(x, c, ang_h) - held
                total = total + (r.double() ** 2 * self.weight).sum()
        return total / len(self.offsets)


def _jittered(lo, hi, n, rng):
    """n points of [lo, hi], one uniformly placed in each of n equal cells."""
    return lo + (np.arange(n) + rng.uniform(0.0, 1.0, n)) * ((hi - lo) / n)


def estimate_center(sino, angles, center, n_steps=30, step=1.0,
                    filter_name="hann", sigma=2.0, phases=8, fit_points=32,
                    fit_halfwidth=1.5, seed=0):
    """Refine the rotation centre from ``center`` with the exact derivative
    of :class:`CenterObjective`.

    First the derivative brackets its zero: steps of ``step`` pixels
    against its sign until the sign flips (at most ``n_steps``).  Then two
    passes fit a line to the derivative sampled at ``fit_points`` centres,
    one placed at random (seeded) in each of as many equal cells, over the
    bracket's middle +/- ``fit_halfwidth`` and then over the first zero
    +/- ``fit_halfwidth`` / 2; the zero of the second line is returned.

    The derivative is exact, but at 45 and 135 degrees whole diagonal lines
    of pixels cross detector bins together, thousands of times per pixel
    of centre, so it scatters widely from point to point about its trend
    (its mean over an interval is the objective's slope there).  The line
    fits average that scatter; random placement keeps a regular grid from
    aliasing with the crossings.  Returns (centre, history of (centre,
    objective, derivative)).
    """
    obj = CenterObjective(sino, angles, filter_name, sigma, phases=phases)
    rng = np.random.default_rng(seed)
    hist = []

    def grad(cv):
        c = torch.tensor(float(cv), dtype=torch.float64, requires_grad=True)
        loss = obj(c)
        (gc,) = torch.autograd.grad(loss, [c])
        hist.append((float(cv), float(loss.detach()), float(gc)))
        return float(gc)

    def line_zero(mid, half):
        cs = _jittered(mid - half, mid + half, fit_points, rng)
        gs = np.array([grad(cv) for cv in cs])
        slope, icpt = np.polyfit(cs - mid, gs, 1)
        if slope <= 0.0:  # no minimum in the window: keep its middle
            return mid
        return float(np.clip(mid - icpt / slope, mid - half, mid + half))

    c_val = float(center)
    g = grad(c_val)
    mid = c_val
    for _ in range(n_steps):
        if g == 0.0:
            break
        c_next = c_val - (step if g > 0 else -step)
        g_next = grad(c_next)
        if (g_next > 0) != (g > 0):
            mid = 0.5 * (c_val + c_next)
            break
        c_val, g, mid = c_next, g_next, c_next
    first = line_zero(mid, fit_halfwidth)
    return line_zero(first, 0.5 * fit_halfwidth), hist


def _descent_step(x, ct, ang, sino, tv_weight, step, loss_out):
    """One gradient step of ||A x - b||^2 / 2 + tv_weight TV(x) on x, in
    place; the loss goes to loss_out (no host synchronisation)."""
    r = forward_projection(x, ct, ang) - sino
    loss = 0.5 * (r * r).sum() + tv_weight * total_variation(x)
    (gx,) = torch.autograd.grad(loss, [x])
    with torch.no_grad():
        x -= step * gx
        loss_out.copy_(loss.detach())


def iterative_reconstruction(sino, angles, center, n_iter=200, tv_weight=1e-3,
                             step=None, refine_center=True, center_steps=30,
                             x0=None):
    """Gradient descent on ||A x - b||^2 / 2 + tv_weight TV(x), A = B^T.

    With ``refine_center`` the centre is first refined from ``center`` with
    :func:`estimate_center` (the exact centre gradient of a cross-validated
    reprojection misfit through the differentiable FBP and projector; a
    joint descent on image and centre barely moves the centre, because with
    far fewer measurements than pixels the image absorbs a centre error).
    The image descent starts from
    zero (or ``x0``) with step 1 / ||A||^2 (power iteration).  (A CUDA
    graph of one descent step replayed 0.71 ms against 0.80 ms eager at
    2048^2 x 60, but its capture and instantiation cost more than the 200
    steps save: 226 against 182 ms per run; the step is kernel-bound, not
    launch-bound.)
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
    hist = torch.empty(n_iter, dtype=torch.float64, device=dev)
    loss_buf = torch.zeros((), dtype=torch.float32, device=dev)
    args = (x, ct, ang, sino, tv_weight, step, loss_buf)
    for k in range(n_iter):
        _descent_step(*args)
        hist[k] = loss_buf
    return x.detach(), c, hist.tolist()
