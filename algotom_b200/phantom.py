"""Seeded analytic ellipse phantoms and their exact parallel-beam sinograms.

Synthetic input for tests and benchmarks (there is no public dataset on this
path).  The geometry is the one the back-projector inverts
(``algotom/rec/reconstruction.py:165-172``): image pixel (row y, column x) of
an ``n x n`` slice sits at ``X = x - ic``, ``Y = y - ic`` with
``ic = (n - 1) / 2``, and projects at angle ``theta`` onto detector coordinate
``t = X cos(theta) - Y sin(theta) + center``.

An ellipse with centre (X0, Y0), semi-axes (A, B), rotation phi and
attenuation mu has, along the ray at detector offset ``u = t - center``, the
exact chord integral ``mu * 2 A B sqrt(a^2 - (u - u0)^2) / a^2`` with
``u0 = X0 cos(theta) - Y0 sin(theta)`` and
``a^2 = A^2 cos^2(theta + phi) + B^2 sin^2(theta + phi)``.

Attenuation is expressed per field width: a pixel of an ellipse with
attenuation ``mu`` attenuates by ``mu / n``, so a chord through the whole
field integrates to about ``mu``.  This keeps transmitted photon counts well
above zero for 12 overlapping ellipses.

Works on NumPy arrays (small sizes, CPU) and on torch tensors (any device),
chosen by the type of ``angles``.
"""
import math

import numpy as np

N_ELLIPSES = 12


def ellipse_params(seed, size, n_ellipses=N_ELLIPSES, semi_axes=(20.0, 300.0)):
    """Draw ellipse parameters for one slice.

    Centres uniform in the inner 70 % of the field, semi-axes uniform in
    ``semi_axes`` (scaled by ``size / 1024`` below 1024 pixels so that small
    test slices keep the same look), rotations uniform in [0, pi),
    attenuations uniform in [0.1, 1.0].  Returns a float64 array [n, 6] of
    (X0, Y0, A, B, phi, mu) in pixel units.
    """
    rng = np.random.default_rng(seed)
    scale = min(1.0, size / 1024.0)
    lo, hi = semi_axes[0] * scale, semi_axes[1] * scale
    half = 0.35 * size
    p = np.empty((n_ellipses, 6))
    p[:, 0] = rng.uniform(-half, half, n_ellipses)
    p[:, 1] = rng.uniform(-half, half, n_ellipses)
    p[:, 2] = rng.uniform(lo, hi, n_ellipses)
    p[:, 3] = rng.uniform(lo, hi, n_ellipses)
    p[:, 4] = rng.uniform(0.0, math.pi, n_ellipses)
    p[:, 5] = rng.uniform(0.1, 1.0, n_ellipses)
    return p


def phantom_image(params, size):
    """Rasterise the ellipses (pixel-centre test) into a float64 image."""
    ic = 0.5 * (size - 1)
    xs = np.arange(size) - ic
    X, Y = np.meshgrid(xs, xs)
    img = np.zeros((size, size))
    for x0, y0, a, b, phi, mu in params:
        dx, dy = X - x0, Y - y0
        c, s = math.cos(phi), math.sin(phi)
        u = (dx * c + dy * s) / a
        v = (-dx * s + dy * c) / b
        img += np.where(u * u + v * v <= 1.0, mu / size, 0.0)
    return img


def analytic_sinogram(params, angles, ncol, center, size=None):
    """Exact line integrals of the ellipses; [len(angles), ncol].

    ``size`` is the field width used for the attenuation unit (defaults to
    ``ncol``).  ``angles`` may be a NumPy array or a torch tensor; the result
    has the same type (and device), in float64.
    """
    size = ncol if size is None else size
    try:
        import torch
        is_torch = isinstance(angles, torch.Tensor)
    except ImportError:  # pragma: no cover
        is_torch = False
    if is_torch:
        import torch as xp
        th = angles.to(torch.float64)[:, None]
        u = (torch.arange(ncol, dtype=torch.float64, device=angles.device)
             - center)[None, :]
        out = torch.zeros((th.shape[0], ncol), dtype=torch.float64,
                          device=angles.device)
        sqrt, cos, sin, clamp = torch.sqrt, torch.cos, torch.sin, torch.clamp
    else:
        xp = np
        th = np.asarray(angles, dtype=np.float64)[:, None]
        u = (np.arange(ncol, dtype=np.float64) - center)[None, :]
        out = np.zeros((th.shape[0], ncol))
        sqrt, cos, sin = np.sqrt, np.cos, np.sin
        clamp = lambda v, min: np.maximum(v, min)  # noqa: E731
    for x0, y0, a, b, phi, mu in np.asarray(params):
        u0 = x0 * cos(th) - y0 * sin(th)
        a2 = (a * cos(th + phi)) ** 2 + (b * sin(th + phi)) ** 2
        d2 = a2 - (u - u0) ** 2
        chord = 2.0 * a * b * sqrt(clamp(d2, min=0.0)) / a2
        out = out + (mu / size) * chord
    del xp
    return out


def poisson_log(line_integrals, photons, seed):
    """Poisson counts at ``photons`` incident, then -log of the transmission.

    Zero counts are raised to one so the logarithm stays finite.  NumPy in,
    NumPy out (float32); torch in, torch out (float32, same device).
    """
    try:
        import torch
        if isinstance(line_integrals, torch.Tensor):
            g = torch.Generator(device=line_integrals.device)
            g.manual_seed(int(seed))
            lam = photons * torch.exp(-line_integrals)
            counts = torch.poisson(lam, generator=g).clamp_(min=1.0)
            return (-torch.log(counts / photons)).to(torch.float32)
    except ImportError:  # pragma: no cover
        pass
    rng = np.random.default_rng(seed)
    lam = photons * np.exp(-np.asarray(line_integrals))
    counts = np.maximum(rng.poisson(lam), 1.0)
    return (-np.log(counts / photons)).astype(np.float32)


def ellipse_sinogram(seed, nrow, ncol, center, photons=1e4, angles=None,
                     device=None):
    """One noisy -log sinogram of a seeded 12-ellipse phantom.

    Angles default to ``nrow`` values uniform over [0, pi) (endpoint
    excluded).  With ``device`` set, the data is generated with torch on that
    device; otherwise with NumPy.  Returns (sinogram float32, angles float64,
    params).
    """
    params = ellipse_params(seed, ncol)
    if angles is None:
        angles = np.linspace(0.0, math.pi, nrow, endpoint=False)
    if device is not None:
        import torch
        ang_t = torch.as_tensor(np.asarray(angles), dtype=torch.float64,
                                device=device)
        clean = analytic_sinogram(params, ang_t, ncol, center)
        sino = clean if photons is None else poisson_log(clean, photons, seed)
        return sino.to(torch.float32), np.asarray(angles), params
    clean = analytic_sinogram(params, angles, ncol, center)
    sino = clean.astype(np.float32) if photons is None else \
        poisson_log(clean, photons, seed)
    return sino, np.asarray(angles), params


def gaussian_noise_sinogram(seed, nrow, ncol, center, noise=0.01,
                            device=None):
    """Sinogram of a seeded 12-ellipse phantom with additive Gaussian noise.

    The sparse-view model-based reconstruction workload: exact line
    integrals at ``nrow`` angles uniform over [0, pi) (endpoint excluded)
    plus zero-mean Gaussian noise of standard deviation ``noise`` times the
    largest clean value.  With ``device`` set the data is made with torch on
    that device.  Returns (sinogram float32, angles float64, params).
    """
    params = ellipse_params(seed, ncol)
    angles = np.linspace(0.0, math.pi, nrow, endpoint=False)
    if device is not None:
        import torch
        ang_t = torch.as_tensor(angles, dtype=torch.float64, device=device)
        clean = analytic_sinogram(params, ang_t, ncol, center)
        g = torch.Generator(device=clean.device)
        g.manual_seed(int(seed))
        sd = noise * float(clean.max())
        sino = clean + sd * torch.randn(clean.shape, generator=g,
                                        dtype=torch.float64,
                                        device=clean.device)
        return sino.to(torch.float32), angles, params
    clean = analytic_sinogram(params, angles, ncol, center)
    rng = np.random.default_rng(seed)
    sino = clean + noise * clean.max() * rng.standard_normal(clean.shape)
    return sino.astype(np.float32), angles, params


def half_acquisition_sinogram(seed, nrow, ncol, cor, photons=1e4,
                              device=None):
    """A 360-degree half-acquisition scan: ``nrow`` angles uniform over
    [0, 2 pi) (endpoint excluded) on a detector of ``ncol`` pixels whose
    rotation axis sits at column ``cor`` near one edge, so that each view
    covers one side of the object and the opposite view the other.  The
    seeded 12-ellipse object is drawn for the field the views cover
    together (width ``2 max(cor, ncol - 1 - cor) + 1``, the width
    ``extend_sinogram`` restores).  Returns (-log sinogram float32, angles
    float64, params, field width)."""
    field = int(2 * max(cor, ncol - 1 - cor) + 1)
    params = ellipse_params(seed, field)
    angles = np.linspace(0.0, 2.0 * math.pi, nrow, endpoint=False)
    if device is not None:
        import torch
        ang_t = torch.as_tensor(angles, dtype=torch.float64, device=device)
        clean = analytic_sinogram(params, ang_t, ncol, cor, size=field)
        sino = clean if photons is None else poisson_log(clean, photons,
                                                         seed)
        return sino.to(torch.float32), angles, params, field
    clean = analytic_sinogram(params, angles, ncol, cor, size=field)
    sino = clean.astype(np.float32) if photons is None else \
        poisson_log(clean, photons, seed)
    return sino, angles, params, field
