"""Row padding with NumPy's modes on the device.

``np.pad(x, ((0, 0), (pad, pad)), mode)`` for 2-D torch tensors, for the
ten modes the reference passes through (``pad_mode`` of
``algotom/rec/reconstruction.py`` and ``algotom/rec/vertrec.py``): edge,
constant (0), reflect, symmetric and wrap as index maps -- periodic maps
that equal NumPy's repeated reflection for any pad width -- and
linear_ramp (to 0), mean, maximum, minimum and median from whole-row
statistics.
"""
import torch


def pad_rows(x, pad, mode):
    """``np.pad(x, ((0, 0), (pad, pad)), mode)`` of a 2-D floating-point
    tensor on its device, for numpy's ten modes (end / constant values 0,
    statistics over the whole row); the index modes map indices, the others
    write the statistic or ramp.  Same dtype as ``x``."""
    rows, n = x.shape
    if pad == 0:
        return x
    dev = x.device
    i = torch.arange(-pad, n + pad, device=dev)
    if mode in ("edge", "reflect", "symmetric", "wrap"):
        if mode == "edge":
            idx = i.clamp(0, n - 1)
        elif mode == "wrap":
            idx = torch.remainder(i, n)
        elif mode == "symmetric":
            r = torch.remainder(i, 2 * n)
            idx = torch.where(r >= n, 2 * n - 1 - r, r)
        elif n == 1:
            idx = torch.zeros_like(i)
        else:  # reflect: period 2 (n - 1), edges not repeated
            r = torch.remainder(i, 2 * (n - 1))
            idx = torch.where(r >= n, 2 * (n - 1) - r, r)
        return x[:, idx]
    out = torch.empty((rows, n + 2 * pad), dtype=x.dtype, device=dev)
    out[:, pad:pad + n] = x
    if mode == "constant":
        out[:, :pad] = 0.0
        out[:, pad + n:] = 0.0
    elif mode == "linear_ramp":  # from 0 at the ends to the edge samples
        k = torch.arange(pad, device=dev, dtype=x.dtype)
        out[:, :pad] = k[None, :] * (x[:, :1] / pad)
        out[:, pad + n:] = torch.flip(k, [0])[None, :] * (x[:, -1:] / pad)
    elif mode in ("mean", "maximum", "minimum", "median"):
        if mode == "mean":
            v = x.mean(dim=1, keepdim=True)
        elif mode == "maximum":
            v = x.amax(dim=1, keepdim=True)
        elif mode == "minimum":
            v = x.amin(dim=1, keepdim=True)
        else:
            srt = torch.sort(x, dim=1).values
            v = 0.5 * (srt[:, (n - 1) // 2:(n - 1) // 2 + 1] +
                       srt[:, n // 2:n // 2 + 1])
        out[:, :pad] = v
        out[:, pad + n:] = v
    else:
        raise ValueError("pad_mode %r is not supported" % (mode,))
    return out
