"""Batched FBP of sinograms of uneven width, angle count and centre.

The reference reconstructs one slice (or one chunk of slices sharing a
geometry) per call (``algotom/rec/reconstruction.py:362-493``).  Here a whole
list of single-slice problems -- each with its own width, angles and centre --
is filtered (one ``atb_filter_rows_batch`` launch per FFT length among the
items: at most four for widths 512-6600) and back-projected in ONE
persistent launch (``atb_backproject_batch``): a device counter hands out
(item, 64 x 64 tile) work units, largest angle counts first.  The whole
sequence can be captured once into a CUDA graph and replayed; the persistent
kernel returns its counter to zero, so replays need no reset.

Every item uses the reference's FBP semantics: filter (window, pad, pad
mode), back-projection without edge padding, circle mask and pi/(nrow-1)
scale.
"""
import ctypes

import numpy as np
import torch

from .. import _native as nat
from . import reconstruction as R


def _pow2_at_least(n):
    top = 16
    while top < n:
        top *= 2
    return top


def _group_lengths(needs):
    """Transform lengths of the items' filters in a batch, from each item's
    exact-embedding bound N + ncol - 1: items whose bounds share a power of
    two share one length, the smallest 7-smooth length covering all of them
    (the per-slice filter's own choice, ``atb_filter_length``, is often N
    itself, which differs with every width, and would cost one launch per
    width)."""
    groups = {}
    for need in needs:
        top = _pow2_at_least(need)
        groups[top] = max(groups.get(top, 0), need)
    length = {}
    for top, need in groups.items():
        m = max(16, need)
        while True:
            r = m
            for q in (2, 3, 5, 7):
                while r % q == 0:
                    r //= q
            if r == 1:
                break
            m += 1
        length[top] = m
    return [length[_pow2_at_least(need)] for need in needs]


class BatchedFBP:
    """A fixed batch geometry with device buffers, runnable and capturable.

    Parameters
    ----------
    shapes : list of (nrow, ncol)
    centers : list of float (rounded to float32 like the reference)
    angles : list of 1-D arrays (radians), one per item
    filter_name, pad, pad_mode, ratio : as ``fbp_reconstruction``
    """

    def __init__(self, shapes, centers, angles, filter_name="hann", pad=None,
                 pad_mode="edge", ratio=1.0, device=None, variant=None):
        self.dev = torch.device(device) if device is not None else R._device()
        self.n = len(shapes)
        if not (len(centers) == len(angles) == self.n) or self.n == 0:
            raise ValueError("shapes, centers and angles must have one entry "
                             "per item")
        self.filter_name, self.pad_mode = filter_name, pad_mode
        self.inputs, self.filtered, self.outputs = [], [], []
        self._trig, self._spec, self._pad, self._flen = [], [], [], []
        self._tw = []
        items = (nat.BpItem * self.n)()
        pads = [min(int(0.15 * int(c)), 150) if pad is None else int(pad)
                for _, c in shapes]
        flens = _group_lengths([2 * int(c) + 2 * q - 1
                                for (_, c), q in zip(shapes, pads)])
        for b, ((nrow, ncol), cen, ang) in enumerate(zip(shapes, centers,
                                                         angles)):
            nrow, ncol = int(nrow), int(ncol)
            if len(ang) != nrow:
                raise ValueError("item %d: %d angles for %d rows"
                                 % (b, len(ang), nrow))
            if cen < 0 or cen >= ncol:
                raise ValueError("item %d: Center is out of the range "
                                 "[0, %d]" % (b, ncol - 1))
            p, flen = pads[b], flens[b]
            spec, _ = R._spectrum(None, filter_name, nrow, ncol, p, flen,
                                  self.dev)
            x = torch.zeros((nrow, ncol), dtype=torch.float32,
                            device=self.dev)
            f = torch.empty_like(x)
            o = torch.empty((ncol, ncol), dtype=torch.float32,
                            device=self.dev)
            trig = R._trig(ang, self.dev)
            self.inputs.append(x)
            self.filtered.append(f)
            self.outputs.append(o)
            self._trig.append(trig)
            self._spec.append(spec)
            self._pad.append(p)
            self._flen.append(flen)
            self._tw.append(R._twiddle(flen, self.dev))
            it = items[b]
            it.sino, it.sino_row_stride = f.data_ptr(), f.stride(0)
            it.trig = trig.data_ptr()
            it.out, it.out_row_stride = o.data_ptr(), o.stride(0)
            it.center = float(np.float32(cen))
            it.mask_r2 = R._mask_r2(ratio, float(cen), ncol)
            it.scale = R._scale(nrow)
            it.nrow, it.ncol, it.edge_pad = nrow, ncol, 0
        self.items_host = items
        raw = bytes(items)
        self.items_dev = torch.frombuffer(bytearray(raw), dtype=torch.uint8
                                          ).to(self.dev)
        # one filter launch per transform length: a device table of the
        # items that share it, each with the index of its first row pair
        self._filter_groups = []
        for flen in sorted(set(self._flen)):
            members = [b for b in range(self.n) if self._flen[b] == flen]
            tab = (nat.FilterItem * len(members))()
            off = 0
            for e, b in enumerate(members):
                x, f = self.inputs[b], self.filtered[b]
                it = tab[e]
                it.src, it.src_row_stride = x.data_ptr(), x.stride(0)
                it.dst, it.dst_row_stride = f.data_ptr(), f.stride(0)
                it.spec = self._spec[b].data_ptr()
                it.nrow, it.ncol, it.pad = x.shape[0], x.shape[1], \
                    self._pad[b]
                it.pair_offset = off
                off += (x.shape[0] + 1) // 2
            dev_tab = torch.frombuffer(bytearray(bytes(tab)),
                                       dtype=torch.uint8).to(self.dev)
            self._filter_groups.append((flen, len(members), off, dev_tab,
                                        self._tw[members[0]]))
        self.counter = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.graph = None
        self.updates = int(sum(r * c * c for r, c in shapes))
        self.shapes = [(int(r), int(c)) for r, c in shapes]
        self._units = {}
        if variant is None:
            from .autotune import tuned_batch_variant
            variant = tuned_batch_variant(self)
        self.set_variant(variant)

    def set_variant(self, variant):
        """Select the tile variant (0: 64 x 64, 1: 32 x 32) and its plan."""
        variant = int(variant)
        if variant not in self._units:
            nunits = nat.call("atb_bp_batch_plan",
                              ctypes.addressof(self.items_host), self.n, None,
                              0, variant)
            units = (ctypes.c_int * nunits)()
            nat.call("atb_bp_batch_plan", ctypes.addressof(self.items_host),
                     self.n, ctypes.addressof(units), nunits, variant)
            self._units[variant] = (
                nunits, torch.frombuffer(bytearray(bytes(units)),
                                         dtype=torch.int32).to(self.dev))
        self.variant = variant
        self.nunits, self.units_dev = self._units[variant]
        self.graph = None

    def launch_plan(self):
        """The launches of one :meth:`launch`: one filter launch per
        transform length among the items, then the persistent
        back-projection."""
        return [("atb_filter_rows_batch", flen, n, pairs)
                for flen, n, pairs, _, _ in self._filter_groups] + \
            [("atb_backproject_batch", self.n, self.nunits)]

    def launch(self, max_ctas=0):
        """Filter every item (one launch per transform length), then one
        persistent back-projection launch."""
        st = R._stream_ptr(self.dev)
        for flen, n, pairs, tab, tw in self._filter_groups:
            nat.call("atb_filter_rows_batch", tab.data_ptr(), n, pairs,
                     nat.PAD_MODES[self.pad_mode], 0, tw.data_ptr(), flen,
                     nat.F32, st)
        nat.call("atb_backproject_batch", self.items_dev.data_ptr(), self.n,
                 self.units_dev.data_ptr(), self.nunits,
                 self.counter.data_ptr(), int(max_ctas), self.variant, st)

    def capture(self):
        """Capture :meth:`launch` into a CUDA graph (after one warm launch)."""
        self.launch()
        torch.cuda.synchronize(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def __call__(self, sinograms):
        """Copy the sinograms in, run (graph if captured), return outputs."""
        for x, s in zip(self.inputs, sinograms):
            x.copy_(torch.as_tensor(s), non_blocking=True)
        if self.graph is not None:
            self.graph.replay()
        else:
            self.launch()
        return self.outputs


def uneven_batch_geometry(seed=3000, n_items=64, wmin=512, wmax=4096,
                          amin=361, amax=3601, half_acq_every=8,
                          axis_offset=0.3):
    """Seeded geometry of the uneven batch workload.

    Detector widths log-uniform in [wmin, wmax], angle counts uniform in
    [amin, amax] over [0, pi), centres jittered +/-3 px around the middle.
    Every ``half_acq_every``-th item is a 360-degree half-acquisition scan
    instead: 2 x the angle count over [0, 2 pi) on a detector of the drawn
    width whose rotation axis sits ``axis_offset`` of the width right of
    the detector centre (jittered +/-3 px), to be widened by
    ``extend_sinogram`` (algotom/prep/conversion.py:395-454) before it is
    batched.  An offset of 0.3 of the width gives an overlap of 0.4 of the
    width and an extended width of 1.6 of it (2 ncol - overlap).  Returns a
    list of dicts with nrow, ncol, center, angles, half_acquisition; for
    the half-acquisition items also raw_ncol and raw_center (the detector
    as scanned), and ncol / center are those of the extended sinogram.
    """
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_items):
        w = int(round(np.exp(rng.uniform(np.log(wmin), np.log(wmax)))))
        nrow = int(rng.integers(amin, amax + 1))
        half = half_acq_every and (b % half_acq_every == half_acq_every - 1)
        jitter = rng.uniform(-3.0, 3.0)
        if not half:
            out.append(dict(nrow=nrow, ncol=w, center=(w - 1) / 2.0 + jitter,
                            angles=np.linspace(0.0, np.pi, nrow,
                                               endpoint=False),
                            half_acquisition=False))
            continue
        cor = (w - 1) / 2.0 + axis_offset * w + jitter
        # extend_sinogram's geometry (conversion.py:425-454)
        overlap = 2.0 * (w - cor) - 1.0
        overlap_int = int(np.round(overlap + 1.0e-3))
        nrow360 = 2 * nrow
        out.append(dict(nrow=nrow360, ncol=2 * w - overlap_int,
                        center=w - overlap_int / 2.0 - 0.5,
                        angles=np.linspace(0.0, 2.0 * np.pi, nrow360,
                                           endpoint=False),
                        half_acquisition=True, raw_ncol=w, raw_center=cor))
    return out


def batch_sinograms(geo, seed0=3000, device=None, photons=1e4):
    """Seeded -log sinograms of :func:`uneven_batch_geometry` items on the
    device, ready to batch: ellipse phantoms; half-acquisition items are
    scanned over 360 degrees with the offset axis and widened with the
    device ``extend_sinogram``.  Returns a list of float32 [nrow, ncol]
    tensors."""
    from .. import phantom
    from ..prep.conversion import extend_sinogram
    sinos = []
    for k, g in enumerate(geo):
        if g["half_acquisition"]:
            raw, _, _, _ = phantom.half_acquisition_sinogram(
                seed0 + k, g["nrow"], g["raw_ncol"], g["raw_center"],
                photons=photons, device=device)
            s, cor = extend_sinogram(raw, g["raw_center"], apply_log=False)
            if abs(cor - g["center"]) > 1e-9 or s.shape[1] != g["ncol"]:
                raise RuntimeError("extended geometry differs from the plan")
        else:
            s, _, _ = phantom.ellipse_sinogram(seed0 + k, g["nrow"],
                                               g["ncol"], g["center"],
                                               photons=photons,
                                               angles=g["angles"],
                                               device=device)
        sinos.append(s)
    return sinos
