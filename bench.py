"""Benchmark: stacked FBP at 2560 detector pixels on B200.

Workload (one "step"): FBP of 256 slices, each a seeded 12-ellipse phantom
at 2560 x 2560, sinograms float32 [1801 angles over [0, pi), 256, 2560],
Poisson noise at 5e3 photons then -log, centre 1278.3, hann filter,
ratio 1.0, pad auto (150).  Metric: pixel-angle updates per second
(updates per slice = 2560^2 * 1801), plus slices/s and the relative L2 error
of a sampled slice against the FP64 oracle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs under torchrun, one rank per GPU; each rank reconstructs its own
256 slices (weak scaling, no collective on the data path).  Timing: CUDA
events on the compute stream around K steps, bracketed by a barrier and a
device synchronize, max over ranks.  Inputs (4.7 GB per rank) are larger
than L2.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NSLICE, NROW, NCOL, CENTER = 256, 1801, 2560, 1278.3
PHOTONS = 5e3
METRIC = ("FBP pixel·angle updates/s and slices/s at 2560 det, "
          "rel-L2 err vs FP64 oracle")
WORKLOAD = ("stacked FBP: 256 slices x 1801 angles x 2560 det, float32, "
            "centre 1278.3, hann, ratio 1.0, pad 150")
# algorithmic FP32 work of one update: position FMA, fraction subtract, tap
# difference, interpolation FMA, accumulate add; an FMA counts as 2 FLOP
FLOP_PER_UPDATE = 7.0
# on-chip bytes one update must read: the two FP32 taps of its bin (held as
# one 8-byte interpolation pair in shared memory)
SMEM_BYTES_PER_UPDATE = 8.0
SMEM_BYTES_PER_CLK_PER_SM = 128.0
N_SM = 148


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slices", type=int, default=NSLICE)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="leave the uneven-batch figure out of the default "
                         "line (profiling runs)")
    ap.add_argument("--storage", default="float32",
                    choices=["float32", "float16", "bfloat16"],
                    help="element type of the filtered sinogram (stack)")
    ap.add_argument("--items", type=int, default=64,
                    help="sinograms of the batch workload")
    ap.add_argument("--rows", type=int, default=512,
                    help="detector rows of the vertical workload")
    ap.add_argument("--workload", default="stack",
                    choices=["stack", "batch", "single", "bpf", "volume",
                             "center", "vertical", "vcenter", "halfacq",
                             "dfi", "autograd", "reference_gpu"],
                    help="stack: the 256-slice benchmark (default); bpf: the "
                         "same data through bpf_reconstruction; volume: 2160 "
                         "slices streamed slab by slab with float32 / float16 "
                         "/ bfloat16 filtered storage and errors on 16 sampled "
                         "slices; batch: "
                         "64 uneven sinograms in one persistent launch under "
                         "a CUDA graph; single: one 1024^2 x 900 slice; "
                         "center: centre search over 128 candidates; "
                         "vertical: vertical slices from 1801 projections; "
                         "vcenter: centre search on a vertical slice; "
                         "reference_gpu: algotom's own Numba CUDA path "
                         "(from baseline/_ref) on the same data; "
                         "halfacq: a 360-degree offset-axis slice extended "
                         "and reconstructed; dfi: direct Fourier inversion "
                         "of one slice; autograd: sparse-view model-based "
                         "reconstruction (60 x 2048, 200 iterations, centre "
                         "gradient) through the differentiable "
                         "back-projection")
    return ap.parse_args()


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        # the samples are summarised into the bench line; the raw file goes
        # where BENCH_CLOCKS_DIR says (default: the system temp folder)
        import tempfile
        base = os.environ.get("BENCH_CLOCKS_DIR",
                              os.path.join(tempfile.gettempdir(),
                                           "algotom_b200_bench"))
        self.path = os.path.join(base, "clocks_rank%d.csv" % gpu_index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "samples": len(sm), "reasons": sorted(reasons)}


TRAFFIC_PROFILE = "profiles/backproject_c2_16slices.md"


def _traffic_per_update():
    """DRAM bytes per update of the back-projection kernel as an ncu capture
    measured them: the `dram_bytes_per_update:` line of the committed
    summary TRAFFIC_PROFILE (dram__bytes_read.sum + dram__bytes_write.sum of
    one launch on 16 slices, divided by its updates; the bench cannot read
    DRAM counters itself).  Returns (bytes per update, the summary's
    `build:` line) or (None, None)."""
    try:
        text = open(os.path.join(ROOT, TRAFFIC_PROFILE)).read()
    except OSError:
        return None, None
    m = re.search(r"dram_bytes_per_update:\s*([0-9.eE+-]+)", text)
    b = re.search(r"build:\s*(.+)", text)
    return (float(m.group(1)) if m else None,
            b.group(1).strip() if b else None)


def make_sinograms(nslice, device, seed0=2000):
    """[NROW, nslice, NCOL] float32 on the device; seed = 2*1000 + slice."""
    import torch
    from algotom_b200 import phantom
    out = torch.empty((NROW, nslice, NCOL), dtype=torch.float32, device=device)
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    for k in range(nslice):
        s, _, _ = phantom.ellipse_sinogram(seed0 + k, NROW, NCOL, CENTER,
                                           photons=PHOTONS, angles=ang,
                                           device=device)
        out[:, k, :] = s
    return out, ang


def _algotom():
    """The unmodified reference (algotom) from its pip install under
    baseline/_ref, or None.  Its pywt / h5py imports are unused on the FBP
    path and are stubbed; Numba caches its kernels under the system temp
    folder."""
    import tempfile
    import types
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "algotom")):
        return None
    try:
        for m in ("pywt", "h5py"):
            sys.modules.setdefault(m, types.ModuleType(m))
        os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(
            tempfile.gettempdir(), "algotom_numba_cache"))
        sys.path.insert(0, ref)
        import algotom.rec.reconstruction as rec
        if not os.path.abspath(rec.__file__).startswith(ref):
            return None
        return rec
    except Exception:  # noqa: BLE001
        return None
    finally:
        if sys.path and sys.path[0] == ref:
            sys.path.pop(0)


def _fp64_fbp(sino, ang):
    """FP64 FBP of one benchmark slice (the checker): the oracle's filter
    and its C FP64 back-projector, circle mask, pi/(nrow-1)."""
    from oracle import cpu_port
    from oracle import fbp_oracle as O
    f = O.apply_ramp_filter(sino, None, "hann", 150, "edge")
    ref = cpu_port.back_projection(f.astype(np.float32), ang, CENTER,
                                   ref_arith=False)
    return ref * O.make_circle_mask(NCOL, 1.0) * (np.pi / (NROW - 1))


def cpu_fbp_sample(nslice_max, budget_s, nthreads=None, check=False):
    """CPU FBP of up to ``nslice_max`` benchmark slices (at least one, more
    while the time stays under ``budget_s``) on all host cores.

    The reference itself when its install is present (``kind``
    "reference": ``fbp_reconstruction(gpu=False)``, its Numba back-projector
    parallel over angles, which races on the shared image, and its joblib
    filter); otherwise the oracle's port of its arithmetic (``kind``
    "port": numpy filter + the C back-projector, race-free).  Returns
    (updates/s, slices, seconds, threads, kind, rel L2 of the first slice
    against FP64 or None)."""
    from algotom_b200 import phantom
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    rec = _algotom()
    if rec is not None:
        import numba
        nt = numba.get_num_threads()
        kind = "reference"

        def fbp(s):
            return rec.fbp_reconstruction(s, CENTER, angles=ang, ratio=1.0,
                                          filter_name="hann",
                                          apply_log=False, gpu=False)
        warm = np.ones((16, 64), np.float32)  # compile Numba's kernels
        rec.fbp_reconstruction(warm, 31.5, angles=np.linspace(0, np.pi, 16),
                               apply_log=False, gpu=False)
    else:
        from oracle import cpu_port
        nt = nthreads or cpu_port.max_threads()
        kind = "port"

        def fbp(s):
            return cpu_port.fbp_reconstruction(s[:, None, :], CENTER, ang,
                                               nthreads=nt)[:, 0, :]
        cpu_port.fbp_reconstruction(np.ones((16, 1, 64), np.float32), 31.5,
                                    np.linspace(0, np.pi, 16), nthreads=nt)
    done, t_total, err = 0, 0.0, None
    while done < 1 or (done < nslice_max and t_total < budget_s):
        s, _, _ = phantom.ellipse_sinogram(2000 + done, NROW, NCOL, CENTER,
                                           photons=PHOTONS, angles=ang)
        t0 = time.perf_counter()
        r = fbp(s)
        t_total += time.perf_counter() - t0
        if check and done == 0:
            from oracle import fbp_oracle as O
            err = O.rel_l2(np.asarray(r, np.float64), _fp64_fbp(s, ang))
        done += 1
    ups = done * NCOL * NCOL * NROW / t_total
    return ups, done, t_total, nt, kind, err


def _cpu_sample_text(kind, done, t=None):
    what = ("algotom's own fbp_reconstruction(gpu=False) from baseline/_ref "
            "(Numba back-projector parallel over angles, joblib filter)"
            if kind == "reference" else
            "numpy filter + C back-projection with the reference's "
            "arithmetic (port; the reference install is absent)")
    return "%d of 256 slices (1801 x 2560)%s: %s" % (
        done, "" if t is None else ", %.1f s" % t, what)


def run_reference(args, rank):
    if rank != 0:
        return
    steps, err, kind, nt = [], None, None, 0
    for i in range(args.warmup + args.steps):
        ups, done, t, nt, kind, e = cpu_fbp_sample(1, 0.0, check=(i == 0))
        if e is not None:
            err = e
        if i >= args.warmup:
            steps.append(t)
    t_step = statistics.mean(steps)
    ups = NCOL * NCOL * NROW / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": ups,
        "unit": "updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded ellipse phantoms)",
        "config": {"workload": WORKLOAD, "slices": NSLICE, "nrow": NROW,
                   "ncol": NCOL, "sample": "1 slice per step"},
        "slices_per_s": 1.0 / t_step,
        "accuracy": {"rel_l2_vs_fp64": err, "slices_checked": 1,
                     "note": "all-core run: the reference's back-projector "
                             "races on its shared image"
                             if kind == "reference" else "port, race-free"},
        "cpu_baseline": {"value": ups, "unit": "updates/s", "cores": nt,
                         "kind": kind,
                         "sample": "1 slice per step; " + _cpu_sample_text(
                             kind, 1)},
        "e2e": {"value": ups, "unit": "updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from algotom_b200.rec import reconstruction as R

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nslice = args.slices
    sino, ang = make_sinograms(nslice, dev, seed0=2000 + rank * nslice)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)

    def step(src, out=None):
        return R.fbp_reconstruction(src, CENTER, angles=ang, ratio=1.0,
                                    filter_name="hann", apply_log=False,
                                    out=out, storage=args.storage)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing (value)
    for _ in range(args.warmup):
        rec = step(sino)
        del rec
    clock = ClockSampler(local_rank)
    barrier()
    clock.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        rec = step(sino)
        del rec
    e1.record(stream)
    barrier()
    clocks = clock.stop()
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    upd_step = nslice * NCOL * NCOL * NROW
    value = world * upd_step * args.steps / t_dev

    # ---- per-kernel timing (roofline): filter and back-projection alone
    from algotom_b200.rec import reconstruction as RR
    filt = RR.filter_sinograms(sino, 150, "edge", False, None, "hann",
                               args.storage)
    mask_r2 = RR._mask_r2(1.0, CENTER, NCOL)
    scale = RR._scale(NROW)
    outb = torch.empty((NCOL, nslice, NCOL), dtype=torch.float32, device=dev)
    for _ in range(2):
        RR.backproject(filt, ang, CENTER, False, mask_r2, scale, out=outb)
    nk = max(2, args.steps)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(stream)
    for _ in range(nk):
        RR.backproject(filt, ang, CENTER, False, mask_r2, scale, out=outb)
    ev[1].record(stream)
    ev[2].record(stream)
    for _ in range(nk):
        f2 = RR.filter_sinograms(sino, 150, "edge", False, None, "hann")
        del f2
    ev[3].record(stream)
    torch.cuda.synchronize()
    t_bp = ev[0].elapsed_time(ev[1]) / 1e3 / nk
    t_filt = ev[2].elapsed_time(ev[3]) / 1e3 / nk
    del filt, outb

    # ---- end-to-end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host_in = torch.empty((NROW, nslice, NCOL), dtype=torch.float32,
                              pin_memory=True)
        host_in.copy_(sino)
        host_out = torch.empty((NCOL, nslice, NCOL), dtype=torch.float32,
                               pin_memory=True)
        hin, hout = host_in.numpy(), host_out.numpy()
        del sino
        torch.cuda.empty_cache()
        step(hin, out=hout)
        barrier()
        t0 = time.perf_counter()
        k_e2e = max(1, min(args.steps, 3))
        for _ in range(k_e2e):
            step(hin, out=hout)
        barrier()
        t_e2e = max_over_ranks((time.perf_counter() - t0) / k_e2e)
        e2e = {"value": world * upd_step / t_e2e, "unit": "updates/s",
               "h2d_bytes_per_step": int(host_in.numel() * 4),
               "d2h_bytes_per_step": int(host_out.numel() * 4),
               "ms_per_step": t_e2e * 1e3, "steps": k_e2e}
        rec_sample = torch.from_numpy(hout[:, 0, :].copy())
        sino_sample = host_in[:, 0, :].numpy().copy()
    else:
        rec_sample = step(sino)[:, 0, :].cpu()
        sino_sample = sino[:, 0, :].cpu().numpy()

    if rank != 0:
        return

    # ---- accuracy of slice 0 against the FP64 oracle; CPU baseline
    err = None
    cpu = None
    if not args.no_oracle:
        from oracle import cpu_port
        from oracle import fbp_oracle as O
        f = O.apply_ramp_filter(sino_sample, None, "hann", 150, "edge")
        ref = cpu_port.back_projection(f.astype(np.float32), ang, CENTER,
                                       ref_arith=False)
        ref = ref * O.make_circle_mask(NCOL, 1.0) * (np.pi / (NROW - 1))
        got = rec_sample.numpy()
        err = {"rel_l2": O.rel_l2(got, ref),
               "max_abs": float(np.abs(got - ref).max()),
               "max_rel_to_peak": float(np.abs(got - ref).max()
                                        / np.abs(ref).max()),
               "slices_checked": 1}
        if world == 1:
            ups, done, t, nt, kind, e = cpu_fbp_sample(8, 15.0, check=True)
            cpu = {"value": ups, "unit": "updates/s", "cores": nt,
                   "kind": kind, "rel_l2_vs_fp64": e,
                   "sample": _cpu_sample_text(kind, done, t)}

    # the uneven batch workload (one persistent launch under a CUDA graph):
    # the batched back-projector's own roofline in the same line
    batch = None if args.no_batch else batch_measure(
        64, steps=3, warmup=3, check=not args.no_oracle)

    peaks, src = _peaks()
    f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    fp32_peak = 2.0 * 128 * N_SM * f_clk / 1e12          # TFLOP/s
    smem_peak = SMEM_BYTES_PER_CLK_PER_SM * N_SM * f_clk / 1e9  # GB/s
    bp_upd = nslice * NCOL * NCOL * NROW
    achieved = FLOP_PER_UPDATE * bp_upd / t_bp / 1e12
    smem_achieved = SMEM_BYTES_PER_UPDATE * bp_upd / t_bp / 1e9
    tpu, tbuild = _traffic_per_update()
    filt_bytes = NROW * nslice * NCOL * 8.0
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 12-ellipse phantoms, Poisson 5e3 photons)",
        "config": {"workload": WORKLOAD, "slices_per_gpu": nslice,
                   "nrow": NROW, "ncol": NCOL, "center": CENTER,
                   "storage": args.storage, "kahan": "chunk",
                   "l2": "inputs larger than L2 (4.7 GB sinogram per GPU)"},
        "slices_per_s": world * nslice * args.steps / t_dev,
        "accuracy": err,
        "roofline": {"bound": "smem", "kernel": "bp_kernel",
                     "achieved": smem_achieved, "peak": smem_peak,
                     "unit": "GB/s", "frac": smem_achieved / smem_peak,
                     "traffic": (tpu * bp_upd if tpu else None),
                     "bytes_per_update": SMEM_BYTES_PER_UPDATE,
                     "updates_per_s": bp_upd / t_bp,
                     "ms_per_launch": t_bp * 1e3,
                     "peak_source": "shared-memory delivery, 128 B/clk x 148 "
                                    "SM x sm_max_mhz (%s)" % src,
                     "traffic_source": ("ncu dram__bytes_read.sum + "
                                        "dram__bytes_write.sum per update "
                                        "from %s (%s), times this launch's "
                                        "updates" % (TRAFFIC_PROFILE, tbuild)
                                        if tpu else None)},
        "fp32_roofline": {"bound": "fp32", "achieved": achieved,
                          "peak": fp32_peak, "unit": "TFLOP/s",
                          "frac": achieved / fp32_peak,
                          "flop_per_update": FLOP_PER_UPDATE,
                          "peak_source": "FP32 FMA pipe, 148 SM x 128 lanes "
                                         "x 2 x sm_max_mhz (%s)" % src},
        "filter_roofline": {"bound": "hbm", "kernel": "filter_rows_kernel",
                            "achieved": filt_bytes / t_filt / 1e9,
                            "peak": float(peaks.get("hbm_gbs", 6650.0)),
                            "unit": "GB/s",
                            "frac": filt_bytes / t_filt / 1e9
                            / float(peaks.get("hbm_gbs", 6650.0)),
                            "ms_per_launch": t_filt * 1e3},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "batch": batch,
        "gpu_launches": 2 * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def batch_measure(n_items=64, steps=3, warmup=3, check=True):
    """The uneven batch workload: 64 sinograms (widths 512-4096
    log-uniform, 361-3601 angles over [0, pi); every 8th a 360-degree
    half-acquisition scan, axis 0.3 of the width off centre, widened by the
    device extend_sinogram to ~1.6x with twice the angles), filter +
    persistent back-projection replayed from a captured CUDA graph.
    Returns a dict: replay time, the persistent back-projection alone
    (CUDA events on its stream) and its shared-memory roofline, and the
    FP64-oracle error of the narrowest item."""
    import torch
    from algotom_b200 import _native as nat
    from algotom_b200.rec import batch as B
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    geo = B.uneven_batch_geometry(n_items=n_items)
    sinos = B.batch_sinograms(geo, device=dev)
    bf = B.BatchedFBP([(g["nrow"], g["ncol"]) for g in geo],
                      [g["center"] for g in geo], [g["angles"] for g in geo])
    for x, s in zip(bf.inputs, sinos):
        x.copy_(s)
    bf.capture()
    for _ in range(warmup):
        bf.replay()
    st = torch.cuda.current_stream(dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        bf.replay()
    e1.record(st)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / steps
    b0, b1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    b0.record(st)
    for _ in range(steps):
        nat.call("atb_backproject_batch", bf.items_dev.data_ptr(), bf.n,
                 bf.units_dev.data_ptr(), bf.nunits, bf.counter.data_ptr(), 0,
                 bf.variant, R._stream_ptr(dev))
    b1.record(st)
    torch.cuda.synchronize()
    t_bp = b0.elapsed_time(b1) / 1e3 / steps
    peaks, src = _peaks()
    f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    smem_peak = SMEM_BYTES_PER_CLK_PER_SM * N_SM * f_clk / 1e9
    smem_achieved = SMEM_BYTES_PER_UPDATE * bf.updates / t_bp / 1e9
    err = None
    if check:
        from oracle import fbp_oracle as O
        k = min(range(len(geo)), key=lambda i: geo[i]["ncol"])
        ref = O.fbp_reconstruction(sinos[k].cpu().numpy(), geo[k]["center"],
                                   angles=geo[k]["angles"], apply_log=False)
        single = R.fbp_reconstruction(sinos[k], geo[k]["center"],
                                      angles=geo[k]["angles"],
                                      apply_log=False)
        got = bf.outputs[k].cpu().numpy()
        err = {"rel_l2": O.rel_l2(got, ref),
               "rel_l2_vs_single_slice_path": O.rel_l2(got,
                                                       single.cpu().numpy()),
               "item": k, "ncol": geo[k]["ncol"]}
    half = [g for g in geo if g["half_acquisition"]]
    out = {
        "updates_per_s": bf.updates / t, "ms_per_replay": t * 1e3,
        "items": len(geo), "updates": bf.updates, "tile_variant": bf.variant,
        "units": bf.nunits,
        "widths": [min(g["ncol"] for g in geo), max(g["ncol"] for g in geo)],
        "angles": [min(g["nrow"] for g in geo), max(g["nrow"] for g in geo)],
        "half_acquisition_items": len(half),
        "roofline": {"bound": "smem", "kernel": "bp_batch_kernel",
                     "achieved": smem_achieved, "peak": smem_peak,
                     "unit": "GB/s", "frac": smem_achieved / smem_peak,
                     "bytes_per_update": SMEM_BYTES_PER_UPDATE,
                     "updates_per_s": bf.updates / t_bp,
                     "ms_per_launch": t_bp * 1e3,
                     "peak_source": "shared-memory delivery, 128 B/clk x 148 "
                                    "SM x sm_max_mhz (%s)" % src},
        "gpu_launches_per_replay": len(bf.launch_plan()),
        "accuracy": err}
    del bf, sinos
    torch.cuda.empty_cache()
    return out


def run_batch(args):
    """The uneven batch workload alone (see batch_measure)."""
    r = batch_measure(args.items, args.steps, args.warmup,
                      check=not args.no_oracle)
    print(json.dumps({
        "metric": "batched uneven FBP pixel-angle updates/s",
        "value": r["updates_per_s"], "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["ms_per_replay"], "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "%d uneven sinograms, one persistent launch "
                               "under a CUDA graph" % r["items"],
                   "items": r["items"], "tile_variant": r["tile_variant"],
                   "units": r["units"], "updates": r["updates"],
                   "widths": r["widths"], "angles": r["angles"],
                   "half_acquisition_items": r["half_acquisition_items"]},
        "roofline": r["roofline"],
        "gpu_launches": (r["gpu_launches_per_replay"] + 1) * args.steps,
        "accuracy": r["accuracy"]}), flush=True)


def run_autograd(args):
    """Sparse-view model-based reconstruction through the differentiable
    back-projection: 60 angles over [0, pi) x 2048 detector pixels of a
    seeded 12-ellipse phantom with Gaussian noise of 1 % of max; the centre
    refined from 1021.0 (true 1023.7) through the exact gradient of the
    reprojection objective, then 200 iterations of least squares + TV
    (1e-3).  One step = the whole run.  Updates per image iteration: one
    projection and one back-projection, 2 x 2048^2 x 60."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import autograd as AG
    dev = torch.device("cuda", 0)
    n, nrow, c_true, c0, n_iter = 2048, 60, 1023.7, 1021.0, 200
    sino, ang, params = phantom.gaussian_noise_sinogram(
        4000, nrow, n, c_true, noise=0.01, device=dev)
    st = torch.cuda.current_stream(dev)

    def run():
        c, _ = AG.estimate_center(sino, ang, c0, n_steps=30)
        t1 = torch.cuda.Event(enable_timing=True)
        t1.record(st)
        x, c, hist = AG.iterative_reconstruction(
            sino, ang, c, n_iter=n_iter, tv_weight=1e-3, refine_center=False)
        return x, c, hist, t1

    for _ in range(max(1, args.warmup)):
        run()
    torch.cuda.synchronize()
    t_tot, t_it = [], []
    for _ in range(args.steps):
        e0, e2 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        e0.record(st)
        x, c, hist, e1 = run()
        e2.record(st)
        torch.cuda.synchronize()
        t_tot.append(e0.elapsed_time(e2) / 1e3)
        t_it.append(e1.elapsed_time(e2) / 1e3)
    t = statistics.median(t_tot)
    t_iter = statistics.median(t_it)
    # the projector and the back-projector alone (CUDA events on their stream)
    trig = AG._trig(ang, dev)
    img = x[:, None, :].contiguous()
    res = torch.empty((nrow, 1, n), dtype=torch.float32, device=dev)
    k = 50

    def timed(fn):
        for _ in range(3):
            fn()
        a0, a1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        a0.record(st)
        for _ in range(k):
            fn()
        a1.record(st)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / 1e3 / k
    t_fp = timed(lambda: AG._radon(img, trig, c, nrow, out=res))
    t_bp = timed(lambda: AG._bp(res, trig, c))
    upd = n * n * nrow
    peaks, src = _peaks()
    f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    l1_peak = SMEM_BYTES_PER_CLK_PER_SM * N_SM * f_clk / 1e9
    truth = phantom.phantom_image(params, n)
    xn = x.cpu().numpy()
    err = float(np.linalg.norm(xn - truth) / np.linalg.norm(truth))
    print(json.dumps({
        "metric": "differentiable sparse-view reconstruction: projection + "
                  "back-projection updates/s over the image iterations",
        "value": 2 * upd * n_iter / t_iter, "unit": "updates/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded 12-ellipse phantom, Gaussian noise 1 % "
                "of max)",
        "config": {"workload": "60 angles x 2048 det, centre 1021.0 -> "
                               "1023.7, 200 iterations LS + TV 1e-3",
                   "nrow": nrow, "ncol": n, "iterations": n_iter,
                   "center_steps": 30},
        "ms_per_iteration": t_iter / n_iter * 1e3,
        "ms_center_refinement": (t - t_iter) * 1e3,
        "center": c, "center_error": c - c_true,
        "image_rel_l2_vs_phantom": err,
        "loss_first_last": [hist[0], hist[-1]],
        "projector": {"kernel": "radon_kernel (+ transpose_kernel)",
                      "ms_per_launch": t_fp * 1e3,
                      "updates_per_s": upd / t_fp,
                      "share_of_iteration": t_fp / (t_iter / n_iter),
                      "roofline": {"bound": "l1", "bytes_per_update": 8.0,
                                   "achieved": 8.0 * upd / t_fp / 1e9,
                                   "peak": l1_peak, "unit": "GB/s",
                                   "frac": 8.0 * upd / t_fp / 1e9 / l1_peak,
                                   "peak_source": "L1/shared-memory delivery, "
                                                  "128 B/clk x 148 SM x "
                                                  "sm_max_mhz (%s)" % src}},
        "back_projector": {"kernel": "bp_kernel", "ms_per_launch": t_bp * 1e3,
                           "updates_per_s": upd / t_bp,
                           "share_of_iteration": t_bp / (t_iter / n_iter)},
    }), flush=True)


def run_single(args):
    """One 1024^2 slice from 900 angles (the reference's CPU-sized case)."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    s, ang, _ = phantom.ellipse_sinogram(1000, 900, 1024, 511.5, photons=1e4,
                                         device=dev)
    for _ in range(args.warmup):
        R.fbp_reconstruction(s, 511.5, angles=ang, apply_log=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        R.fbp_reconstruction(s, 511.5, angles=ang, apply_log=False)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    print(json.dumps({
        "metric": "single-slice FBP pixel-angle updates/s",
        "value": 1024 * 1024 * 900 / t, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "1 slice 1024^2 x 900 angles, centre 511.5"}}),
        flush=True)


def run_bpf(args):
    """The stacked benchmark data through bpf_reconstruction (device)."""
    import torch
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    nslice = args.slices
    sino, ang = make_sinograms(nslice, dev)
    torch.cuda.synchronize()

    def step():
        return R.bpf_reconstruction(sino, CENTER, angles=ang, ratio=1.0,
                                    filter_name="hann", apply_log=False)
    for _ in range(args.warmup):
        r = step()
        del r
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = step()
        del r
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    err = None
    if not args.no_oracle:
        from oracle import cpu_port
        from oracle import fbp_oracle as O
        s0 = sino[:, 0, :].cpu().numpy()
        bp = cpu_port.back_projection(s0, ang, CENTER, edge_pad=True,
                                      ref_arith=False)
        ref = O.apply_circular_ramp_filter(bp, None, "hann", 150, "edge")
        ref = ref * O.make_circle_mask(NCOL, 1.0) * (np.pi / (NROW - 1))
        got = step()[:, 0, :].cpu().numpy()
        err = {"rel_l2": O.rel_l2(got, ref), "slices_checked": 1}
    upd = nslice * NCOL * NCOL * NROW
    print(json.dumps({
        "metric": "BPF pixel-angle updates/s at 2560 det",
        "value": upd / t, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "stacked BPF: %d slices x 1801 angles x 2560 "
                               "det, 2-D circular filter on 2860^2" % nslice},
        "slices_per_s": nslice / t, "accuracy": err}), flush=True)


def run_volume(args):
    """Mixed-precision volume: NVOL slices (default 2160) of 1801 x 2560,
    generated and reconstructed slab by slab through HBM with float32,
    float16 and bfloat16 storage of the filtered sinogram (FP32 chunked-Kahan
    accumulation in all three); per-slice relative L2 and max error against
    the FP64 oracle on 16 sampled slices (photons 1e4)."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    nvol = args.slices if args.slices != NSLICE else 2160
    slab = 32
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    modes = ("float32", "float16", "bfloat16")
    sample = sorted(set(np.linspace(0, nvol - 1, 16).astype(int).tolist()))
    kept = {m: {} for m in modes}
    sino_kept = {}
    t_mode = {m: 0.0 for m in modes}
    buf = torch.empty((NROW, slab, NCOL), dtype=torch.float32, device=dev)
    warm = True
    for k0 in range(0, nvol, slab):
        kk = min(slab, nvol - k0)
        for j in range(kk):
            s, _, _ = phantom.ellipse_sinogram(5000 + k0 + j, NROW, NCOL,
                                               CENTER, photons=1e4,
                                               angles=ang, device=dev)
            buf[:, j, :] = s
            if k0 + j in sample:
                sino_kept[k0 + j] = s.cpu().numpy()
        x = buf[:, :kk, :]
        for m in modes:
            if warm:
                R.fbp_reconstruction(x, CENTER, angles=ang, apply_log=False,
                                     storage=m)
            e0, e1 = torch.cuda.Event(enable_timing=True), \
                torch.cuda.Event(enable_timing=True)
            e0.record()
            rec = R.fbp_reconstruction(x, CENTER, angles=ang,
                                       apply_log=False, storage=m)
            e1.record()
            e1.synchronize()
            t_mode[m] += e0.elapsed_time(e1) / 1e3
            for j in range(kk):
                if k0 + j in sample:
                    kept[m][k0 + j] = rec[:, j, :].cpu().numpy()
            del rec
        warm = False
    errs = {m: [] for m in modes}
    if not args.no_oracle:
        from oracle import cpu_port
        from oracle import fbp_oracle as O
        mask = O.make_circle_mask(NCOL, 1.0) * (np.pi / (NROW - 1))
        for k in sample:
            f = O.apply_ramp_filter(sino_kept[k], None, "hann", 150, "edge")
            ref = cpu_port.back_projection(f.astype(np.float32), ang, CENTER,
                                           ref_arith=False) * mask
            for m in modes:
                got = kept[m][k]
                errs[m].append({"slice": int(k),
                                "rel_l2": O.rel_l2(got, ref),
                                "max_abs_rel_to_peak": float(
                                    np.abs(got - ref).max()
                                    / np.abs(ref).max())})
    upd = nvol * NCOL * NCOL * NROW
    out = {"metric": "mixed-precision volume FBP pixel-angle updates/s",
           "unit": "updates/s", "n_gpus": 1, "higher_is_better": True,
           "dtype": "f32 accumulate", "data": "synthetic",
           "config": {"workload": "%d slices x 1801 angles x 2560 det, slabs "
                                  "of %d through HBM" % (nvol, slab),
                      "sampled_slices": sample},
           "modes": {}}
    for m in modes:
        e = errs[m]
        out["modes"][m] = {
            "value": upd / t_mode[m], "seconds": t_mode[m],
            "rel_l2_max": max((x["rel_l2"] for x in e), default=None),
            "rel_l2_median": (float(np.median([x["rel_l2"] for x in e]))
                              if e else None),
            "max_abs_rel_to_peak": max((x["max_abs_rel_to_peak"] for x in e),
                                       default=None),
            "per_slice": e}
    out["value"] = out["modes"]["float32"]["value"]
    print(json.dumps(out), flush=True)


def run_center(args):
    """Centre search on one benchmark slice (1801 angles x 2560 det, centre
    1278.3): the entropy metric of 128 candidate centres at step 0.25
    through ``_find_center_based_slice_metric`` (Gaussian smoothing sigma 2,
    one ramp filter, the candidates back-projected four per CTA -- one
    launch per residue class of centres 1 px apart -- device metrics),
    from a device tensor (``value``) and from a host NumPy array
    (``e2e``); plus the two-pass ``find_center_based_slice_metric`` (coarse
    zoom 0.5, +/-16 px).  CPU baseline: the oracle port's reference-
    arithmetic FBP and the metric on 2 candidates (plus the normalisation
    image); its metrics also check the device ones."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import center as CC
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    s, _, _ = phantom.ellipse_sinogram(2000, NROW, NCOL, CENTER,
                                       photons=PHOTONS, angles=ang)
    s = np.ascontiguousarray(s, dtype=np.float32)
    host = torch.from_numpy(s).pin_memory()
    sdev = host.to(dev)
    ncand, step = 128, 0.25
    start = CENTER - 16.0
    stop = start + (ncand - 0.5) * step
    kw = dict(angles=ang, apply_log=False, sigma=2, metric="entropy",
              return_metric=True)

    def timed(src, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            res = R._find_center_based_slice_metric(src, start, stop, step,
                                                    **kw)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / n, res

    for _ in range(args.warmup):
        timed(sdev, 1)
    sampler = ClockSampler(0)
    sampler.start()
    t_dev, (cs, ms) = timed(sdev, args.steps)
    t_e2e, _ = timed(host.numpy(), args.steps)
    clocks = sampler.stop()
    assert len(cs) == ncand
    upd = ncand * NCOL * NCOL * NROW
    # two-pass search (coarse on the half-size sinogram, fine at 0.25)
    t0 = time.perf_counter()
    found = R.find_center_based_slice_metric(sdev, CENTER - 16, CENTER + 16,
                                             step=0.25, zoom=0.5, angles=ang,
                                             apply_log=False)
    t_find = time.perf_counter() - t0
    cpu = acc = None
    if not args.no_oracle:
        from oracle import center_oracle as CO
        from oracle import cpu_port
        nt = cpu_port.max_threads()
        sm = CC.gaussian_filter_rows(sdev, 2).cpu().numpy()
        picks = [int(np.argmin(ms)), 0]
        t0 = time.perf_counter()
        mean_img = cpu_port.fbp_reconstruction(sm[:, None, :],
                                               float(np.mean(cs)), ang,
                                               nthreads=nt)[:, 0, :]
        nmin, nmax = np.min(mean_img), np.max(mean_img)
        ref = []
        for k in picks:
            img = cpu_port.fbp_reconstruction(sm[:, None, :], float(cs[k]),
                                              ang, nthreads=nt)[:, 0, :]
            ref.append(CO.histogram_entropy(CO.normalise_u8(img, nmin,
                                                            nmax)))
        t_cpu = time.perf_counter() - t0
        cpu = {"value": (len(picks) + 1) * NCOL * NCOL * NROW / t_cpu,
               "unit": "updates/s", "cores": nt, "kind": "port",
               "sample": "%d FBPs of one 1801 x 2560 slice (normalisation "
                         "image + 2 candidates), reference arithmetic, "
                         "%.1f s" % (len(picks) + 1, t_cpu)}
        acc = {"metric_rel_diff_vs_port": max(
            abs(ms[k] - r) / abs(r) for k, r in zip(picks, ref)),
            "candidates_checked": len(picks)}
    print(json.dumps({
        "metric": "centre-search pixel-angle updates/s at 2560 det "
                  "(candidate reconstructions + entropy metric)",
        "value": upd / t_dev, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 12-ellipse phantom, Poisson 5e3)",
        "config": {"workload": "centre search: 128 candidates x 1801 angles "
                               "x 2560^2, step 0.25, entropy, sigma 2",
                   "candidates": ncand},
        "candidates_per_s": ncand / t_dev,
        "e2e": {"value": upd / t_e2e, "unit": "updates/s",
                "h2d_bytes_per_step": int(s.nbytes),
                "d2h_bytes_per_step": 8 * ncand + 8,
                "ms_per_step": t_e2e * 1e3},
        "find_center": {"seconds": t_find, "center": float(found),
                        "true_center": CENTER},
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clocks,
        # per step: Gaussian rows, row filter, normalisation image
        # (batched back-projection + 2 range kernels), candidates (the
        # centre-group back-projections, histogram, entropy)
        "gpu_launches": (7 + _group_launches(CC, cs)) * args.steps}),
        flush=True)


def _group_launches(CC, centers):
    """Back-projection launches of a centre search over ``centers``: per
    residue class, 4-centre CTAs and then the 2- and 1-centre remainder
    (one batched launch when the centres do not form such classes)."""
    groups = CC._centre_groups(centers)
    if groups is None:
        return 1
    n = 0
    for _, _, _, _, cnt in groups:
        rem = cnt % 4
        n += int(cnt >= 4) + int(rem >= 2) + int(rem % 2)
    return n


def _profile_figure(prefix, key):
    """A figure `key: value` from a committed ncu summary under profiles/
    whose name starts with `prefix`."""
    d = os.path.join(ROOT, "profiles")
    try:
        names = sorted(os.listdir(d))
    except OSError:
        return None
    for n in names:
        if n.startswith(prefix) and n.endswith(".md"):
            m = re.search(key + r":\s*([0-9.eE+-]+)",
                          open(os.path.join(d, n)).read())
            if m:
                return float(m.group(1))
    return None


def _vertical_bytes(xs, ys, ang, center, width, height):
    """Algorithmic DRAM bytes of one vertical back-projection launch: per
    angle the detector bins the slice's points touch (a contiguous run, for
    unit-spaced points, plus an edge bin where points are clamped), read
    once for every detector row, and the FP64 accumulator read and written
    (float32-rounded geometry, as the default gpu=True path)."""
    r32 = lambda v: np.float32(v).astype(np.float64)  # noqa: E731
    a = r32(ang)
    p = (r32(xs)[None, :] * np.cos(a)[:, None] +
         r32(ys)[None, :] * np.sin(a)[:, None] + float(np.float32(center)))
    w1 = width - 1
    inr = (p >= 0) & (p <= w1)
    d0 = np.where(inr, np.floor(p), np.inf).min(axis=1)
    d1 = np.where(inr, np.ceil(p), -np.inf).max(axis=1)
    bins = np.where(np.isfinite(d0), d1 - d0 + 1, 0)
    bins = bins + ((p < 0).any(axis=1) & (d0 > 0)) + \
        ((p > w1).any(axis=1) & (d1 < w1))
    return float(bins.sum()) * height * 4 + height * len(xs) * 16.0


def run_vertical(args):
    """Vertical slices from a projection stack of 1801 x 512 x 2560 float32
    (the benchmark's 512 slices read as projections, 9.4 GB, device-
    resident): one vertical slice through the middle at 30 degrees
    (``vertical_reconstruction``, ramp filter after, chunks of 30
    projections) and 64 parallel slices 32 px apart
    (``vertical_reconstruction_multiple``).  The single slice reads every
    projection byte once: its roofline is HBM.  e2e: the single slice from
    a pinned host array (9.4 GB host-to-device per step).  CPU baseline: the
    FP64 oracle's vertical back-projection on 4 detector rows; accuracy: the
    device slice against the FP64 oracle on those rows."""
    import torch
    from algotom_b200.rec import vertrec as VR
    dev = torch.device("cuda", 0)
    height = args.rows
    proj, ang = make_sinograms(height, dev)  # [1801][rows][2560]
    torch.cuda.synchronize()
    kw = dict(angles=ang, apply_log=False, show_progress=False)

    def single(src):
        return VR.vertical_reconstruction(src, NCOL // 2, CENTER, alpha=30.0,
                                          **kw)

    def multi(src):
        return VR.vertical_reconstruction_multiple(src, 256, 256 + 63 * 32,
                                                   CENTER, alpha=30.0,
                                                   step_index=32, **kw)

    def timed(fn, src, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            r = fn(src)
            del r
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / n

    # the back-projection launch alone (atb_vertical_backproject and its
    # angle-group reduction) for the slice of `single`
    xs1, ys1 = VR._get_points_single_line(NCOL // 2, 30.0, NCOL)
    trig1 = VR._trig_plus(ang, dev, True)
    pts1 = VR._points(xs1, ys1, NCOL, dev, True)
    acc1 = torch.zeros((1, height, NCOL), dtype=torch.float64, device=dev)

    def kernel_only(src):
        VR._backproject(src, trig1, pts1, float(np.float32(CENTER)), True,
                        acc1)
        return None

    for _ in range(args.warmup):
        single(proj)
        multi(proj)
        kernel_only(proj)
    sampler = ClockSampler(0)
    sampler.start()
    t1 = timed(single, proj, args.steps)
    t64 = timed(multi, proj, args.steps)
    t_bp = timed(kernel_only, proj, args.steps)
    clocks = sampler.stop()
    alg_bytes = _vertical_bytes(np.asarray(xs1, np.float64),
                                np.asarray(ys1, np.float64), ang, CENTER,
                                NCOL, height)
    per_row = _profile_figure("vertical_slice", "dram_bytes_per_row_single")
    t_e2e = None
    nbytes = proj.numel() * 4
    if not args.no_e2e:
        host = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(proj)
        single(host.numpy())
        t_e2e = timed(single, host.numpy(), max(1, args.steps // 2))
        del host
    upd1 = NROW * height * NCOL
    pk, src = _peaks()
    hbm = float(pk.get("hbm_gbs", 6650.0))
    acc = cpu = None
    if not args.no_oracle:
        from oracle import fbp_oracle as O
        from oracle import vertical_oracle as VO
        rows = sorted({0, height // 5, (3 * height) // 5, height - 1})
        sub = proj[:, rows, :].cpu().numpy()
        xs, ys = VO.points_single_line(NCOL // 2, 30.0, NCOL)
        # the default gpu=True takes float32-rounded angles, points and
        # centre (as the reference's GPU kernel); the oracle gets the same
        r32 = lambda v: np.float32(v).astype(np.float64)  # noqa: E731
        t0 = time.perf_counter()
        bp = VO.vertical_back_projection(sub, r32(ang), r32(xs), r32(ys),
                                         float(np.float32(CENTER)), True)
        t_cpu = time.perf_counter() - t0
        ref = VO.ver_ramp_filter(bp, "hann", 150, "edge") * np.pi / (NROW - 1)
        got = single(proj)[rows].cpu().numpy()
        acc = {"rel_l2_vs_fp64_oracle": O.rel_l2(got, ref),
               "rows_checked": len(rows)}
        cpu = {"value": len(rows) * NROW * NCOL / t_cpu, "unit": "updates/s",
               "cores": 1, "kind": "port",
               "sample": "FP64 NumPy vertical back-projection of %d detector "
                         "rows, %.1f s" % (len(rows), t_cpu)}
    print(json.dumps({
        "metric": "vertical-slice FBP pixel-angle updates/s at 2560 det",
        "value": upd1 / t1, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t1 * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded 12-ellipse phantoms)",
        "config": {"workload": "vertical slice at 30 deg through 1801 "
                               "projections of %d x 2560 (device-resident)"
                               % height,
                   "l2": "inputs larger than L2 (9.4 GB)"},
        "roofline": {"bound": "hbm", "kernel": "vbp_kernel",
                     "achieved": alg_bytes / t_bp / 1e9,
                     "peak": hbm, "unit": "GB/s",
                     "frac": alg_bytes / t_bp / 1e9 / hbm,
                     "traffic": None if per_row is None else per_row * height,
                     "algorithmic_bytes": alg_bytes,
                     "bytes": "detector bins the slice touches (%.2f of the "
                              "projections), read once per row, + the FP64 "
                              "accumulator" % (alg_bytes / nbytes),
                     "ms_per_launch": t_bp * 1e3,
                     "peak_source": src},
        "multiple_64": {"value": 64 * upd1 / t64, "unit": "updates/s",
                        "ms_per_step": t64 * 1e3},
        "e2e": None if t_e2e is None else {
            "value": upd1 / t_e2e, "unit": "updates/s",
            "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": height * NCOL * 8,
            "ms_per_step": t_e2e * 1e3},
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clocks,
        # per step: the single slice (back-projection + angle-group
        # reduction; the FP64 filter after it is library FFT work), the 64
        # slices (one back-projection) and the kernel-only launch pair
        "gpu_launches": 5 * args.steps}), flush=True)


def run_vcenter(args):
    """Centre search on a vertical slice (``find_center_vertical_slice``)
    over a projection stack of 1801 x rows x 2560 float32 (device-resident,
    9.4 GB at 512 rows): Gaussian smoothing (sigma 3) of every projection,
    41 candidate centres 0.5 px apart plus the mean centre as lines of one
    vertical back-projection per chunk slab, FP64 "after" ramp filter,
    entropy of every candidate slice.  The metric counts the pixel-angle
    updates of the candidate slices.  e2e: from a pinned host array.
    Accuracy: the search's metrics against a sequential check -- one
    ``vertical_reconstruction`` per sampled candidate on the smoothed
    projections and the entropy computed on the host with NumPy.  CPU
    baseline: the FP64 oracle's vertical back-projection on 4 rows."""
    import torch
    from algotom_b200 import _native as nat
    from algotom_b200.rec import vertrec as VR
    dev = torch.device("cuda", 0)
    height = args.rows
    proj, ang = make_sinograms(height, dev)  # attenuation [1801][rows][2560]
    torch.cuda.synchronize()
    start, stop, step = CENTER - 10.0, CENTER + 10.0, 0.5
    ncand = len(np.arange(start, stop + step, step))
    kw = dict(angles=ang, apply_log=False, show_progress=False,
              return_metric=True)

    def search(src):
        return VR.find_center_vertical_slice(src, NCOL // 2, start, stop,
                                             step=step, **kw)

    def timed(src, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            r = search(src)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / n, r

    for _ in range(args.warmup):
        search(proj)
    sampler = ClockSampler(0)
    sampler.start()
    t, (cs, ms) = timed(proj, args.steps)
    clocks = sampler.stop()
    nbytes = proj.numel() * 4
    t_e2e = None
    if not args.no_e2e:
        host = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(proj)
        search(host.numpy())
        t_e2e, _ = timed(host.numpy(), max(1, args.steps // 2))
        del host
    upd = ncand * NROW * height * NCOL
    # per slab of chunks: two Gaussian passes, the back-projection (+ the
    # reduction of its angle groups when it splits them); then the entropy
    # histogram and its reduction
    nchunk = -(-NROW // 30)
    nslab = len(VR._slabs([None] * nchunk, 30 * height * NCOL * 4, True,
                          True))
    per_slab = 30 * max(1, (1 << 29) // (30 * height * NCOL * 4))
    split = nat.call("atb_vertical_workspace", min(NROW, per_slab), height,
                     NCOL, ncand + 1) > 0
    launches = nslab * (3 + int(split)) + 2
    acc = cpu = None
    if not args.no_oracle:
        # sequential check: smoothed projections, one reconstruction per
        # sampled candidate, the reference's entropy on the host
        w = torch.from_numpy(VR._gaussian_weights(3)).to(dev)
        sm, tmp = torch.empty_like(proj), torch.empty_like(proj)
        VR._gaussian_slab(proj, w, tmp, sm)
        del tmp
        one = dict(angles=ang, apply_log=False, show_progress=False,
                   pad=min(int(0.15 * NCOL), 150))
        first = VR.vertical_reconstruction(sm, NCOL // 2, np.mean(cs),
                                           **one).cpu().numpy()
        nmin, nmax = first.min(), first.max()
        rad = int(min(np.min(cs), NCOL - np.min(cs)))
        mask = np.zeros(NCOL)
        mask[(NCOL - 2 * rad) // 2:(NCOL - 2 * rad) // 2 + 2 * rad] = 1.0
        errs = []
        for i in (0, ncand // 2, ncand - 1):
            r = VR.vertical_reconstruction(sm, NCOL // 2, cs[i],
                                           **one).cpu().numpy() * mask
            lv = np.uint8(np.clip((r - nmin) / (nmax - nmin), 0, 1) * 255)
            h = 1.0 + np.bincount(lv.ravel(), minlength=256)
            b = np.convolve(h, np.ones(7), mode="valid")
            e = -np.sum(b * np.log2(b))
            errs.append(abs(ms[i] - e) / abs(e))
        del sm
        acc = {"metric_rel_err_vs_sequential": float(max(errs)),
               "candidates_checked": 3}
        from oracle import vertical_oracle as VO
        rows = sorted({0, height // 5, (3 * height) // 5, height - 1})
        sub = proj[:, rows, :].cpu().numpy()
        xs, ys = VO.points_single_line(NCOL // 2, 0.0, NCOL)
        t0 = time.perf_counter()
        VO.vertical_back_projection(sub, ang, xs, ys, CENTER, True)
        t_cpu = time.perf_counter() - t0
        cpu = {"value": len(rows) * NROW * NCOL / t_cpu, "unit": "updates/s",
               "cores": 1, "kind": "port",
               "sample": "FP64 NumPy vertical back-projection of %d detector "
                         "rows for one centre, %.1f s" % (len(rows), t_cpu)}
    pk, src = _peaks()
    print(json.dumps({
        "metric": "vertical centre-search pixel-angle updates/s at 2560 det",
        "value": upd / t, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded 12-ellipse phantoms)",
        "config": {"workload": "find_center_vertical_slice, %d candidates, "
                               "entropy, sigma 3, over 1801 projections of "
                               "%d x 2560 (device-resident)" % (ncand, height),
                   "l2": "inputs larger than L2 (%.1f GB)" % (nbytes / 1e9)},
        "best_center": float(cs[np.argmin(ms)]),
        "roofline": {"bound": "smem", "achieved": upd / t, "unit":
                     "updates/s", "note": "whole search per step; the "
                     "back-projection's own roofline is the vertical "
                     "workload's", "peak_source": src},
        "e2e": None if t_e2e is None else {
            "value": upd / t_e2e, "unit": "updates/s",
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": ncand * 8,
            "ms_per_step": t_e2e * 1e3},
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clocks,
        "gpu_launches": launches * args.steps}), flush=True)


def run_reference_gpu(args):
    """The reference's own GPU path (Numba CUDA), unmodified, imported from a
    pip install of algotom under baseline/_ref (``pip install --target
    baseline/_ref``; not part of this repository): ``back_projection_gpu``
    on one 1024^2 x 900 slice, ``back_projection_gpu_chunk`` and
    ``fbp_reconstruction(gpu=True)`` on the first ``--slices`` (default 16)
    slices of the stacked benchmark.  Host arrays in and out, as its API
    takes them (its kernels copy to and from the device on every call); the
    filter of its fbp_reconstruction runs on the host.  Prints an
    ``unavailable`` line when the install or Numba's CUDA target is
    missing."""
    import types
    ref = os.path.join(ROOT, "baseline", "_ref")
    try:
        for m in ("pywt", "h5py"):  # imported by algotom, unused on this path
            sys.modules.setdefault(m, types.ModuleType(m))
        os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
        sys.path.insert(0, ref)
        from numba import cuda
        if not cuda.is_available():
            raise RuntimeError("Numba's CUDA target is not available")
        import algotom.rec.reconstruction as rec
        if not os.path.abspath(rec.__file__).startswith(ref):
            raise RuntimeError("algotom not found under baseline/_ref")
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference-gpu",
                          "unavailable": "%s: %s" % (type(e).__name__, e)}))
        return
    from algotom_b200 import phantom

    def timed(fn, n):
        fn()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        return (time.perf_counter() - t0) / n

    s1, a1, _ = phantom.ellipse_sinogram(1000, 900, 1024, 511.5, photons=1e4)
    s1 = np.float32(s1)
    u1 = 1024 * 1024 * 900
    t_bp1 = timed(lambda: rec.back_projection_gpu(s1, a1, 511.5),
                  max(1, args.steps))
    t_fbp1 = timed(lambda: rec.fbp_reconstruction(s1, 511.5, angles=a1,
                                                  apply_log=False, gpu=True),
                   max(1, args.steps))
    # the same slice through this build and the FP64 oracle
    from algotom_b200.rec import reconstruction as R
    from oracle import fbp_oracle as O
    ref1 = rec.fbp_reconstruction(s1, 511.5, angles=a1, apply_log=False,
                                  gpu=True)
    ours1 = R.fbp_reconstruction(s1, 511.5, angles=a1, apply_log=False)
    fp64 = O.fbp_reconstruction(s1, 511.5, angles=a1, apply_log=False)
    acc = {"slice": "1024^2 x 900",
           "reference_gpu_vs_fp64_oracle": O.rel_l2(ref1, fp64),
           "this_build_vs_fp64_oracle": O.rel_l2(ours1, fp64),
           "this_build_vs_reference_gpu": O.rel_l2(ours1, ref1)}
    nsl = args.slices if args.slices != NSLICE else 16
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    st = np.empty((NROW, nsl, NCOL), np.float32)
    for k in range(nsl):
        st[:, k, :] = phantom.ellipse_sinogram(2000 + k, NROW, NCOL, CENTER,
                                               photons=PHOTONS,
                                               angles=ang)[0]
    u2 = nsl * NCOL * NCOL * NROW
    t_bp2 = timed(lambda: rec.back_projection_gpu_chunk(st, ang, CENTER), 1)
    t_fbp2 = timed(lambda: rec.fbp_reconstruction(st, CENTER, angles=ang,
                                                  apply_log=False, gpu=True),
                   1)
    print(json.dumps({
        "impl": "reference-gpu",
        "metric": METRIC, "value": u2 / t_fbp2, "unit": "updates/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
        "data": "synthetic (seeded 12-ellipse phantoms)",
        "config": {"workload": "algotom's fbp_reconstruction(gpu=True) on %d "
                               "of the 256 slices (1801 x 2560), host arrays "
                               "in and out" % nsl},
        "seconds": {"fbp_reconstruction_gpu_stack": t_fbp2,
                    "back_projection_gpu_chunk_stack": t_bp2,
                    "fbp_reconstruction_gpu_1024": t_fbp1,
                    "back_projection_gpu_1024": t_bp1},
        "accuracy": acc,
        "updates_per_s": {"fbp_reconstruction_gpu_stack": u2 / t_fbp2,
                          "back_projection_gpu_chunk_stack": u2 / t_bp2,
                          "fbp_reconstruction_gpu_1024": u1 / t_fbp1,
                          "back_projection_gpu_1024": u1 / t_bp1}}),
          flush=True)


def run_halfacq(args):
    """Half-acquisition slice: a 360-degree sinogram of 3601 angles x 2560
    detector pixels whose rotation axis sits at 2300.4 (offset), extended on
    the device (``extend_sinogram``: -log, sub-pixel cubic-spline shift,
    overlap ramp, padding to 2 x 2560 - 518 = 4602 columns) and
    reconstructed by FBP at the returned centre (4602^2 pixels).  ``value``: pixel-angle updates/s of
    extend + FBP from a device-resident transmission sinogram; the extend
    step alone is reported against HBM (4 B read + 6.8 B written per input
    sample).  CPU baseline: the oracle's FP64 extend_sinogram on 64 rows."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.prep import conversion as PC
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    nrow, ncol, cor = 3601, NCOL, 2300.4
    ang = np.linspace(0.0, 2.0 * np.pi, nrow)
    att, _, _ = phantom.ellipse_sinogram(3000, nrow, ncol, cor, photons=None,
                                         angles=ang)
    trans = torch.as_tensor(np.exp(-0.2 * att).astype(np.float32),
                            device=dev)

    def extend():
        return PC.extend_sinogram(trans, cor)

    def step():
        e, c = extend()
        return R.fbp_reconstruction(e, c, angles=ang, apply_log=False)

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), \
            torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            r = fn()
            del r
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / n

    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(0)
    sampler.start()
    t_ext = timed(extend, args.steps)
    t_all = timed(step, args.steps)
    clocks = sampler.stop()
    e, c = extend()
    width = e.shape[1]
    upd = nrow * width * width
    pk, src = _peaks()
    hbm = float(pk.get("hbm_gbs", 6650.0))
    ext_bytes = nrow * ncol * 4 + nrow * width * 4
    acc = cpu = None
    if not args.no_oracle:
        from oracle import conversion_oracle as CO
        from oracle import fbp_oracle as O
        rows = np.arange(0, nrow, nrow // 64)[:64]
        sub = trans[rows].cpu().numpy()
        t0 = time.perf_counter()
        ref, _ = CO.extend_sinogram(sub, cor)
        t_cpu = time.perf_counter() - t0
        acc = {"extend_rel_l2_vs_fp64_oracle": O.rel_l2(e[rows].cpu().numpy(),
                                                         ref),
               "rows_checked": len(rows)}
        cpu = {"value": len(rows) / t_cpu, "unit": "rows/s (extend)",
               "cores": 1, "kind": "port",
               "sample": "FP64 NumPy extend_sinogram of %d rows, %.2f s"
                         % (len(rows), t_cpu)}
    print(json.dumps({
        "metric": "half-acquisition FBP pixel-angle updates/s (extend + FBP)",
        "value": upd / t_all, "unit": "updates/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_all * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 12-ellipse phantom, 360 degrees)",
        "config": {"workload": "360-degree sinogram 3601 x 2560, rotation "
                               "axis 2300.4, extended to %d columns, FBP "
                               "%d^2" % (width, width), "centre": c},
        "extend": {"ms": t_ext * 1e3, "rows_per_s": nrow / t_ext,
                   "roofline": {"bound": "hbm",
                                "achieved": ext_bytes / t_ext / 1e9,
                                "peak": hbm, "unit": "GB/s",
                                "frac": ext_bytes / t_ext / 1e9 / hbm,
                                "peak_source": src}},
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clocks,
        "gpu_launches": 3 * args.steps}), flush=True)


def run_dfi(args):
    """DFI of one benchmark slice (1801 angles x 2560 det, centre 1278.3):
    padded to 2561 + 2 x 640 = 3841 columns, row transform, quintic
    regridding of the 1801 x 3841 polar spectrum onto 3841^2, inverse 2-D
    transform, device-resident input.  ``value``: slices/s.  CPU baseline:
    the same steps through scipy.ndimage's compiled spline routines and
    NumPy's FFT, as the reference calls them (one slice, one core); its
    output is also the accuracy reference."""
    import torch
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as R
    dev = torch.device("cuda", 0)
    ang = np.linspace(0.0, np.pi, NROW, endpoint=False)
    s, _, _ = phantom.ellipse_sinogram(2000, NROW, NCOL, CENTER,
                                       photons=PHOTONS, angles=ang)
    sd = torch.as_tensor(s, device=dev)

    def step():
        return R.dfi_reconstruction(sd, CENTER, apply_log=False)

    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(0)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), \
        torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        r = step()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    acc = cpu = None
    if not args.no_oracle:
        from oracle import dfi_oracle as DO
        from oracle import fbp_oracle as O
        t0 = time.perf_counter()
        ref = DO.dfi_reconstruction_scipy(s, CENTER)
        t_cpu = time.perf_counter() - t0
        acc = {"rel_l2_vs_scipy_port": O.rel_l2(r.cpu().numpy(), ref)}
        cpu = {"value": 1.0 / t_cpu, "unit": "slices/s", "cores": 1,
               "kind": "port",
               "sample": "one 1801 x 2560 slice through scipy.ndimage "
                         "(shift, map_coordinates order 5) and NumPy FFTs, "
                         "%.1f s" % t_cpu}
    print(json.dumps({
        "metric": "DFI slices/s at 2560 det", "value": 1.0 / t,
        "unit": "slices/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded 12-ellipse phantom)",
        "config": {"workload": "DFI of one 1801 x 2560 slice, padded to "
                               "3841, regridded to 3841^2"},
        "cpu_baseline": cpu, "accuracy": acc, "clocks": clocks,
        # centring shift, padded row transform, spline prefilter x 2,
        # regridded inverse (rows, columns)
        "gpu_launches": 6 * args.steps}), flush=True)


def _spawn_ranks(n):
    """Re-run this command as n ranks (one process per GPU) under
    torch.distributed.run on this node; returns its exit code."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(n), "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = _args()
    if args.workload == "dfi":
        run_dfi(args)
        return
    if args.workload == "autograd":
        run_autograd(args)
        return
    if args.workload == "halfacq":
        run_halfacq(args)
        return
    if args.workload == "vertical":
        run_vertical(args)
        return
    if args.workload == "vcenter":
        run_vcenter(args)
        return
    if args.workload == "reference_gpu":
        run_reference_gpu(args)
        return
    if args.workload == "center":
        run_center(args)
        return
    if args.workload == "volume":
        run_volume(args)
        return
    if args.workload == "bpf":
        run_bpf(args)
        return
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "single":
        run_single(args)
        return
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(_spawn_ranks(args.gpus))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit("bench.py: --gpus %d but WORLD_SIZE=%d"
                         % (args.gpus, world))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
