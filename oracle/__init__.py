"""Oracle for the FBP/BPF hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` (the
``cpu_baseline`` sample and ``--impl reference``) may import it.  The product
package ``algotom_b200`` never imports anything from here and has no CPU
fallback.

Contents
--------
fbp_oracle
    FP64 NumPy restatement of algotom 1.6.0's padded ramp filter,
    linear-interpolation back-projector and the FBP / BPF drivers
    (``algotom/rec/reconstruction.py:50-684``, ``algotom/util/utility.py``).
cpu_port
    ctypes binding of ``bp_port.c``: a C restatement of
    ``back_projection_cpu`` (``algotom/rec/reconstruction.py:307-359``) with
    the reference's own arithmetic (float32 trig, float64 position, float32
    accumulation), race-free over image rows, used as the timed CPU baseline
    and as a fast FP64 checker for large sizes.

Parity pin: ``tests/golden/*.npz`` were produced by running the reference
itself (``tests/golden/make_golden.py``); ``tests/test_oracle.py`` checks this
oracle against every one of them.
"""
