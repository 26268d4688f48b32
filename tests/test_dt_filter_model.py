"""Host model of the third stage's filtered dt fold (fold_dt_filtered / step_end_kernel), on
oracle states: the float estimates stay inside their error bound, and whenever the check passes
the filtered minimum / maximum equal the exact ones over every interior cell.

The kernel evaluates the CFL limit ww1 = dd/sqrt(c^2) and the Mach term ogamma*uu/tt of
src/step.cpp:125-196 exactly only for cells whose float estimates are not clearly beyond
thresholds taken from the previous step's limits; step_end_kernel accepts the result when the
minimum found is <= the threshold (maximum >= its threshold) and otherwise re-evaluates every
cell.  This test restates that decision in numpy (float32 arithmetic, IEEE division where the
kernel uses the 2-ulp __fdividef) and checks it on real trajectories.
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle

EST_BOUND = 2.0 ** -17   # relative error the kernel's comparison margin (2^-12) relies on
MARGIN = 1.0 / 64.0      # default threshold margin


def limits(o, p):
    """Exact FP64 ww1 and Mach term of every interior cell off the top/bottom planes (those
    two planes are folded by the BCON kernel, unfiltered)."""
    s = (slice(2, -2), slice(1, -1), slice(1, -1))
    ru, rv, rw, ro, tt = (o.field(n)[s] for n in ("ru", "rv", "rw", "ro", "tt"))
    ddx, ddy, ddz = o.line("ddx")[1:-1], o.line("ddy")[1:-1], o.line("ddz")[2:-2]
    a, b = ddx[None, None, :], ddy[None, :, None]
    m = np.where(b < a, b, a)
    dd = np.where(ddz[:, None, None] < m, ddz[:, None, None], m)
    r = 1.0 / ro
    uu = (ru * ru + rv * rv + rw * rw) * r * r
    um = (1.0 / p.gamma) * uu / tt
    c2 = uu + p.gamma * tt + 2.0 * np.sqrt(uu * p.gamma * tt)
    w1 = dd / np.sqrt(c2)
    # float32 estimates, in the kernel's operation order
    f = np.float32
    rof, ttf = ro.astype(f), tt.astype(f)
    ruf, rvf, rwf = ru.astype(f), rv.astype(f), rw.astype(f)
    rf = f(1.0) / rof
    uuf = (ruf * ruf + rvf * rvf + rwf * rwf) * rf * rf
    umf = (f(1.0 / p.gamma) * uuf) / ttf
    gtf = f(p.gamma) * ttf
    c2f = uuf + gtf + f(2.0) * np.sqrt(uuf * gtf)
    w1f = dd.astype(f) / np.sqrt(c2f)
    return w1, um, w1f.astype(np.float64), umf.astype(np.float64)


def filtered(w1, um, w1f, umf, t1, tu):
    """Threshold part of the skip rule (the running bounds only ever skip more safely)."""
    skip = (w1f * (1.0 - 2.0 ** -12) > t1) & ((tu > 2.0 ** -40) & (umf * (1.0 + 2.0 ** -12) < tu))
    keep = ~skip
    m1 = w1[keep].min() if keep.any() else 1e300
    mu = um[keep].max() if keep.any() else 0.0
    return m1, mu, int(skip.sum())


@pytest.mark.parametrize("flags,seed", [
    (["--npx", "32", "--npy", "32", "--npz", "64"], 1),
    (["--npx", "24", "--npy", "20", "--npz", "48", "--ngrid", "2", "--izcon", "1", "--itcon", "0"], 5),
])
def test_filter_exact_on_trajectory(flags, seed):
    p = R.parse(flags)
    o = Oracle(flags).init(seed)
    prev = None
    skipped_total = 0
    for step in range(8):
        w1, um, w1f, umf = limits(o, p)
        with np.errstate(divide="ignore", invalid="ignore"):
            assert np.max(np.abs(w1f - w1) / w1) < EST_BOUND
            nz = um > 0
            if nz.any():
                assert np.max(np.abs(umf[nz] - um[nz]) / um[nz]) < EST_BOUND
        if prev is not None:
            t1, tu = prev[0] * (1 + MARGIN), prev[1] * (1 - MARGIN)
            m1, mu, nskip = filtered(w1, um, w1f, umf, t1, tu)
            skipped_total += nskip
            if m1 <= t1 and mu >= tu:        # check passed: the filtered fold is exact
                assert m1 == w1.min() and mu == um.max()
            # a negative margin always fails the check (every step re-evaluates)
            m1b, mub, _ = filtered(w1, um, w1f, umf, prev[0] * 0.5, prev[1] * 1.5)
            assert not (m1b <= prev[0] * 0.5 and mub >= prev[1] * 1.5)
        prev = (w1.min(), um.max())
        o.step(3)
    assert skipped_total > 0  # the filter does skip cells on these trajectories
