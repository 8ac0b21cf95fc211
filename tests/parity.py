"""Shared parity rules for the ray-query tests.

The reference rejects a candidate unless t < Max - 1e-5
(Core/Shape/IndexedTriangle.cpp:115), so of two hits closer than 1e-5 the one
visited first wins and the winner depends on the tree. A mismatch between two
implementations is a *near tie* when both answers are valid hits of the
reference's own triangle test whose distances differ by less than that
window; every other mismatch is an error.
"""
from __future__ import annotations

import numpy as np

TIE_WINDOW = 1e-5
# The relative form of the tie rule, |t_a - t_b| < 1e-5 * t: a stricter
# window than the reference's absolute one wherever t < 1.
REL_TIE_WINDOW = 1e-5


def classify(pos, idx, o4, d4, a, b, oracle):
    """Compare two (prim, t, u, v) results. Returns (n_exact, n_tie, bad_indices, bits_ok).

    Rays where both agree must agree bit for bit in t, u and v.
    """
    r = classify_rates(pos, idx, o4, d4, a, b, oracle)
    return r["same_id"], r["near_ties"], r["bad"], r["bits_ok"]


def classify_rates(pos, idx, o4, d4, a, b, oracle):
    """classify() with both tie rules: `near_ties` counts mismatches inside the
    reference's absolute window (both hits valid, |dt| < 1e-5), of which
    `near_ties_relative` also satisfy |dt| < 1e-5 * min(t_a, t_b); `bad`
    lists every other mismatch."""
    pa, ta, ua, va = a
    pb, tb, ub, vb = b
    same = pa == pb
    hit = same & (pa >= 0)
    bits_ok = (np.array_equal(ta[hit].view(np.uint32), tb[hit].view(np.uint32))
               and np.array_equal(ua[hit].view(np.uint32), ub[hit].view(np.uint32))
               and np.array_equal(va[hit].view(np.uint32), vb[hit].view(np.uint32)))
    bad = []
    ties = ties_rel = 0
    for i in np.nonzero(~same)[0]:
        dt = abs(float(ta[i]) - float(tb[i]))
        ok = pa[i] >= 0 and pb[i] >= 0 and dt < TIE_WINDOW
        if ok:
            # both must be genuine hits of the reference's test for this ray
            for p in (pa[i], pb[i]):
                acc, t, _, _ = oracle.shirley(pos, idx.reshape(-1), p, o4[i], d4[i], d4[i, 3])
                ok = ok and acc
        if ok:
            ties += 1
            if dt < REL_TIE_WINDOW * min(float(ta[i]), float(tb[i])):
                ties_rel += 1
        else:
            bad.append(int(i))
    return {"same_id": int(same.sum()), "near_ties": ties, "near_ties_relative": ties_rel, "bad": bad,
            "bits_ok": bits_ok}
