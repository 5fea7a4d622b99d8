"""CPU restatement of the photo-ionisation-rate smoothing of
smooth_photoion_rate.c (test infrastructure only: the checker of the CUDA
stencil in argot_b200/csrc/smooth.cu, itself checked against the reference
build in oracle/_ref).

Per cell and rate field (smooth_photoion_rate.c:1060-1517): the 27 cells
ix-1..ix+1 (outer), iy-1..iy+1, iz-1..iz+1 (inner), the centre weighted by
CENTRAL_WEIGHT = 30, summed left to right -- the first 13 terms in single
precision, the weighted centre and everything after it in double (the
double literal promotes the running sum) -- and scaled by 1/56 in double,
stored as float.  The halo on one rank (:142-1057): the periodic image, or
with the reference Makefile's default `isolated = yes` (mpi_rank.c) a copy
of the nearest cell.
"""
from __future__ import annotations

import numpy as np

CENTRAL_WEIGHT = 30.0
NORMAL = 1.0 / (CENTRAL_WEIGHT + 26.0)


def smooth_rates(rates6, edge: int, isolated: bool = True):
    f = np.asarray(rates6, np.float32).reshape(6, edge, edge, edge)
    out = np.empty_like(f)
    for s in range(6):
        g = f[s]
        mode = "edge" if isolated else "wrap"
        p = np.pad(g, 1, mode=mode)
        terms = [p[1 + a:1 + a + edge, 1 + b:1 + b + edge, 1 + c:1 + c + edge]
                 for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
        acc = terms[0].astype(np.float32)
        for t in terms[1:13]:
            acc = (acc + t).astype(np.float32)
        d = acc.astype(np.float64) + CENTRAL_WEIGHT * terms[13].astype(np.float64)
        for t in terms[14:]:
            d = d + t.astype(np.float64)
        out[s] = (NORMAL * d).astype(np.float32)
    return out.reshape(6, -1)
