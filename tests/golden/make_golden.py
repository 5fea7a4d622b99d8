"""Generates the golden fixtures in this directory by running ARGOT's own C
(the O1 build of oracle/build.py, compiled from the reference sources) on
small seeded inputs.  Run from the repository root:

    python tests/golden/make_golden.py

The fixtures pin the CPU restatement (oracle/argot_oracle.c) and the CUDA
kernels without needing the reference sources at test time.

golden_tables.npz   frequency grid, cross sections, photon rates
golden_march.npz    16^3 lognormal mesh; segments incl. edge cases
                    (axis-aligned, corner-crossing, same cell, zero
                    length, start outside, end on the box face) -> columns
golden_path.npz     16^3 mesh, 6 sources: the reference's light rays for
                    every cell (target, source position, spectrum sum,
                    columns) and per-cell rates (one thread)
golden_path_ragged.npz
                    the same on a ragged 19^3 mesh (no axis a multiple of
                    the 2x4x4 target blocks), 7 sources, opening angle 0.6
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from argot_b200 import workload as W  # noqa: E402
from oracle.oracle import RefLib  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def edge_case_segments(edge: int, rng) -> np.ndarray:
    d = 1.0 / edge
    c = lambda i: (i + 0.5) * d  # noqa: E731
    segs = [
        [c(0), c(3), c(5), c(12), c(3), c(5)],             # +x axis-aligned
        [c(12), c(3), c(5), c(0), c(3), c(5)],             # -x axis-aligned
        [c(4), c(9), c(2), c(4), c(9), c(14)],             # +z axis-aligned
        [c(4), c(15), c(2), c(4), c(1), c(2)],             # -y axis-aligned
        [c(1), c(1), c(1), c(14), c(14), c(14)],           # main diagonal: corner crossings
        [c(14), c(1), c(14), c(1), c(14), c(1)],           # anti-diagonal
        [c(2), c(2), c(7), c(12), c(12), c(7)],            # xy diagonal (edge crossings)
        [c(5) + 0.1 * d, c(5), c(5), c(5) - 0.2 * d, c(5), c(5)],  # same cell
        [c(6), c(6), c(6), c(6), c(6), c(6)],              # zero length
        [5 * d, c(7), c(7), c(11), c(2), c(9)],            # start on a face
        [0.0, 0.3, 0.7, c(8), c(8), c(8)],                 # start on the box face
        [-0.05, 0.5, 0.5, c(10), c(7), c(7)],              # start outside (clamped)
        [c(3), c(3), c(3), 1.0, c(3), c(3)],               # end on the upper face
        [c(0), c(0), c(0), c(15), c(15), c(15)],           # corner to corner
    ]
    rnd = []
    for _ in range(2000):
        a = rng.uniform(0.0, 1.0, 3)
        b = (rng.integers(0, edge, 3) + 0.5) * d
        rnd.append([*a, *b])
    return np.asarray(segs + rnd, np.float32)


def path_fixture(R, wl, edge, name):
    R.set_sources(wl.src_type, wl.src_param, wl.src_pos, wl.src_rate)
    R.zero_rates()
    out = R.run_range(0, edge ** 3, True, want=("tgt", "src", "seg", "tau", "spec_sum"))
    rates = R.get_rates()
    np.savez_compressed(os.path.join(OUT, name), edge=edge, dens=wl.dens, fHI=wl.fHI,
                        fHeI=wl.fHeI, fHeII=wl.fHeII, src_pos=wl.src_pos, src_rate=wl.src_rate,
                        src_type=wl.src_type, src_param=wl.src_param, theta=wl.theta,
                        lunit=wl.lunit, denstonh=wl.denstonh, tgt=out["tgt"], src=out["src"],
                        seg=out["seg"], tau=out["tau"], spec_sum=out["spec_sum"], rates=rates)


def main():
    rng = np.random.default_rng(20261203)
    edge = 16
    R = RefLib(edge)

    # tables
    R.init(1.0, 1.0, 0.5, 1)
    nu, cs, meta = R.tables()
    prs = []
    for typ, par, tot in [(0, 1.0e5, 3.0e49), (0, 3.0e4, 1.0e50), (1, -1.5, 1.0e49)]:
        prs.append(R.photon_rate(typ, par, tot))
    np.savez_compressed(os.path.join(OUT, "golden_tables.npz"), nu=nu, csect=cs, meta=meta,
                        photon_rate=np.asarray(prs),
                        photon_rate_args=np.asarray([[0, 1.0e5, 3.0e49], [0, 3.0e4, 1.0e50],
                                                     [1, -1.5, 1.0e49]]))

    # march on explicit segments
    wl = W.tiny(edge, 6, seed=11)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    segs = edge_case_segments(edge, rng)
    tau, _ = R.march_segments(segs)
    np.savez_compressed(os.path.join(OUT, "golden_march.npz"), edge=edge, dens=wl.dens, fHI=wl.fHI,
                        fHeI=wl.fHeI, fHeII=wl.fHeII, seg=segs, tau=tau, lunit=wl.lunit,
                        denstonh=wl.denstonh)

    # the whole path on every cell
    path_fixture(R, wl, edge, "golden_path.npz")
    wl = W.tiny(19, 7, seed=5)
    wl.theta = 0.6
    R = RefLib(19)
    R.init(wl.lunit, wl.denstonh, wl.theta, 1)
    R.set_mesh(*wl.fields())
    path_fixture(R, wl, 19, "golden_path_ragged.npz")
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
