"""Generate the golden fixtures of tests/test_golden.py with the CPU oracle.

The reference cannot run here (Fortran, no compiler), so these fixtures pin
the oracle's own output on the 8 mm Cartesian and the cylindrical case:
after the initial refinement loop and two main-loop blocks, the tree, the
step sizes and the interiors of n_e, n_i, phi and |E|. Run:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import a5ref  # noqa: E402
from a5_streamer_b200 import config  # noqa: E402

CASES = {"cartesian_8mm": config.cartesian_8mm, "cylindrical_16mm": config.cylindrical_16mm}
VARS = (0, 1, 4, 5)


def interiors(meta, data, nc):
    out = []
    for i in range(1, meta.shape[0]):
        if not meta[i, 0]:
            continue
        n = meta[i, 14]
        g = n + 2
        out.append(data[i, :g * g].reshape(g, g)[1:n + 1, 1:n + 1].reshape(-1))
    return np.concatenate(out)


def make(name):
    cfg = CASES[name]()
    sim = a5ref.Sim(cfg, n_threads=1)
    n_init = sim.init()
    dts = [sim.advance(True) for _ in range(2)]
    meta = sim.meta()
    rec = {"n_init": np.int32(n_init), "dts": np.asarray(dts), "meta": meta,
           "time": np.float64(sim.time), "dt_red": sim.dt_reductions()}
    for iv in VARS:
        rec[f"v{iv}"] = interiors(meta, sim.cc(iv), cfg.box_size)
    return rec


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}_2blocks.npz"), **make(name))
        print("wrote", name)
