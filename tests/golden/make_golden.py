"""Extract golden vectors from the reference's own committed solver outputs.

The reference (franciscoparrao/hydroflux) commits four verification profiles
written by solver-2d/examples/gen_verification_data.rs:46-256 with its
solver; this script copies their simulated-depth columns (already rounded by
the reference to 6 or 5 decimals) into tests/golden/reference_verif.npz so
the parity tests can run where the reference tree is absent.

It also copies the reference's forward-mode (Dual) calibration record,
m1_inverse_manning.csv, written by solver-2d/examples/
m1_inverse_manning_demo.rs:124-156: twelve Newton iterations on a 3 x 60
dam break with columns iter, n_estimate, centroid, loss, dc_dn, step (10
significant digits), into tests/golden/reference_m1_inverse_manning.npz.

Run here (where the reference is mounted):
    python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import os
import sys

import numpy as np

FILES = {
    "stoker": ("verif_stoker.csv", 2),        # x, h_analytical, h_sim
    "macdonald": ("verif_macdonald.csv", 2),
    "thacker": ("verif_thacker.csv", 2),
    "uk_ea_t6": ("verif_uk_ea_t6.csv", 2),    # x, y, h, is_building
}


def main(ref_root: str) -> None:
    data_dir = os.path.join(ref_root, "papers", "01_review", "figures", "data")
    out = {}
    for key, (name, col) in FILES.items():
        arr = np.loadtxt(os.path.join(data_dir, name), delimiter=",", skiprows=1)
        out[key] = arr[:, col].astype(np.float64)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_verif.npz")
    np.savez_compressed(dst, **out)
    print(dst, {k: v.shape for k, v in out.items()})
    m1 = np.loadtxt(os.path.join(data_dir, "m1_inverse_manning.csv"), delimiter=",", skiprows=1)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "reference_m1_inverse_manning.npz")
    np.savez_compressed(dst, table=m1.astype(np.float64),
                        columns=np.array(["iter", "n_estimate", "centroid", "loss", "dc_dn",
                                          "step"]))
    print(dst, m1.shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
