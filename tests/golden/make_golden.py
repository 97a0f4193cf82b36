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

It also copies the inputs of the two UK Environment Agency decks the
reference ships (benchmarks/data/uk_ea/test4: the 5 m floodplain with a line
inflow, and test8a_glasgow: the 2 m urban DEM with rain and a point inflow),
byte for byte, into tests/golden/uk_ea/, so the real-terrain parity tests run
without the reference tree. Test 4's two published LISFLOOD-FP stage records
(test4/reference/*.stage) come along for the deck-reader test.

Run where a checkout of the reference is available:
    python tests/golden/make_golden.py <path of the reference checkout>
"""
from __future__ import annotations

import os
import shutil
import sys

import numpy as np

FILES = {
    "stoker": ("verif_stoker.csv", 2),        # x, h_analytical, h_sim
    "macdonald": ("verif_macdonald.csv", 2),
    "thacker": ("verif_thacker.csv", 2),
    "uk_ea_t6": ("verif_uk_ea_t6.csv", 2),    # x, y, h, is_building
}


UK_EA = {
    "test4": ["ea4.par", "ea4.bci", "ea4.bdy", "ea4.stage", "ea4-5m.dem.gz",
              "reference/ea4-5m-dg2.stage", "reference/ea4-1m-acc.stage"],
    "test8a_glasgow": ["ea8-2m.par", "ea8-2m.bci", "ea8-2m.bdy", "ea8-2m.stage",
                       "ea8-2m.rain", "ea8-2m.dem.gz", "ea8-2m.n.gz"],
}


def copy_uk_ea(ref_root: str) -> None:
    src_root = os.path.join(ref_root, "benchmarks", "data", "uk_ea")
    dst_root = os.path.join(os.path.dirname(os.path.abspath(__file__)), "uk_ea")
    for deck, files in UK_EA.items():
        for rel in files:
            dst = os.path.join(dst_root, deck, rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            shutil.copyfile(os.path.join(src_root, deck, rel), dst)
    print(dst_root, {k: len(v) for k, v in UK_EA.items()})


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
    copy_uk_ea(ref_root)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
