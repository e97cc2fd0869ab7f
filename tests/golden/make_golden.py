"""Extract the reference's own golden data for this path into reference_golden.npz.

Reads (as text) the committed fixtures of the reference project:
  tests/test_cmb/test_benchmark_evolve_background.csv        (tau and x_e at 5 scale factors)
  tests/test_cmb/test_benchmark_evolve_perturbations_batched.csv (full states of 3 modes, 320 outputs)
  tests/resources/CLASS_data.json                            (CLASS P_bc(k) at a = 0.01)
  tests/resources/RECFAST_DISCO_EB_data.json                 (x_e(a) of DISCO-EB v0.1.0)
Usage: python tests/golden/make_golden.py /path/to/reference
"""
import csv
import json
import os
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.npz")


def read_csv(path):
    with open(path) as fh:
        rows = list(csv.reader(fh))
    head = rows[0]
    cols = {h: [] for h in head[1:]}
    for r in rows[1:]:
        for h, v in zip(head[1:], r[1:]):
            if v != "":
                cols[h].append(float(v))
    return {h: np.array(v) for h, v in cols.items()}


bg = read_csv(os.path.join(ref, "tests/test_cmb/test_benchmark_evolve_background.csv"))
pb = read_csv(os.path.join(ref, "tests/test_cmb/test_benchmark_evolve_perturbations_batched.csv"))
cl = json.load(open(os.path.join(ref, "tests/resources/CLASS_data.json")))
rf = json.load(open(os.path.join(ref, "tests/resources/RECFAST_DISCO_EB_data.json")))
# keep every 4th of the 320 output times plus the last (fixture size), all 72 variables
sel = np.unique(np.concatenate([np.arange(0, 320, 4), [319]]))
data = {
    "bg_a": np.array([0.001, 0.01, 0.1, 0.5, 1.0]),
    "bg_tau": bg["tau_at_test_points"],
    "bg_exp_xe": bg["xe_at_test_points"],
    "bg_grhom": bg["grhom"],
    "pert_kmodes": pb["kmodes"],
    "pert_out_index": sel,
    "pert_y_k0": pb["yout_k0_flat"].reshape(320, 72)[sel],
    "pert_y_k31": pb["yout_k31_flat"].reshape(320, 72)[sel],
    "pert_y_k63": pb["yout_k63_flat"].reshape(320, 72)[sel],
    "class_k": np.array(cl["k"]),
    "class_pkbc": np.array(cl["Pkbc"]),
    "recfast_a": np.array(rf["a"]),
    "recfast_xe": np.array(rf["xe"]),
}
np.savez_compressed(out, **data)
print(out, os.path.getsize(out), "bytes")
