"""Extract the reference's own golden data for this path into reference_golden.npz.

Reads (as text) the committed fixtures of the reference project:
  tests/test_cmb/test_benchmark_evolve_background.csv        (tau and x_e at 5 scale factors)
  tests/test_cmb/test_benchmark_evolve_perturbations_batched.csv (full states of 3 modes, 320 outputs)
  tests/resources/CLASS_data.json                            (CLASS P_bc(k) at a = 0.01)
  tests/resources/RECFAST_DISCO_EB_data.json                 (x_e(a) of DISCO-EB v0.1.0)
and, into reference_cmb_golden.npz, the CMB chain's fixtures (DISCO-Notebook cosmology, 1024-point
thermal history, 128 camb-sampled modes, 320 output times, lmax 11/11/11/8/3, rtol = atol = 1e-4):
  tests/test_cmb/test_benchmark_compute_{time_derivatives, visibility_functions,
  background_quantities, neutrino_perturbations, metric_perturbations, polarization_terms,
  source_term_sachs_wolfe, source_term_doppler, source_term_polarization, theta_ell, Cell,
  Dell}.csv and test_benchmark_extract_perturbations.csv
and the CLASS TT, EE and TE spectra of tests/resources/class_benchmarks/DISCO-Notebook.csv.
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

cmb = {}
d = os.path.join(ref, "tests/test_cmb")
for stem in ("compute_visibility_functions", "compute_background_quantities", "extract_perturbations",
             "compute_neutrino_perturbations", "compute_metric_perturbations", "compute_polarization_terms",
             "compute_source_term_sachs_wolfe", "compute_source_term_doppler", "compute_source_term_polarization",
             "compute_theta_ell", "compute_Cell", "compute_Dell"):
    for key, v in read_csv(os.path.join(d, f"test_benchmark_{stem}.csv")).items():
        cmb[f"{stem}:{key}"] = v
td = read_csv(os.path.join(d, "test_benchmark_compute_time_derivatives.csv"))
for key, v in td.items():  # [320, 72] per mode; every 4th output time plus the last
    cmb[f"compute_time_derivatives:{key}"] = v.reshape(320, 72)[sel]
cmb["compute_time_derivatives:out_index"] = sel
# the reference's C_l^TT accuracy record against CAMB (|D_disco - D_camb| / D_camb per l = 2..2500)
# and the CAMB spectrum it was measured against
acc = read_csv(os.path.join(d, "test_cmb_vs_camb_DISCO_Notebook_.csv"))
cmb["camb:disco_relative_error"] = acc["relative_error"]
with open(os.path.join(ref, "tests/resources/camb_benchmarks/DISCO-Notebook.csv")) as fh:
    cb = np.array([[float(v) for v in r] for r in list(csv.reader(fh))[1:]])  # columns ell, D_ell
cmb["camb:ell"] = cb[:, 0]
cmb["camb:D_ell"] = cb[:, 1]
# the CLASS spectra the reference's test_cmb_vs_class compares with (no reionisation, no lensing;
# columns ell, D_ell_TT, D_ell_EE, D_ell_TE): TT pins the temperature chain, EE and TE the E-mode
# polarisation spectra, which the reference itself does not compute
with open(os.path.join(ref, "tests/resources/class_benchmarks/DISCO-Notebook.csv")) as fh:
    rows = list(csv.reader(fh))
head, vals = rows[0], np.array([[float(v) for v in r] for r in rows[1:]])
for i, name in enumerate(head):
    cmb[f"class:{name}"] = vals[:, i]
out2 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cmb_golden.npz")
np.savez_compressed(out2, **cmb)
print(out2, os.path.getsize(out2), "bytes")
