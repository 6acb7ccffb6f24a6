"""Regenerate the golden fixtures in this directory from the reference itself.

Runs oracle/_ref/apf_ref_dump (the reference's own templates compiled by
oracle/Makefile against oracle/shim) on small uniform meshes and packs each case
into one .npz: mesh and DOF maps, assembled blocks, and the reference's whole inner
iteration (direct main solve, slab reconstruction, vertex-patch flux solves,
per-cell indicators), the driver's X-marking indicators, on the cases marked APF_REF_G the
driver's G^delta estimator (its space's restriction, A_G, f_G, rhs_G, lambda_G and
||lambda_G - lambda_delta||^2_{A_G}), and the reference's binary
artifacts of the estimate (cellwise_error.bin, cellwise_error_components.bin, as bytes).  Also extracts the uniform-refinement rows (exact DOF counts and
6-significant-digit estimator values) of the reference's published paper data
(algorithm_data_plot/{1d,2d}/*.csv) into paper_uniform_rows.json.

usage: python tests/golden/make_golden.py REFERENCE_ROOT [CASE ...]
"""
from __future__ import annotations

import csv
import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "apf_ref_dump")

CASES = [
    # (name, dim, p, outer level, example[, environment of the adaptive mode])
    ("p1_l1_smooth", 2, 1, 1, "smooth_initial"),
    ("p1_l2_smooth", 2, 1, 2, "smooth_initial", {"APF_REF_G": "1"}),
    ("p2_l1_smooth", 2, 2, 1, "smooth_initial"),
    ("p1_l1_nonmatching", 2, 1, 1, "non_matching_initial"),
    ("p1_l3_smooth", 2, 1, 3, "smooth_initial"),
    # 1+1D P1 (geometry rows x0 x1 t0 t1); level 5 is the 64 x 64 = 4,096-element mesh
    ("d1_l2_smooth", 1, 1, 2, "smooth_initial"),
    ("d1_l2_nonmatching", 1, 1, 2, "non_matching_initial"),
    ("d1_l5_smooth", 1, 1, 5, "smooth_initial"),
    # adaptive meshes: X refined locally at seeded space-time points by the reference's
    # refine_points_n_times (hanging nodes: weighted restriction rows), Y refined beyond X by
    # one pass of the reference's inner loop (marking + refine_test_space_from_marked_source_cells),
    # optionally a diffusivity kappa per X cell log-uniform in [lo, hi]
    ("p1_adapt_smooth", 2, 1, 2, "smooth_initial",
     {"APF_REF_X_POINTS": "0.3,0.3,0.3;0.71,0.62,0.8", "APF_REF_X_ROUNDS": "3", "APF_REF_Y_PASSES": "1",
      "APF_REF_G": "1"}),
    ("p1_adapt_kappa", 2, 1, 2, "smooth_initial",
     {"APF_REF_X_POINTS": "0.3,0.3,0.3;0.71,0.62,0.8", "APF_REF_X_ROUNDS": "3", "APF_REF_Y_PASSES": "1",
      "APF_REF_KAPPA": "7:0.01:100", "APF_REF_G": "1"}),
    ("p1_adapt_nonmatching", 2, 1, 1, "non_matching_initial",
     {"APF_REF_X_POINTS": "0.2,0.45,0.1", "APF_REF_X_ROUNDS": "4", "APF_REF_Y_PASSES": "1"}),
    ("p1_kappa_uniform", 2, 1, 2, "smooth_initial", {"APF_REF_KAPPA": "3:0.1:10"}),
    # the mesh of the reference's own adaptive driver after three outer cycles (its X and Y
    # marking and refinement; Y cells of the refined-in-time X span several slabs), kappa per
    # square of a 4 x 4 partition
    ("p1_driver_kappa", 2, 1, 1, "smooth_initial",
     {"APF_REF_KAPPA": "11:0.1:10", "APF_REF_KAPPA_BLOCKS": "4", "APF_REF_DRIVER_OUTER": "3"}),
    ("p2_adapt_smooth", 2, 2, 1, "smooth_initial",
     {"APF_REF_X_POINTS": "0.3,0.3,0.3", "APF_REF_X_ROUNDS": "2", "APF_REF_Y_PASSES": "1"}),
    # 1+1D (points x,t)
    ("d1_adapt_smooth", 1, 1, 2, "smooth_initial",
     {"APF_REF_X_POINTS": "0.3,0.3;0.7,0.8", "APF_REF_X_ROUNDS": "3", "APF_REF_Y_PASSES": "1"}),
    ("d1_adapt_nonmatching", 1, 1, 2, "non_matching_initial",
     {"APF_REF_X_POINTS": "0.15,0.05", "APF_REF_X_ROUNDS": "4", "APF_REF_Y_PASSES": "1"}),
]


def dump_case(dim, p, level, example, outdir, extra_env=None):
    env = dict(os.environ, APF_REF_ESTIMATE="1", **(extra_env or {}))
    subprocess.run([REF_BIN, str(dim), str(p), str(level), example, outdir], check=True, env=env)
    arrays = {}
    for f in sorted(glob.glob(os.path.join(outdir, "*.npy"))):
        arrays[os.path.basename(f)[:-4]] = np.load(f)
    # the reference's binary artifacts, byte for byte
    for f in sorted(glob.glob(os.path.join(outdir, "*.bin"))):
        arrays["bin_" + os.path.basename(f)[:-4]] = np.fromfile(f, dtype=np.uint8)
    return arrays


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("APF_REFERENCE_ROOT")
    if not ref_root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [CASE ...] (or set APF_REFERENCE_ROOT)")
    subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), f"REF={ref_root}"], check=True)
    only = set(sys.argv[2:])
    for name, dim, p, level, example, *extra in CASES:
        if only and name not in only:
            continue
        env = extra[0] if extra else {}
        with tempfile.TemporaryDirectory() as tmp:
            arrays = dump_case(dim, p, level, example, tmp, env)
        for key, value in env.items():
            arrays["meta_" + key.lower()] = np.array([value])
        arrays["meta_dim"] = np.array([dim])
        arrays["meta_p"] = np.array([p])
        arrays["meta_level"] = np.array([level])
        arrays["meta_example"] = np.array([example])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        print("wrote", name)
    rows = []
    for dim in ("1d", "2d"):
        for path in sorted(glob.glob(os.path.join(ref_root, "algorithm_data_plot", dim, "*.csv"))):
            with open(path) as fh:
                for r in csv.DictReader(fh):
                    if r.get("record_type") != "outer" or r.get("mode_short") != "uniform":
                        continue
                    rows.append({k: r.get(k) for k in (
                        "dimension", "example", "p", "outer_iteration", "x_true_dofs_before",
                        "y_true_dofs_after", "eta_squared", "y_flux_squared", "y_reconstruction_squared",
                        "divergence_residual_squared", "y_estimator_squared", "iteration_seconds", "source_group",
                        "job_id", "lambda_y_squared", "configured_rho", "y_estimator_threshold_squared")})
    with open(os.path.join(HERE, "paper_uniform_rows.json"), "w") as fh:
        json.dump(rows, fh, indent=0)
    print("wrote paper_uniform_rows.json", len(rows))


if __name__ == "__main__":
    main()
