"""Generates golden fixtures by running the compiled, unmodified reference GMRES-FMM path
(oracle/_ref/bem_ref_pP, built by oracle/ref/build_ref.sh from the reference sources) on
small seeded tanks: the solve, its intermediates, and the MEL quantities of the solution
(point phi, the velocity gradPhi and Dphi/Dt of a node moving with the fluid).  Writes
tests/golden/<name>.npz.  Needs the reference checkout at
build time only; the fixtures themselves are self-contained.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from bem_for_nonlinear_waves_b200.tank import make_tank  # noqa: E402
import refrun  # noqa: E402

CASES = {
    # flat free surface, p=8
    "tank_h0p1_p8": dict(tank=dict(h=0.1), p=8, tol=1e-12),
    # free surface with seeded z-noise (sigma = 0.2 h), p=10
    "tank_h0p1_noise_p10": dict(tank=dict(h=0.1, noise_sigma=0.02, seed=7), p=10, tol=1e-12),
    # the 2,802-point plain FP64 configuration: 2.0 x 1.0 x 0.5 m tank, h = 0.05, p = 8
    "tank_h0p05_p8": dict(tank=dict(length=2.0, width=1.0, depth=0.5, h=0.05), p=8, tol=1e-12),
}

SAMPLE_ROWS = 12  # near-field rows stored in full; the others as checksums


def make(name, spec):
    t = make_tank(**spec["tank"])
    R = refrun.run(spec["p"], t, tol=spec["tol"], max_iter=2000)
    L = float(np.sqrt(((t.X.max(0) - t.X.min(0)) ** 2).sum()))
    # near rows: checksums for every point, full rows for a seeded sample
    pts = np.array(sorted(R["near_rows"].keys()))
    cnt = np.array([len(R["near_rows"][p][0]) for p in pts])
    sg = np.array([R["near_rows"][p][1].sum() for p in pts])
    sgn = np.array([R["near_rows"][p][2].sum() for p in pts])
    sag = np.array([np.abs(R["near_rows"][p][1]).sum() for p in pts])
    rng = np.random.default_rng(0)
    sample = np.sort(rng.choice(pts, size=min(SAMPLE_ROWS, len(pts)), replace=False))
    rows_idx, rows_g, rows_gn, rows_off = [], [], [], [0]
    for p in sample:
        i, g, gn = R["near_rows"][p]
        rows_idx.append(i)
        rows_g.append(g)
        rows_gn.append(gn)
        rows_off.append(rows_off[-1] + len(i))
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        X=t.X, tri=t.tri, face_dirichlet=t.face_dirichlet,
        tank=np.array([t.length, t.width, t.depth, t.amplitude, t.wavenumber, t.g]),
        p=spec["p"], tol=spec["tol"], L=L,
        dof_point=R["dof_point"], dof_face=R["dof_face"], dof_index=R["dof_index"], ans=R["ans"], diag=R["diag"],
        gmres_iter=R["gmres_iter"], matvec=R["matvec"], face_leaf=R["face_leaf"],
        near_points=pts, near_count=cnt, near_sum_g=sg, near_sum_gn=sgn, near_sumabs_g=sag,
        sample_points=sample, sample_off=np.array(rows_off), sample_idx=np.concatenate(rows_idx),
        sample_g=np.concatenate(rows_g), sample_gn=np.concatenate(rows_gn),
        time_setup=R["time_setup"], time_solve=R["time_solve"],
        mel_point=R["mel_point"], mel_phi=R["mel_phi"], mel_u=R["mel_u"], mel_dphidt=R["mel_dphidt"],
    )
    print(name, "ref iters", R["gmres_iter"], "setup", R["time_setup"], "solve", R["time_solve"])


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        if not refrun.available(CASES[n]["p"]):
            raise SystemExit(f"reference binary for p={CASES[n]['p']} missing; run oracle/ref/build_ref.sh")
        make(n, CASES[n])
