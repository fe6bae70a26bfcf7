"""Runs the compiled reference (oracle/_ref/bem_ref_pP, built by oracle/ref/build_ref.sh)
on a tank and parses its dump.  Test infrastructure only."""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def ref_binary(p: int) -> str:
    return os.path.join(REF_DIR, f"bem_ref_p{p}")


def available(p: int) -> bool:
    return os.path.exists(ref_binary(p))


def write_input(path, tank, tol, max_iter):
    X = np.ascontiguousarray(tank.X, np.float64)
    tri = np.ascontiguousarray(tank.tri, np.int32)
    fd = np.ascontiguousarray(tank.face_dirichlet, np.uint8)
    with open(path, "wb") as f:
        f.write(struct.pack("<iii", X.shape[0], tri.shape[0], int(max_iter)))
        f.write(struct.pack("<5d", tank.amplitude, tank.wavenumber, tank.depth, tank.g, tol))
        f.write(X.tobytes())
        f.write(tri.tobytes())
        f.write(fd.tobytes())


def run(p, tank, tol=1e-10, max_iter=500, threads=None, workdir=None, timeout=3600):
    """Returns a dict with the reference's DOF keys, solution, diagonal, leaf of each face,
    near rows, one mat-vec and timings."""
    wd = workdir or tempfile.mkdtemp(prefix="bemref_")
    os.makedirs(wd, exist_ok=True)
    inp = os.path.join(wd, "in.bin")
    out = os.path.join(wd, "out.txt")
    write_input(inp, tank, tol, max_iter)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([ref_binary(p), inp, out, os.path.join(wd, "work")], env=env, capture_output=True, text=True,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference run failed: " + r.stderr[-2000:] + r.stdout[-2000:])
    return parse(out, log=r.stdout)


def parse(path, log=""):
    res = {"log": log}
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0

    def nxt():
        nonlocal i
        s = lines[i]
        i += 1
        return s

    while i < len(lines):
        s = nxt().strip()
        if not s:
            continue
        key, *rest = s.split()
        if key in ("time_setup", "time_solve", "L"):
            res[key] = float(rest[0])
        elif key in ("gmres_iter", "matrix_size", "leaves"):
            res[key] = int(rest[0])
        elif key == "dofs":
            n = int(rest[0])
            a = np.array([list(map(float, nxt().split())) for _ in range(n)]) if n else np.zeros((0, 5))
            res["dof_point"] = a[:, 0].astype(np.int64)
            res["dof_face"] = a[:, 1].astype(np.int64)
            res["dof_index"] = a[:, 2].astype(np.int64)
            res["ans"] = a[:, 3]
            res["diag"] = a[:, 4]
        elif key == "face_leaf":
            n = int(rest[0])
            a = np.array([list(map(float, nxt().split())) for _ in range(n)])
            res["face_leaf"] = a
        elif key == "near_rows":
            n = int(rest[0])
            rows = {}
            for _ in range(n):
                t, m = map(int, nxt().split())
                a = np.array([list(map(float, nxt().split())) for _ in range(m)]) if m else np.zeros((0, 3))
                rows[t] = (a[:, 0].astype(np.int64), a[:, 1], a[:, 2])
            res["near_rows"] = rows
        elif key == "mel":
            n = int(rest[0])
            a = np.array([list(map(float, nxt().split())) for _ in range(n)]) if n else np.zeros((0, 6))
            res["mel_point"] = a[:, 0].astype(np.int64)
            res["mel_phi"] = a[:, 1]
            res["mel_u"] = a[:, 2:5]
            res["mel_dphidt"] = a[:, 5]
        elif key == "matvec":
            n = int(rest[0])
            res["matvec"] = np.array([float(nxt()) for _ in range(n)])
    return res
