"""Loading of the reference golden fixtures (tests/golden/*.npz) and mapping of the
reference's DOF numbering onto the (point, face)-key numbering used here."""
import glob
import os

import numpy as np

from conftest import GOLDEN
from bem_for_nonlinear_waves_b200.tank import Tank


def names():
    return sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz")))


class Golden:
    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.z = z
        self.name = name
        ln, wd, dp, A, k, g = z["tank"]
        self.tank = Tank(X=z["X"], tri=z["tri"], face_dirichlet=z["face_dirichlet"], length=ln, width=wd, depth=dp,
                         amplitude=A, wavenumber=k, g=g)
        self.p = int(z["p"])
        self.tol = float(z["tol"])

    def maps(self, dofs):
        """perm[j]: our DOF of reference row j; ours_of_ref_index[i]: our DOF of reference index i."""
        keys = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(dofs["dof_point"], dofs["dof_face"]))}
        rk = list(zip(self.z["dof_point"].tolist(), self.z["dof_face"].tolist()))
        assert set(keys) == set(rk), "DOF key sets differ from the reference"
        perm = np.array([keys[k] for k in rk])
        ours = np.empty(len(perm), int)
        ours[self.z["dof_index"]] = perm
        return perm, ours

    def matvec_input(self, dofs):
        """The reference's mat-vec input v_i = sin(1.7 i + 0.3) in its own index space, as our
        per-DOF (phi, phin) and the expected output in our numbering."""
        perm, ours = self.maps(dofs)
        n = len(perm)
        v = np.zeros(n)
        v[ours] = np.sin(1.7 * np.arange(n) + 0.3)
        kind = dofs["dof_kind"]
        phi = np.where(kind == 0, 0.0, v)
        phin = np.where(kind == 0, v, 0.0)
        out = np.zeros(n)
        out[ours] = self.z["matvec"]
        return phi, phin, out

    def solution(self, dofs):
        perm, _ = self.maps(dofs)
        sol = np.zeros(len(perm))
        sol[perm] = self.z["ans"]
        return sol

    def diag(self, dofs):
        perm, _ = self.maps(dofs)
        d = np.zeros(len(perm))
        d[perm] = self.z["diag"]
        return d

    def surface_values(self, dofs):
        """Per-DOF (phi, phin) of the reference's solution: the known values (the analytic
        linear Stokes potential the reference run was given) with the solved unknowns."""
        from bem_for_nonlinear_waves_b200 import known_values, point_normals

        kv = known_values(self.tank, dofs["dof_point"], dofs["dof_face"], dofs["dof_kind"], point_normals(self.tank))
        sol = self.solution(dofs)
        dirichlet = dofs["dof_kind"] == 0
        return np.where(dirichlet, kv, sol), np.where(dirichlet, sol, kv)

    def mel(self):
        """The reference's MEL quantities of its solution, per point: phi, gradPhi (u) and
        Dphi/Dt of a node moving with the fluid (0.5 |u|^2 - g z at zero pressure)."""
        z = self.z
        n = self.tank.X.shape[0]
        assert np.array_equal(z["mel_point"], np.arange(n))
        return z["mel_phi"], z["mel_u"], z["mel_dphidt"]
