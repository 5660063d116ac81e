"""Host-side helpers of sdfo.contact (no GPU): the SO(3) left Jacobian used
by the contact_force backward, and the rotation-vector map, against scipy."""
import numpy as np
import torch
from scipy.spatial.transform import Rotation


def test_so3_left_jacobian_matches_finite_differences():
    from sdfo.contact import so3_left_jacobian

    th = np.random.default_rng(1).normal(size=(6, 3)) * 0.6
    th[4] = [1e-6, 0.0, 2e-6]   # series branch
    th[5] = [0.0, 0.0, 0.0]
    J = so3_left_jacobian(torch.tensor(th)).numpy()
    for p in range(len(th)):
        num = np.zeros((3, 3))
        base = Rotation.from_rotvec(th[p])
        for k in range(3):
            e = np.zeros(3)
            e[k] = 1e-6
            dp = (Rotation.from_rotvec(th[p] + e) * base.inv()).as_rotvec()
            dm = (Rotation.from_rotvec(th[p] - e) * base.inv()).as_rotvec()
            num[:, k] = (dp - dm) / 2e-6
        assert np.abs(num - J[p]).max() <= 1e-8, p


def test_rotvec_to_matrix_matches_scipy():
    from sdfo.contact import rotvec_to_matrix

    th = np.random.default_rng(2).normal(size=(8, 3))
    th[0] = 0.0
    R = rotvec_to_matrix(torch.tensor(th)).numpy()
    assert np.abs(R - Rotation.from_rotvec(th).as_matrix()).max() <= 1e-14
