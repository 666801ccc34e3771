"""The Newton-Raphson Jacobian builder (ybus_b200/configs.py), on the CPU: its columns are the
derivatives of the power injections S = V conj(Ybus V) (`newtonpf`'s mismatch, ybus_powerflow/src/
ac.rs:1107-1132) by central differences, its order is the PV and PQ angles plus the PQ magnitudes,
and its host LU reconstructs it and solves it like a dense solve."""
import numpy as np

import oracle.oracle as orc
from ybus_b200 import configs


def _injection_vector(ybus, vm, va, pv, pq):
    s = configs.power_injections(ybus, vm * np.exp(1j * va))
    return np.concatenate([s.real[np.concatenate([pv, pq])], s.imag[pq]])


def test_jacobian_columns_are_the_injections_derivatives():
    sys_ = configs.jacobian_system(300, count=4)
    pv, pq, v = sys_.pv, sys_.pq, sys_.voltage
    vm, va = np.abs(v), np.angle(v)
    j = sys_.jacobian.to_dense()
    pvpq = np.concatenate([pv, pq])
    assert j.shape == (pvpq.size + pq.size,) * 2
    h = 1e-6
    rng = np.random.default_rng(3)
    for col in rng.choice(j.shape[1], 40, replace=False):
        dm, da = np.zeros_like(vm), np.zeros_like(va)
        if col < pvpq.size:
            da[pvpq[col]] = h
        else:
            dm[pq[col - pvpq.size]] = h
        fd = (_injection_vector(sys_.ybus, vm + dm, va + da, pv, pq) -
              _injection_vector(sys_.ybus, vm - dm, va - da, pv, pq)) / (2 * h)
        assert np.abs(fd - j[:, col]).max() <= 1e-6 * max(1.0, np.abs(j[:, col]).max()), col


def test_jacobian_lu_reconstructs_and_solves():
    sys_ = configs.jacobian_system(300, count=6)
    assert orc.lu_reconstruction_error(sys_.lu, sys_.jacobian.to_dense()) < 1e-12
    x = orc.solve_many_lu(sys_.lu, sys_.rhs)
    dense = np.linalg.solve(sys_.jacobian.to_dense(), sys_.rhs.T).T
    assert np.abs(x - dense).max() <= 1e-9 * np.abs(dense).max()
