"""The analytic Kirkwood oracle and the sphere case of the baseline
(20,480-triangle icosphere of radius 20 A, 500 seeded charges, p=3, MAC 0.8,
eps 1/80, kappa 0.1257, GMRES tol 1e-4).

* CPU: the Kirkwood series reduces to the Born energy of a centred charge,
  E = -(332.0716 q^2 / 2a) (1/eps_in - 1/(eps_out (1 + kappa a))).
* GPU: the solved energy is within 1% of the series (the flat-triangle
  discretisation error of this mesh is a few tenths of a percent), in FP64
  and in mixed precision, and the two precisions agree to 1e-4.
"""
import os
import tempfile

import numpy as np
import pytest

from fabipb_b200 import meshgen, meshio

KCAL = 2.0 * np.pi * 332.0716


def test_kirkwood_born_limit():
    a, q, ein, eout, kap = 20.0, 1.7, 2.0, 80.0, 0.1257
    e = meshgen.kirkwood_energy(np.array([[1e-12, 0.0, 0.0]]), np.array([q]), a, ein, eout, kap, lmax=10)
    born = -332.0716 * q * q / (2 * a) * (1 / ein - 1 / (eout * (1 + kap * a)))
    assert abs(e - born) <= 1e-9 * abs(born)


@pytest.fixture(scope="module")
def sphere20480():
    d = tempfile.mkdtemp(prefix="fabipb_kirkwood_")
    base = os.path.join(d, "sphere20480")
    meshgen.sphere_case(base, nsub=5, radius=20.0, n_charges=500, seed=0)
    return base


@pytest.mark.gpu
def test_sphere_energy_matches_kirkwood(sphere20480):
    from fabipb_b200 import lib
    pan, ch = meshio.load_case(sphere20480)
    assert pan.n == 20480
    ek = meshgen.kirkwood_energy(ch.pos, ch.q, 20.0, 1.0, 80.0, 0.1257)
    energies = {}
    for prec in (lib.FP64, lib.MIXED):
        s = lib.Surface(pan, lib.params(order=3, depth=3, sep_ratio=0.8, eps1=1.0, eps2=80.0, precision=prec), ch)
        b = s.rhs()
        s.precond_setup(2)
        x, it, res, info = s.solve(b, b.copy(), restart=10, maxit=100, tol=1e-4)
        assert info == 0
        energies[prec] = s.energy_raw(x) * KCAL
        assert abs(energies[prec] - ek) <= 0.01 * abs(ek), (prec, energies[prec], ek)
    assert abs(energies[lib.MIXED] - energies[lib.FP64]) <= 1e-4 * abs(energies[lib.FP64])
