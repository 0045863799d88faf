"""RHF nuclear gradient on the B200 against the oracle's restatement of
Fock::compute_forces / compute_2body_fock_deriv<1> and against central
differences of the GPU SCF energy.

Bars: same D, W as the oracle: every component within 1e-9 Eh/bohr;
analytic vs central differences (step 1e-4 bohr): 1e-6 Eh/bohr.
"""
import numpy as np
import pytest

import oracle
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet

pytestmark = pytest.mark.gpu


def _engine(b):
    from molecular2_b200.engine import IntegralEngine
    return IntegralEngine(b)


def _dens(b, seed):
    n, o = b.nbf, b.mol.nocc
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.normal(size=(n, o)))
    eps = -np.sort(rng.uniform(0.2, 20.0, size=o))
    return 2.0 * C @ C.T, C @ np.diag(eps) @ C.T


def _oracle_forces(b, D, W):
    S1, T1, V1 = oracle.one_body_deriv(b)
    na = b.mol.natom
    F1 = np.array([np.sum((T1[i] + V1[i]) * D) for i in range(3 * na)]).reshape(na, 3)
    Fp = -np.array([2.0 * np.sum(S1[i] * W) for i in range(3 * na)]).reshape(na, 3)
    F2 = oracle.grad2e(b, D, oracle.schwarz(b), 1e-12)
    return F1 + Fp + F2 + b.mol.enuc_grad(), F2


@pytest.mark.parametrize("basis,spherical,k", [("cc-pvdz", True, 1), ("cc-pvdz", False, 1), ("6-311g**", True, 1),
                                               ("cc-pvdz", True, 2)])
def test_gradient_matches_oracle(basis, spherical, k):
    mol = geometry.water() if k == 1 else geometry.water_cluster(k, 5.0, seed=3)
    b = BasisSet(mol, basis, spherical=spherical)
    D, W = _dens(b, 9)
    g, g2 = _engine(b).compute_forces(D, W)
    gr, g2r = _oracle_forces(b, D, W)
    assert np.max(np.abs(g2 - g2r)) < 1e-9
    assert np.max(np.abs(g - gr)) < 1e-9
    # translational invariance of the total
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9


def test_gradient_central_differences():
    mol = geometry.water_cluster(2, 5.0, seed=3)
    b = BasisSet(mol, "cc-pvdz")
    conv = dict(densconverge=1e-9, enconverge=1e-11, maxiter=100)
    eng = _engine(b)
    r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), want=True, **conv)
    assert r.converged
    C = ex["C"][:, :mol.nocc]
    W = C @ np.diag(ex["eps"][:mol.nocc]) @ C.T
    g, _ = eng.compute_forces(ex["D"], W)
    h = 1e-4
    for a, x in [(0, 0), (1, 2), (4, 1)]:
        Es = []
        for sgn in (1, -1):
            m2 = mol.displaced(a, x, sgn * h)
            r2, _ = _engine(b.with_geometry(m2)).scf_rhf(m2.nocc, m2.enuc(), **conv)
            assert r2.converged
            Es.append(r2.energy)
        fd = (Es[0] - Es[1]) / (2 * h)
        assert abs(fd - g[a, x]) < 1e-6, (a, x, fd, g[a, x])


def test_autograd_shim():
    """torch.autograd.Function over jk_scf_rhf / jk_grad_rhf: backward equals
    compute_forces at the converged SCF and central differences of forward."""
    import torch
    from molecular2_b200.autograd import rhf_energy
    mol = geometry.water_cluster(2, 5.0, seed=3)
    x = torch.tensor(mol.xyz, dtype=torch.float64, requires_grad=True)
    E = rhf_energy(x, mol.symbols, "cc-pvdz")
    E.backward()
    g = x.grad.numpy()
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9
    h = 1e-4
    for a, c in [(2, 0), (3, 1)]:
        Es = []
        for sgn in (1, -1):
            xd = x.detach().clone()
            xd[a, c] += sgn * h
            Es.append(float(rhf_energy(xd, mol.symbols, "cc-pvdz")))
        assert abs((Es[0] - Es[1]) / (2 * h) - g[a, c]) < 1e-6
