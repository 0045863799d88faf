"""The oracle's DF gradient restatement (oracle.df_grad2e: analytic three-
and two-index derivative integrals of the oracle's Obara-Saika/HGP code,
contracted with the DF energy's weights) against central differences of the
oracle's own DF two-electron energy at fixed orbital coefficients."""
import numpy as np

import oracle
from molecular2_b200 import geometry
from molecular2_b200.basis import BasisSet


def _e2(mol, C, obs_name, aux_name):
    o, a = BasisSet(mol, obs_name), BasisSet(mol, aux_name)
    n, naux = o.nbf, a.nbf
    Tp = oracle.eri3(o, a)
    T = np.zeros((naux, n, n))
    iu = np.tril_indices(n)
    T[:, iu[0], iu[1]] = Tp.T
    T[:, iu[1], iu[0]] = Tp.T
    V = oracle.eri2(a)
    D = 2.0 * C @ C.T
    d = np.einsum("pmn,mn->p", T, D)
    Tij = np.einsum("mi,pmn,nj->pij", C, T, C).reshape(naux, -1)
    return 0.5 * d @ np.linalg.solve(V, d) - np.sum(np.linalg.solve(V, Tij) * Tij)


def test_oracle_df_gradient_matches_central_differences():
    mol = geometry.water()
    obs, aux = BasisSet(mol, "cc-pvdz"), BasisSet(mol, "vdz-jkfit")
    rng = np.random.default_rng(0)
    C, _ = np.linalg.qr(rng.normal(size=(obs.nbf, mol.nocc)))
    C *= 0.3
    g = oracle.df_grad2e(obs, aux, C)
    assert np.max(np.abs(g.sum(axis=0))) < 1e-12
    h = 1e-4
    for a in range(mol.natom):
        for x in range(3):
            fd = (_e2(mol.displaced(a, x, h), C, "cc-pvdz", "vdz-jkfit")
                  - _e2(mol.displaced(a, x, -h), C, "cc-pvdz", "vdz-jkfit")) / (2 * h)
            assert abs(fd - g[a, x]) < 1e-8, (a, x, fd, g[a, x])
