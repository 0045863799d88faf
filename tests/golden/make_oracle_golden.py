"""Oracle outputs too slow to recompute inside a test, kept as fixtures.

    python tests/golden/make_oracle_golden.py

Writes ``oracle_grad_water8.json``: the two-electron RHF gradient
(compute_2body_fock_deriv<1> contracted as compute_forces does, molecular2
src/rhfgrad.cpp:419-598, :15-89) of the (H2O)8 / cc-pVDZ workload (seed 8,
7 A cube, spherical d) for a seeded density, computed by the oracle's scalar
restatement (about six minutes on eight host threads).  The density is
D = 2 C C^T for the orthonormalised columns of a seeded normal matrix
(numpy default_rng(SEED), n x nocc), so the test regenerates it exactly.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

SEED = 808


def density(nbf, nocc, seed=SEED):
    C, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(nbf, nocc)))
    return 2.0 * C @ C.T


def main():
    import oracle
    from molecular2_b200 import geometry
    from molecular2_b200.basis import BasisSet
    mol = geometry.water8()
    b = BasisSet(mol, "cc-pvdz")
    D = density(b.nbf, mol.nocc)
    g = oracle.grad2e(b, D, oracle.schwarz(b), 1e-12)
    out = {"workload": "(H2O)8 / cc-pVDZ, geometry.water8() (seed 8, 7 A cube), spherical d",
           "density": f"D = 2 C C^T, C = orthonormalised default_rng({SEED}).normal(size=(n, nocc))",
           "precision": 1e-12, "grad2e": g.tolist()}
    dst = os.path.join(HERE, "oracle_grad_water8.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
