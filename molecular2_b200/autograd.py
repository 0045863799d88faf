"""torch.autograd shim over the C ABI: the RHF energy as a differentiable
function of the nuclear coordinates.

Forward runs the SCF on the device (``jk_scf_rhf``; SCF::rhf, molecular2
src/scf.cpp:90-185) for the geometry in ``coords``; backward contracts the
derivative integrals with the converged D and W through ``jk_grad_rhf``
(Fock::compute_forces, src/rhfgrad.cpp:15-89), the call molecular2's
optimiser makes (src/optimiser.cpp:410).  Nothing here computes integrals:
the shim only moves arrays between torch and the library.

    E = rhf_energy(coords_bohr, symbols, "cc-pvdz")
    E.backward()          # coords_bohr.grad = dE/dx, natom x 3
"""
import numpy as np
import torch

from .basis import BasisSet, Molecule
from .engine import IntegralEngine


class RHFEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coords, symbols, basis, spherical, scf_opts):
        xyz = coords.detach().cpu().numpy().astype(np.float64)
        mol = Molecule(symbols, xyz, angstrom=False)
        eng = IntegralEngine(BasisSet(mol, basis, spherical=spherical))
        r, ex = eng.scf_rhf(mol.nocc, mol.enuc(), want=True, **scf_opts)
        if not r.converged:
            raise RuntimeError(f"SCF did not converge in {r.iterations} iterations")
        ctx.engine = eng
        ctx.D = ex["D"]
        C = ex["C"][:, :mol.nocc]
        ctx.W = C @ np.diag(ex["eps"][:mol.nocc]) @ C.T
        ctx.precision = scf_opts.get("precision", 1e-12)
        ctx.device = coords.device
        return torch.tensor(r.energy, dtype=torch.float64, device=coords.device)

    @staticmethod
    def backward(ctx, grad_out):
        g, _ = ctx.engine.compute_forces(ctx.D, ctx.W, ctx.precision)
        ctx.engine.close()
        grad = torch.from_numpy(g).to(ctx.device) * grad_out
        return grad, None, None, None, None


def rhf_energy(coords, symbols, basis="cc-pvdz", spherical=True, **scf_opts):
    """RHF energy (Eh) at coords (natom x 3 bohr tensor); differentiable in coords."""
    opts = dict(densconverge=1e-9, enconverge=1e-10, maxiter=100)
    opts.update(scf_opts)
    return RHFEnergy.apply(coords, list(symbols), basis, spherical, opts)
