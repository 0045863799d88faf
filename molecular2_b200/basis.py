"""Molecules and Gaussian basis sets in the struct-of-arrays form of ``jk_basis``.

Mirrors how molecular2 assembles its shell lists: ``Molecule::buildShellBasis``
(``src/molecule.cpp:655-671``) walks the atoms in input order and appends each
atom's shells in library order (``src/basisreader.cpp:92-132``,
``src/basis.cpp:33-66``).  One contraction column is one shell
(``basislibrary/parsebasis.py:55-68``).  Coefficients stay as printed in the
library; the engine normalises them the way ``libint2::Shell`` does.

Basis-function ordering and normalisation conventions (shared by the CUDA
engine and the oracle):
  * shells in atom order, functions of a shell contiguous (``src/integrals.cpp:358-369``);
  * Cartesian components ``for a=l..0, for b=l-a..0: x^a y^b z^(l-a-b)``;
  * pure (spherical) shells for l >= 2 when ``spherical=True``, ``m=-l..l``.
"""
import ctypes
import json
import os

import numpy as np

TOBOHR = 1.889726124565          # src/logger.cpp:31
ZNUC = {"h": 1, "he": 2, "c": 6, "n": 7, "o": 8}
SYMBOL = {v: k for k, v in ZNUC.items()}

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis_sets.json")
_CACHE = {}


def library():
    if "lib" not in _CACHE:
        with open(_DATA) as f:
            _CACHE["lib"] = json.load(f)
    return _CACHE["lib"]


class Molecule:
    """Atoms with nuclear charges and bohr coordinates (``Molecule``, ``inc/molecule.hpp:68-133``)."""

    def __init__(self, symbols, coords, angstrom=True, charge=0):
        self.symbols = [s.lower() for s in symbols]
        xyz = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
        self.xyz = xyz * (TOBOHR if angstrom else 1.0)
        self.Z = np.array([ZNUC[s] for s in self.symbols], dtype=np.float64)
        self.charge = charge

    @property
    def natom(self):
        return len(self.symbols)

    @property
    def nelec(self):
        return int(self.Z.sum()) - self.charge

    @property
    def nocc(self):
        return self.nelec // 2

    def enuc(self):
        """Nuclear repulsion energy (``Molecule::calcEnuc``, ``src/molecule.cpp:443-457``)."""
        e = 0.0
        for i in range(self.natom):
            for j in range(i + 1, self.natom):
                e += self.Z[i] * self.Z[j] / np.linalg.norm(self.xyz[i] - self.xyz[j])
        return e

    def enuc_grad(self):
        """d E_nuc / d x, natom x 3 (the FN term of ``src/rhfgrad.cpp:59-86``)."""
        g = np.zeros((self.natom, 3))
        for a1 in range(1, self.natom):
            for a2 in range(a1):
                r = self.xyz[a1] - self.xyz[a2]
                d = np.linalg.norm(r)
                f = -r * self.Z[a1] * self.Z[a2] / d ** 3
                g[a1] += f
                g[a2] -= f
        return g

    def displaced(self, atom, xyz, h):
        m = Molecule(self.symbols, self.xyz.copy(), angstrom=False, charge=self.charge)
        m.xyz[atom, xyz] += h
        return m


class JKBasisStruct(ctypes.Structure):
    """ctypes image of ``jk_basis`` (include/jk_engine.h)."""
    _fields_ = [
        ("nshell", ctypes.c_int),
        ("l", ctypes.POINTER(ctypes.c_int)),
        ("nprim", ctypes.POINTER(ctypes.c_int)),
        ("prim_off", ctypes.POINTER(ctypes.c_int)),
        ("exps", ctypes.POINTER(ctypes.c_double)),
        ("coefs", ctypes.POINTER(ctypes.c_double)),
        ("xyz", ctypes.POINTER(ctypes.c_double)),
        ("pure", ctypes.POINTER(ctypes.c_int)),
        ("atom", ctypes.POINTER(ctypes.c_int)),
    ]


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class BasisSet:
    """A list of contracted shells with SoA arrays ready for the C ABI."""

    def __init__(self, mol, name, spherical=True):
        lib = library()
        if name not in lib:
            raise KeyError(f"basis {name!r} not in the library")
        shells = []
        for a, sym in enumerate(mol.symbols):
            if sym not in lib[name]:
                # molecular2 throws Error("BASISLIB", ...) here (src/basisreader.cpp:127-131)
                raise KeyError(f"BASISLIB: could not read basis {name} for atom {sym}")
            for sh in lib[name][sym]:
                shells.append((sh["l"], sh["exps"], sh["coefs"], a))
        self.name = name
        self.spherical = spherical
        self._set(shells, mol)

    @classmethod
    def from_shells(cls, shells, mol, spherical=True, name="custom"):
        """shells: list of (l, exps, coefs, atom)."""
        obj = cls.__new__(cls)
        obj.name = name
        obj.spherical = spherical
        obj._set(shells, mol)
        return obj

    def _set(self, shells, mol):
        self.mol = mol
        self.shells = shells
        ns = len(shells)
        self.l = np.array([s[0] for s in shells], dtype=np.int32)
        self.nprim = np.array([len(s[1]) for s in shells], dtype=np.int32)
        self.prim_off = np.zeros(ns, dtype=np.int32)
        if ns:
            self.prim_off[1:] = np.cumsum(self.nprim)[:-1]
        self.exps = np.array([e for s in shells for e in s[1]], dtype=np.float64)
        self.coefs = np.array([c for s in shells for c in s[2]], dtype=np.float64)
        self.atom = np.array([s[3] for s in shells], dtype=np.int32)
        self.xyz = np.ascontiguousarray(mol.xyz[self.atom].reshape(-1), dtype=np.float64)
        self.pure = np.array([1 if (self.spherical and s[0] >= 2) else 0 for s in shells], dtype=np.int32)
        sizes = [(2 * l + 1) if p else (l + 1) * (l + 2) // 2 for l, p in zip(self.l, self.pure)]
        self.bf_off = np.zeros(ns + 1, dtype=np.int64)
        self.bf_off[1:] = np.cumsum(sizes)
        self._struct = None

    @property
    def nshell(self):
        return len(self.shells)

    @property
    def nbf(self):
        return int(self.bf_off[-1])

    @property
    def max_l(self):
        return int(self.l.max()) if self.nshell else 0

    def with_geometry(self, mol):
        return BasisSet.from_shells(self.shells, mol, self.spherical, self.name)

    def struct(self):
        """A ctypes ``jk_basis`` pointing into this object's arrays (keep self alive)."""
        if self._struct is None:
            self.xyz = np.ascontiguousarray(self.mol.xyz[self.atom].reshape(-1), dtype=np.float64)
            self._struct = JKBasisStruct(self.nshell, _iptr(self.l), _iptr(self.nprim), _iptr(self.prim_off),
                                         _dptr(self.exps), _dptr(self.coefs), _dptr(self.xyz),
                                         _iptr(self.pure), _iptr(self.atom))
        return self._struct


def sto3g_density(mol):
    """Minimal-basis SOAD density, shell-diagonal, as ``Fock::compute_soad_guess``
    builds it (``src/fock.cpp:174-225`` with ``inc/sto3g_atomic_density.hpp``):
    spherically averaged neutral-atom occupations on the diagonal, times 0.5."""
    occ = []
    for z in mol.Z.astype(int):
        ne = z
        sub = [1] if z <= 2 else [1, 1, 3]
        vec = []
        for size in sub:
            alloc = min(ne, 2 * size)
            ne -= alloc
            vec += [alloc / size] * size
        occ += vec
    return 0.5 * np.diag(np.array(occ, dtype=np.float64))
