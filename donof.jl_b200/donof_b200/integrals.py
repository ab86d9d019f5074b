"""Integral front end: molecules, basis sets from Gaussian94-format text, and
``compute_integrals`` (src/integrals.jl:1-66; src/io.jl:27-59) over the
library's McMurchie-Davidson engine (csrc/ints.cu, C ABI donof_basis_* and
donof_int*).  The reference obtains the same matrices from GaussianBasis.jl
(libcint); here the operator supplies the basis-set text (for example the
cc-pVDZ and cc-pVDZ-jkfit files of a basis-set library), since no basis data
ships with this package.

Conventions: geometry in Angstrom as in the reference's molecule strings,
converted to bohr with 1/0.52917721092 for the integrals; compute_E_nuc keeps
the reference's own factor 1.88973 (src/utils.jl:299-312).  Spherical shells
order p as (x, y, z) and l >= 2 as m = -l..l; Cartesian shells xx..x, xx..y,
..., zz..z, normalised like x^l (the libcint convention).
"""
from __future__ import annotations

import ctypes as ct
import re
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .param import Param

ANGSTROM_TO_BOHR = 1.0 / 0.52917721092
E_NUC_FACTOR = 1.88973  # src/utils.jl:305

ELEMENTS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar",
            "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br",
            "Kr"]
_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5}


@dataclass
class Atom:
    symbol: str
    Z: int
    xyz: np.ndarray  # Angstrom


def parse_molecule(mol: str) -> Tuple[List[Atom], int, int]:
    """Atoms, charge and multiplicity of a molecule string: an optional first
    line "charge multiplicity", then "Symbol x y z" lines in Angstrom
    (src/io.jl:27-44)."""
    lines = [ln for ln in mol.strip().split("\n") if ln.strip()]
    charge, mult = 0, 1
    if lines and len(lines[0].split()) == 2:
        charge, mult = (int(x) for x in lines[0].split())
        lines = lines[1:]
    atoms = []
    for ln in lines:
        tok = ln.split()
        sym = tok[0].capitalize()
        if sym not in ELEMENTS:
            raise ValueError(f"unknown element {tok[0]!r}")
        atoms.append(Atom(sym, ELEMENTS.index(sym) + 1, np.array([float(v) for v in tok[1:4]])))
    return atoms, charge, mult


def _num(s: str) -> float:
    return float(s.replace("D", "E").replace("d", "e"))


def parse_gbs(text: str) -> Dict[str, List[Tuple[int, np.ndarray, np.ndarray]]]:
    """Shells per element of a Gaussian94-format basis set: blocks "El 0",
    shell lines "L nprim scale" (L in S, P, D, F, G, H, or SP with an s and a p
    coefficient column), primitives "exponent coefficient(s)", blocks ended by
    "****"; "!" starts a comment.  Returns {symbol: [(l, exponents,
    coefficients), ...]}."""
    out: Dict[str, List[Tuple[int, np.ndarray, np.ndarray]]] = {}
    lines = [ln.split("!")[0].strip() for ln in text.split("\n")]
    lines = [ln for ln in lines if ln]
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        if tok[0] == "****" or tok[0].startswith("$"):
            i += 1
            continue
        sym = tok[0].capitalize()
        if sym not in ELEMENTS or len(tok) < 2 or not re.fullmatch(r"-?\d+", tok[1]):
            raise ValueError(f"basis text: expected an element header, got {lines[i]!r}")
        shells = out.setdefault(sym, [])
        i += 1
        while i < len(lines) and lines[i] != "****":
            head = lines[i].split()
            kind, nprim = head[0].upper(), int(head[1])
            scale = _num(head[2]) if len(head) > 2 else 1.0
            rows = [[_num(x) for x in lines[i + 1 + k].split()] for k in range(nprim)]
            ex = np.array([r[0] for r in rows]) * scale * scale
            if kind == "SP":
                shells.append((0, ex, np.array([r[1] for r in rows])))
                shells.append((1, ex, np.array([r[2] for r in rows])))
            elif kind in _L:
                shells.append((_L[kind], ex, np.array([r[1] for r in rows])))
            else:
                raise ValueError(f"basis text: unknown shell type {kind!r}")
            i += 1 + nprim
        i += 1
    return out


class BasisSet:
    """A basis on a molecule: the shells of each atom's element, centred on the
    atom (bohr), held by the library as a donof_basis.  ``nbas`` and ``natoms``
    as in GaussianBasis.jl's BasisSet."""

    def __init__(self, name: str, atoms: Sequence[Atom], shells: Dict[str, list], spherical: bool = True):
        self.name, self.atoms, self.spherical = name, list(atoms), bool(spherical)
        ls, ctr, npr, ex, co = [], [], [], [], []
        for a in self.atoms:
            if a.symbol not in shells:
                raise ValueError(f"basis {name!r} has no shells for {a.symbol}")
            for l, e, c in shells[a.symbol]:
                ls.append(l)
                ctr.extend(a.xyz * ANGSTROM_TO_BOHR)
                npr.append(len(e))
                ex.extend(e)
                co.extend(c)
        self.shell_l = np.array(ls, dtype=np.int32)
        self._ctr = np.array(ctr, dtype=np.float64)
        self._npr = np.array(npr, dtype=np.int32)
        self._ex = np.array(ex, dtype=np.float64)
        self._co = np.array(co, dtype=np.float64)
        self.lib = _lib.load()
        h = ct.c_void_p()
        _lib.check(self.lib.donof_basis_create(len(ls), self.shell_l.ctypes.data, self._ctr.ctypes.data,
                                               self._npr.ctypes.data, self._ex.ctypes.data, self._co.ctypes.data,
                                               int(self.spherical), ct.byref(h)))
        self.handle = h
        self.nbas = int(self.lib.donof_basis_nbf(h))
        self.natoms = len(self.atoms)

    @classmethod
    def from_text(cls, name: str, text: str, atoms: Sequence[Atom], spherical: bool = True) -> "BasisSet":
        return cls(name, atoms, parse_gbs(text), spherical)

    def free(self) -> None:
        if getattr(self, "handle", None):
            self.lib.donof_basis_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _nuclei(atoms: Sequence[Atom]):
    Z = np.array([a.Z for a in atoms], dtype=np.float64)
    xyz = np.ascontiguousarray(np.array([a.xyz for a in atoms], dtype=np.float64) * ANGSTROM_TO_BOHR)
    return Z, xyz


def one_electron(bset: BasisSet, nuclei: Optional[Sequence[Atom]] = None):
    """S, T, V (column-major nbf x nbf); V over the basis' atoms, or over the
    given nuclei."""
    n = bset.nbas
    S, T, V = (np.zeros((n, n), order="F") for _ in range(3))
    Z, xyz = _nuclei(bset.atoms if nuclei is None else nuclei)
    _lib.check(bset.lib.donof_int1e(bset.handle, len(Z), Z.ctypes.data, xyz.ctypes.data, S.ctypes.data,
                                    T.ctypes.data, V.ctypes.data))
    return S, T, V


def overlap(bset: BasisSet) -> np.ndarray:
    return one_electron(bset)[0]


def kinetic(bset: BasisSet) -> np.ndarray:
    return one_electron(bset)[1]


def nuclear(bset: BasisSet) -> np.ndarray:
    return one_electron(bset)[2]


def ERI_2e2c(aux: BasisSet) -> np.ndarray:
    """G[P, Q] = (P|Q)."""
    G = np.zeros((aux.nbas, aux.nbas), order="F")
    _lib.check(aux.lib.donof_int2c2e(aux.handle, G.ctypes.data))
    return G


def ERI_2e3c(bset: BasisSet, aux: BasisSet) -> np.ndarray:
    """I[m, n, P] = (mn|P) (column-major nbf x nbf x naux), on host threads."""
    I = np.zeros((bset.nbas, bset.nbas, aux.nbas), order="F")
    _lib.check(bset.lib.donof_int3c2e(bset.handle, aux.handle, I.ctypes.data))
    return I


def ERI_2e3c_dev(bset: BasisSet, aux: BasisSet, ctx):
    """(mn|P) computed on the context's B200 into a CUDA tensor holding the
    column-major nbf x nbf x naux array (orbital shells up to f, auxiliary up
    to g)."""
    import torch

    out = torch.empty(bset.nbas * bset.nbas * aux.nbas, dtype=torch.float64, device=f"cuda:{ctx.device}")
    torch.cuda.synchronize(ctx.device)
    ctx.check(bset.lib.donof_int3c2e_dev(ctx.handle, bset.handle, aux.handle, ct.c_void_p(out.data_ptr())))
    return out


def ERI_2e4c(bset: BasisSet) -> np.ndarray:
    """I[m, n, l, s] = (mn|ls) (nbf^4, small bases)."""
    n = bset.nbas
    I = np.zeros((n, n, n, n), order="F")
    _lib.check(bset.lib.donof_int4c2e(bset.handle, I.ctypes.data))
    return I


def compute_E_nuc(bset: BasisSet, p: Optional[Param] = None) -> float:
    """sum_{i<j} Z_i Z_j / (|R_i - R_j| 1.88973) with R in Angstrom (src/utils.jl:299-312)."""
    E = 0.0
    at = bset.atoms
    for i in range(len(at)):
        for j in range(i + 1, len(at)):
            E += at[i].Z * at[j].Z / (np.linalg.norm(at[i].xyz - at[j].xyz) * E_NUC_FACTOR)
    return E


def molecule(mol: str, basis_text: str, spherical: bool = False, name: str = "basis"):
    """bset, p = molecule(mol, basis) (src/io.jl:27-59): the basis on the
    molecule and the job parameters from its electron count, charge and
    multiplicity (src/param.jl:60-125); p.nbfaux is set by compute_integrals."""
    atoms, charge, mult = parse_molecule(mol)
    bset = BasisSet.from_text(name, basis_text, atoms, spherical)
    ne = sum(a.Z for a in atoms) - charge
    if (ne + mult - 1) % 2:
        raise ValueError(f"{ne} electrons cannot have multiplicity {mult}")
    nalpha, nbeta = (ne + mult - 1) // 2, (ne - mult + 1) // 2
    p = Param(nbf=bset.nbas, nbfaux=0, nalpha=nalpha, nbeta=nbeta)
    p.extra.update(mol=mol, spherical=spherical, charge=charge, mul=mult, natoms=len(atoms))
    return bset, p


def compute_integrals(bset: BasisSet, aux, p: Param, ctx=None, precision: str = "fp64",
                      device_3c: bool = True):
    """S, T, V, H, b = compute_integrals(bset, aux, p) (src/integrals.jl:1-66):
    the one-electron matrices symmetrised as the reference does (aux: a
    BasisSet, or the auxiliary basis' Gaussian94 text, placed on bset's atoms in
    bset's spherical or Cartesian form as the reference does); with p.RI,
    G = (P|Q) symmetrised, (mn|P) (on the B200 when its shells fit the device
    kernel and device_3c, else on host threads), then b = I G^{-1/2} built on
    the device (Iaux_gpu) and kept there as the job's RI tensor, and p.nbfaux
    set; without p.RI the four-index (mn|ls) array (ERI_2e4c, host) in place
    of b."""
    from . import api

    if isinstance(aux, str):  # the auxiliary basis' text: on the same atoms, in the same form (src/integrals.jl:17-39)
        aux = BasisSet.from_text(bset.name + "-jkfit", aux, bset.atoms, bset.spherical)
    S, T, V = one_electron(bset)
    S, T, V = (S + S.T) / 2, (T + T.T) / 2, (V + V.T) / 2
    H = T + V
    if not p.RI:
        return (np.asfortranarray(S), np.asfortranarray(T), np.asfortranarray(V), np.asfortranarray(H),
                ERI_2e4c(bset))
    ctx = ctx or api.default_context()
    G = ERI_2e2c(aux)
    G = (G + G.T) / 2
    lmax_orb = int(bset.shell_l.max()) if len(bset.shell_l) else 0
    lmax_aux = int(aux.shell_l.max()) if len(aux.shell_l) else 0
    if device_3c and lmax_orb <= 3 and lmax_aux <= 4:
        I = ERI_2e3c_dev(bset, aux, ctx).cpu().numpy().reshape((bset.nbas, bset.nbas, aux.nbas), order="F")
    else:
        I = ERI_2e3c(bset, aux)
    b = api.Iaux_gpu(G, I, precision, ctx)
    p.nbfaux = aux.nbas
    return np.asfortranarray(S), np.asfortranarray(T), np.asfortranarray(V), np.asfortranarray(H), b
