"""Formatted checkpoint output of a converged GNOF energy: the ``.fchk`` file
that ``fchk(filename, p, bset, jobtype, E_t, elag, n, C)`` writes in
src/output.jl:1-283 (called from src/energy.jl:274 and :569).

The reference takes the basis from GaussianBasis.jl (``bset``) and re-reads
the raw contraction coefficients from the basis library's ``.gbs`` file.  This
build has no basis library, so the caller passes the same facts as a
:class:`BasisDescription`: atoms (Z, coordinates in the units the reference's
``bset.atoms[i].xyz`` holds, Angstrom), and shells (angular momentum, atom
index, primitive exponents, raw contraction coefficients).  The layout of every
record (labels, field widths, values per line, the cartesian reordering of d/f/g
shells and the density 2 sum_i n_i C_mi C_ni over the first nbf5 orbitals)
follows src/output.jl line by line, because the file is read by other programs.

Two properties of the reference are kept as they are: the coordinates of each
shell are printed without the Angstrom -> Bohr factor that the atomic
coordinates get (src/output.jl:186-197), and the shell-to-atom map is printed
from a floating-point array (same digits).  For cartesian g shells the
reference divides by ``np.sqrt(35)`` (src/output.jl:43-45), which Julia cannot
evaluate; the intended 1/sqrt(35) is used here.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

BOHR_PER_ANGSTROM = 1.88973  # the factor src/output.jl:155 uses


@dataclass
class Shell:
    l: int                      # angular momentum
    atom: int                   # 0-based atom index
    exponents: Sequence[float]
    coefficients: Sequence[float]  # raw contraction coefficients, as in the .gbs file


@dataclass
class BasisDescription:
    name: str                   # basis set name (the second title line)
    Z: Sequence[int]            # atomic numbers
    xyz: np.ndarray             # natoms x 3 atomic coordinates (Angstrom)
    shells: List[Shell] = field(default_factory=list)
    spherical: bool = True

    @property
    def natoms(self) -> int:
        return len(self.Z)

    @property
    def nshells(self) -> int:
        return len(self.shells)


def _cart_reorder(C: np.ndarray, shells: Sequence[Shell]) -> np.ndarray:
    """Rows of C in the fchk order of cartesian d, f and g functions, scaled to
    the normalisation the format expects (src/output.jl:8-50)."""
    Cnew = np.zeros_like(C)
    i = 0
    r3, r5, r15, r7, r35 = np.sqrt(3.0), np.sqrt(5.0), np.sqrt(15.0), np.sqrt(7.0), np.sqrt(35.0)
    # (destination offset, source offset, factor) per shell type, 1-based offsets as in the reference
    maps = {
        2: [(1, 1, 1), (2, 4, 1), (3, 6, 1), (4, 2, 1 / r3), (5, 3, 1 / r3), (6, 5, 1 / r3)],
        3: [(1, 1, 1), (2, 7, 1), (3, 10, 1), (4, 4, 1 / r5), (5, 2, 1 / r5), (6, 3, 1 / r5), (7, 6, 1 / r5),
            (8, 9, 1 / r5), (9, 8, 1 / r5), (10, 5, 1 / r15)],
        4: [(1, 1, 1), (2, 11, 1), (3, 15, 1), (4, 2, 1 / r7), (5, 3, 1 / r7), (6, 7, 1 / r7), (7, 12, 1 / r7),
            (8, 10, 1 / r7), (9, 14, 1 / r7), (10, 4, r3 / r35), (11, 6, r3 / r35), (12, 13, r3 / r35),
            (13, 5, 1 / r35), (14, 8, 1 / r35), (15, 9, 1 / r35)],
    }
    for sh in shells:
        ori = (sh.l + 1) * (sh.l + 2) // 2
        if sh.l in maps:
            for dst, src, f in maps[sh.l]:
                Cnew[i + dst - 1, :] = C[i + src - 1, :] * f
        elif sh.l > 4:
            warnings.warn("Warning: l>4, incorrect order in fchk")  # rows left at zero, as the reference does
        else:
            Cnew[i:i + ori, :] = C[i:i + ori, :]
        i += ori
    return Cnew


def _label(text: str, kind: str) -> str:
    return f"{text:<43s}{kind}"


def _rows(f, values, fmt: str, per_line: int, last: int) -> None:
    """Values `fmt`-formatted, a newline after every `per_line` and after item `last` (1-based)."""
    for i, v in enumerate(values, start=1):
        f.write(fmt % v)
        if i % per_line == 0 or i == last:
            f.write("\n")


def fchk(filename: str, p, basis: BasisDescription, jobtype: str, E_t: float, elag, n, C) -> str:
    """Write ``filename + ".fchk"`` as src/output.jl:1-283 does and return its path.

    p: the job's Param (ipnof, ista, nalpha, nbeta, nbf, nbf5); the multiplicity
    is nalpha - nbeta + 1 and the electron count nalpha + nbeta.  elag: the
    nbf x nbf Lagrangian (its diagonal is written as the orbital energies); n:
    the nbf5 occupations; C: the nbf x nbf orbitals.  The charge record is the
    reference's (electrons minus nuclear charge)."""
    C = np.asarray(C, dtype=np.float64)
    n = np.asarray(n, dtype=np.float64)
    nbf, nbf5 = p.nbf, p.nbf5
    Cnew = C.copy() if basis.spherical else _cart_reorder(C, basis.shells)
    natoms, nshells = basis.natoms, basis.nshells
    charge = -int(sum(basis.Z)) + p.nalpha + p.nbeta
    max_l = max((s.l for s in basis.shells), default=0)
    max_nprim = max((len(s.exponents) for s in basis.shells), default=0)
    nprim = sum(len(s.exponents) for s in basis.shells)
    path = filename + ".fchk"
    with open(path, "w") as f:
        f.write(f"{filename}\n")
        f.write(f"{jobtype} PNOF{p.ipnof}{'' if p.ista == 0 else 's'} {basis.name}\n")
        for text, v in (("Number of atoms", natoms), ("Charge", charge), ("Multiplicity", p.nalpha - p.nbeta + 1),
                        ("Number of electrons", p.nalpha + p.nbeta), ("Number of alpha electrons", p.nalpha),
                        ("Number of beta electrons", p.nbeta), ("Number of basis functions", nbf),
                        ("Number of independant functions", nbf5), ("Number of contracted shells", nshells),
                        ("Highest angular momentum", max_l), ("Largest degree of contraction", max_nprim),
                        ("Number of primitive shells", nprim)):
            f.write(_label(text, "I") + "           %6d\n" % v)
        f.write(_label("Atomic numbers", "I") + "   N=      %6d\n" % natoms)
        _rows(f, [int(z) for z in basis.Z], " %11d", 6, natoms)
        f.write(_label("Nuclear Charges", "R") + "   N=      %6d\n" % natoms)
        _rows(f, [float(z) for z in basis.Z], " %.8e", 6, natoms)
        xyz = np.asarray(basis.xyz, dtype=np.float64).reshape(natoms, 3)
        f.write(_label("Current cartesian coordinates", "R") + "   N=      %6d\n" % (natoms * 3))
        _rows(f, (xyz * BOHR_PER_ANGSTROM).reshape(-1), " % .8e", 5, natoms * 3)
        f.write(_label("Shell types", "I") + "   N=      %6d\n" % nshells)
        _rows(f, [-s.l if (basis.spherical and s.l > 1) else s.l for s in basis.shells], " %11d", 6, nshells)
        f.write(_label("Number of primitives per shell", "I") + "   N=      %6d\n" % nshells)
        _rows(f, [len(s.exponents) for s in basis.shells], " %11d", 6, nshells)
        f.write(_label("Shell to atom map", "I") + "   N=      %6d\n" % nshells)
        _rows(f, [s.atom + 1 for s in basis.shells], " %11d", 6, nshells)
        f.write(_label("Coordinates of each shell", "R") + "   N=      %6d\n" % (nshells * 3))
        _rows(f, np.array([xyz[s.atom] for s in basis.shells]).reshape(-1), " % 8e", 5, nshells * 3)
        f.write(_label("Total Energy", "R") + "     %.15e\n" % E_t)
        f.write(_label("Primitive exponents", "R") + "   N=      %6d\n" % nprim)
        _rows(f, [e for s in basis.shells for e in s.exponents], " % .8e", 5, nprim)
        f.write(_label("Contraction coefficients", "R") + "   N=      %6d\n" % nprim)
        _rows(f, [c for s in basis.shells for c in s.coefficients], " % .8e", 5, nprim)
        f.write(_label("Alpha Orbital Energies", "R") + "   N=      %6d\n" % nbf)
        _rows(f, np.diag(np.asarray(elag, dtype=np.float64))[:nbf], " % .8e", 5, nbf)
        f.write(_label("Alpha MO coefficients", "R") + "   N=      %6d\n" % (nbf * nbf))
        _rows(f, Cnew.reshape(-1, order="F"), " % .8e", 5, nbf * nbf)
        ntri = nbf * (nbf + 1) // 2
        f.write(_label("Total SCF Density", "R") + "   N=       %6d\n" % ntri)
        C5 = Cnew[:, :nbf5]
        DM = 2.0 * (C5 * n[None, :nbf5]) @ C5.T
        _rows(f, [DM[mu, nu] for mu in range(nbf) for nu in range(mu + 1)], " % .8e", 5, ntri)
        f.write(_label("Natural orbital occupancies", "R") + "   N=       %6d\n" % nbf5)
        _rows(f, n[:nbf5], " % .8e", 5, nbf5)
    return path


def save_restart(title: str, E: float, C, n, fmiug0=None) -> str:
    """The restart record of src/energy.jl:209-213 (``save(title.jld2, "E", E,
    "C", C, "n", n[, "fmiug0", fmiug0])``) with the same keys, written as
    ``title.npz`` (this build has no JLD2/HDF5 writer).  Returns the path."""
    arrays = {"E": np.float64(E), "C": np.asarray(C, dtype=np.float64), "n": np.asarray(n, dtype=np.float64)}
    if fmiug0 is not None:
        arrays["fmiug0"] = np.asarray(fmiug0, dtype=np.float64)
    path = title + ".npz"
    np.savez(path, **arrays)
    return path


def load_restart(path: str, p):
    """(E, C, gamma) from a restart record: the occupations are turned back into
    the optimiser's variables by n_to_gammas, as src/energy.jl:95-99 does when a
    run restarts from occupations."""
    from . import gnof
    with np.load(path) as z:
        E, C, n = float(z["E"]), np.asfortranarray(z["C"]), np.asarray(z["n"])
    return E, C, gnof.n_to_gammas(n, p)
