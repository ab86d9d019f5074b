"""Job parameters: the subset of DoNOF.jl's ``Param`` (src/param.jl:3-222)
that the RI hot path and its optimiser loops read, with the same names,
defaults and derived sizes."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Param:
    nbf: int
    nbfaux: int
    nalpha: int
    nbeta: int
    ncwo: int = -1          # -1: trunc(nvir / ndoc) as in src/param.jl:107-118
    no1: int = 0
    ipnof: int = 8
    ista: int = 0
    HighSpin: bool = False
    MSpin: int = 0
    occ_method: str = "Softmax"
    orb_method: str = "ADAM"
    alpha: float = 0.01
    maxloop: int = 10
    maxit: int = 1000
    threshgorb: float = 4e-3
    threshgocc: float = 1e-3
    threshen: float = 1e-4
    h_cut: float = 0.02 * math.sqrt(2.0)
    title: str = "donof"
    RI: bool = True
    # occoptr's conjugate gradient on the GPU (one CTA) instead of the host: measured
    # slower than the host solver at nbf5 = 20-198, so off by default
    occ_device: bool = False
    extra: dict = field(default_factory=dict)

    def __post_init__(self):
        if self.ncwo == -1:
            ndoc = self.nbeta - self.no1
            nvir = self.nbf - self.nalpha
            self.ncwo = (nvir // ndoc) if ndoc > 0 else 0

    @property
    def ndoc(self) -> int:
        return self.nbeta - self.no1

    @property
    def nsoc(self) -> int:
        return self.nalpha - self.nbeta

    @property
    def ndns(self) -> int:
        return self.ndoc + self.nsoc

    @property
    def nvir(self) -> int:
        return self.nbf - self.nalpha

    @property
    def nbf5(self) -> int:
        return self.no1 + self.ndoc * (1 + self.ncwo) + self.nsoc

    @property
    def no0(self) -> int:
        return self.nbf - self.nbf5

    @property
    def nv(self) -> int:
        return self.ncwo * self.ndoc

    @property
    def nvar(self) -> int:
        return self.nbf * (self.nbf - 1) // 2 - self.no0 * (self.no0 - 1) // 2

    def pair_table(self) -> np.ndarray:
        """(ndoc, ncwo) table of the 0-based weak orbitals coupled to each strong
        orbital: row g-1 is Julia's ``ll:ndoc:ul`` for strong orbital g."""
        g = np.arange(1, self.ndoc + 1)[:, None]
        return self.no1 + self.ndns + (self.ndoc - g) + self.ndoc * np.arange(self.ncwo)[None, :]

    def gamma_table(self) -> np.ndarray:
        """(ndoc, ncwo) table of the 0-based softmax parameters of each pair."""
        g = np.arange(1, self.ndoc + 1)[:, None]
        return (self.ndoc - g) + self.ndoc * np.arange(self.ncwo)[None, :]
