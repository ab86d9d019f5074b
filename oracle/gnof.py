"""numpy oracle for the GNOF functional and occupation layer -- TEST INFRASTRUCTURE ONLY.

A line-by-line restatement, with 0-based indices, of the reference's FP64 CPU
functions that feed and consume the RI hot path:

  ocupacion_softmax        src/pnof.jl:1122-1163  (incl. the ``n[i]`` quirk at :1152)
  ocupacion_trigonometric  src/pnof.jl:1047-1120
  CJCKD8 / PNOFi_selector  src/pnof.jl:488-601, 1-53 (diagonals zeroed at :49-50)
  der_CJCKD8 / der_PNOFi_selector  src/pnof.jl:603-793, 55-117
  calce / calcocce / calcoccg      src/pnof.jl:1273-1377
  computeE_elec (2 methods), computeLagrangeConvergency  src/utils.jl:191-236
  guess_gamma_softmax / _trigonometric  src/guess.jl:184-213
  n_to_gammas_softmax, order_occupations_softmax  src/utils.jl:539-561, 586-616

Only tests, the smoke check and the benchmark's CPU-baseline leg use this
module; the product never imports it.  Parity against reference-run outputs
is unpinned (no Julia here, no reference fixtures); it is pinned by the
identities the reference implies (see tests/test_oracle_identities.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Sizes:
    """Derived sizes of ``Param`` (src/param.jl:59-165) for a closed or open shell."""

    nbf: int
    nbeta: int
    nalpha: int
    ncwo: int
    naux: int = 0
    no1: int = 0
    ipnof: int = 8
    ista: int = 0
    HighSpin: bool = False
    MSpin: int = 0
    h_cut: float = 0.02 * math.sqrt(2.0)
    occ_method: str = "Softmax"

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


def _cwo(no1: int, ndns: int, ndoc: int, ncwo: int, i: int) -> np.ndarray:
    """0-based indices of the weak orbitals coupled to strong orbital i (1-based),
    i.e. Julia's ``ll:ndoc:ul`` with ll = no1+ndns+(ndoc-i)+1 (src/pnof.jl:1138-1139)."""
    ll = no1 + ndns + (ndoc - i)
    return ll + ndoc * np.arange(ncwo)


def ocupacion_softmax(gamma, no1, ndoc, nalpha, nv, nbf5, ndns, ncwo, HighSpin):
    """src/pnof.jl:1122-1163."""
    gamma = np.asarray(gamma, dtype=np.float64)
    n = np.zeros(nbf5)
    dn = np.zeros((nbf5, nv))
    n[:no1] = 1.0
    n[no1 + ndoc:no1 + ndns] = 1.0 if HighSpin else 0.5
    eg = np.exp(gamma)
    for i in range(1, ndoc + 1):
        cw = _cwo(no1, ndns, ndoc, ncwo, i)
        gi = (ndoc - i) + ndoc * np.arange(ncwo)
        den = 1.0 + eg[gi].sum()
        n[no1 + i - 1] = 1.0 / den
        n_pi = eg[gi] / den
        n[cw] = n_pi
        # quirk kept: Julia uses n[i], not n[no1+i] (identical for no1 = 0)
        dn[no1 + i - 1, gi] = -n[i - 1] * n_pi
        dn[np.ix_(cw, gi)] = -np.outer(n_pi, n_pi)
        dn[cw, gi] += n_pi
    return n, dn


def ocupacion_trigonometric(gamma, no1, ndoc, nalpha, nv, nbf5, ndns, ncwo, HighSpin):
    """src/pnof.jl:1047-1120."""
    gamma = np.asarray(gamma, dtype=np.float64)
    n = np.zeros(nbf5)
    dni = np.zeros(nbf5)
    n[:no1] = 1.0
    n[no1:no1 + ndoc] = 0.5 * (1.0 + np.cos(gamma[:ndoc]) ** 2)
    dni[no1:no1 + ndoc] = -0.5 * np.sin(2.0 * gamma[:ndoc])
    n[no1 + ndoc:no1 + ndns] = 1.0 if HighSpin else 0.5
    dn = np.zeros((nbf5, nv))
    h = 1.0 - n
    for i in range(1, ndoc + 1):
        cw = _cwo(no1, ndns, ndoc, ncwo, i)
        gl = ndoc + (ndoc - i) + ndoc * np.arange(ncwo - 1)  # ll_gamma:ndoc:ul_gamma
        gpi = gamma[gl]
        n_pi = np.full(ncwo, h[no1 + i - 1])
        for kw in range(ncwo - 1):
            n_pi[kw] *= math.sin(gpi[kw]) ** 2
            n_pi[kw + 1:] *= math.cos(gpi[kw]) ** 2
        n[cw] = n_pi
        dn[no1 + i - 1, i - 1] = dni[no1 + i - 1]
        col = np.full(ncwo, -dni[no1 + i - 1])
        for kw in range(ncwo - 1):
            col[kw] *= math.sin(gpi[kw]) ** 2
            col[kw + 1:] *= math.cos(gpi[kw]) ** 2
        dn[cw, i - 1] = col
        blk = dn[np.ix_(cw, gl)]  # copy; written back below
        for jw in range(ncwo - 1):
            blk[jw + 1:, jw] = n[no1 + i - 1] - 1.0
            for kw in range(jw):
                blk[jw + 1:, jw] *= math.cos(gpi[kw]) ** 2
            blk[jw + 1:, jw] *= math.sin(2.0 * gpi[jw])
            for kw in range(jw + 1, ncwo - 1):
                blk[kw, jw] *= math.sin(gpi[kw]) ** 2
                blk[kw + 1:, jw] *= math.cos(gpi[kw]) ** 2
        for jw in range(ncwo - 1):
            blk[jw, jw] = 1.0 - n[no1 + i - 1]
        for kw in range(ncwo - 1):
            blk[kw, kw] *= math.sin(2.0 * gpi[kw])
            for lw in range(kw + 1, ncwo - 1):
                blk[lw, lw] *= math.cos(gpi[kw]) ** 2
        dn[np.ix_(cw, gl)] = blk
    return n, dn


def ocupacion(gamma, p: Sizes):
    """src/pnof.jl:1024-1045 (Softmax / Trigonometric)."""
    args = (gamma, p.no1, p.ndoc, p.nalpha, p.nv, p.nbf5, p.ndns, p.ncwo, p.HighSpin)
    if p.occ_method == "Softmax":
        return ocupacion_softmax(*args)
    if p.occ_method == "Trigonometric":
        return ocupacion_trigonometric(*args)
    raise ValueError(f"occ_method {p.occ_method!r} not supported")


def _fi(n, ista):
    fi = n * (1.0 - n)
    fi[fi <= 0] = 0.0
    if ista in (0, 1, 5):
        return np.sqrt(fi)
    if ista == 2:
        return 0.9 * np.sqrt(fi)
    if ista == 3:
        alpha = 0.55
        aa = (2.0 ** (2.0 * alpha - 1.0)) ** (1.0 / alpha)
        return (aa * fi) ** alpha
    if ista == 4:
        return np.sqrt(fi) * np.exp(-(n - 0.5) ** 2)
    raise ValueError(f"ista {ista}")


def CJCKD8(n, no1, ndoc, nsoc, nbeta, nalpha, ndns, ncwo, MSpin, h_cut, ista):
    """GNOF coefficients, src/pnof.jl:488-601."""
    n = np.asarray(n, dtype=np.float64)
    nbf5 = n.shape[0]
    n_d = np.zeros(nbf5)
    c = 0.8 if ista == 5 else 1.0
    for i in range(1, ndoc + 1):
        idx = no1 + i - 1
        cw = _cwo(no1, ndns, ndoc, ncwo, i)
        coc = (1.0 - n[idx]) / h_cut
        F = c * math.exp(-coc * coc)
        n_d[idx] = n[idx] * F
        n_d[cw] = n[cw] * F
    n_d12 = np.sqrt(n_d)
    fi = _fi(n, ista)
    beta = slice(no1, nbeta)
    alpha = slice(nbeta, nalpha)
    cwo = slice(nalpha, nbf5)
    cj12 = 2.0 * np.outer(n, n)
    if ista == 0:
        ck12 = np.outer(n, n)
        ck12[beta, cwo] += np.outer(fi[beta], fi[cwo])
        ck12[cwo, beta] += np.outer(fi[cwo], fi[beta])
        ck12[cwo, cwo] += np.outer(fi[cwo], fi[cwo])
        if nsoc > 0:
            ck12[beta, alpha] += (0.5 * fi[beta] * 0.5)[:, None]
            ck12[alpha, beta] += (0.5 * 0.5 * fi[beta])[None, :]
            ck12[alpha, cwo] += (0.5 * fi[cwo])[None, :]
            ck12[cwo, alpha] += (fi[cwo] * 0.5)[:, None]
        if nsoc > 1:
            ck12[alpha, alpha] = 0.5
    else:
        ck12 = np.outer(n, n) + np.outer(fi, fi)
    ck12[beta, cwo] += np.outer(n_d12[beta], n_d12[cwo]) - np.outer(n_d[beta], n_d[cwo])
    ck12[cwo, beta] += np.outer(n_d12[cwo], n_d12[beta]) - np.outer(n_d[cwo], n_d[beta])
    ck12[cwo, cwo] += -np.outer(n_d12[cwo], n_d12[cwo]) - np.outer(n_d[cwo], n_d[cwo])
    for l in range(1, ndoc + 1):
        ldx = no1 + l - 1
        cw = _cwo(no1, ndns, ndoc, ncwo, l)
        cj12[ldx, cw] = 0.0
        cj12[cw, ldx] = 0.0
        cj12[np.ix_(cw, cw)] = 0.0
        ck12[ldx, cw] = np.sqrt(n[ldx] * n[cw])
        ck12[cw, ldx] = np.sqrt(n[ldx] * n[cw])
        ck12[np.ix_(cw, cw)] = -np.sqrt(np.outer(n[cw], n[cw]))
    return cj12, ck12


def PNOFi_selector(n, p: Sizes):
    """src/pnof.jl:1-53 for ipnof = 8 (GNOF), diagonals zeroed (:49-50)."""
    if p.ipnof != 8:
        raise ValueError("only GNOF (ipnof = 8) is on this path")
    cj12, ck12 = CJCKD8(n, p.no1, p.ndoc, p.nsoc, p.nbeta, p.nalpha, p.ndns, p.ncwo,
                        p.MSpin, p.h_cut, p.ista)
    np.fill_diagonal(cj12, 0.0)
    np.fill_diagonal(ck12, 0.0)
    return cj12, ck12


def der_CJCKD8(n, dn_dgamma, no1, ndoc, nalpha, nbeta, nv, nbf5, ndns, ncwo, MSpin,
               nsoc, h_cut, ista):
    """src/pnof.jl:603-793."""
    n = np.asarray(n, dtype=np.float64)
    nbf5 = n.shape[0]
    n_d = np.zeros(nbf5)
    dnd = np.zeros((nbf5, nv))
    c = 0.8 if ista == 5 else 1.0
    for i in range(1, ndoc + 1):
        idx = no1 + i - 1
        cw = _cwo(no1, ndns, ndoc, ncwo, i)
        coc = (1.0 - n[idx]) / h_cut
        F = c * math.exp(-coc * coc)
        n_d[idx] = n[idx] * F
        n_d[cw] = n[cw] * F
        dnd[idx, :] = F * dn_dgamma[idx, :] * (1.0 - n[idx] * (-2.0 * coc / h_cut))
        dnd[cw, :] = F * dn_dgamma[cw, :]
        dnd[cw, :] += F * (2.0 * coc / h_cut) * np.outer(n[cw], dn_dgamma[idx, :])
    n_d12 = np.sqrt(n_d)
    dnd12 = 0.5 * dnd / np.maximum(n_d12, 1e-15)[:, None]
    fi = n * (1.0 - n)
    fi[fi <= 0] = 0.0
    dfi = np.zeros((nbf5, nv))
    if ista in (0, 1, 5):
        fi = np.sqrt(fi)
        for i in range(no1, nbf5):
            a = max(fi[i], 1e-15)
            dfi[i, :] = 1.0 / (2.0 * a) * (1.0 - 2.0 * n[i]) * dn_dgamma[i, :]
    elif ista == 2:
        alpha_ = 0.9
        fi = alpha_ * np.sqrt(fi)
        for i in range(no1, nbf5):
            a = max(fi[i], 1e-15)
            dfi[i, :] = alpha_ ** 2 / (2.0 * a) * (1.0 - 2.0 * n[i]) * dn_dgamma[i, :]
    elif ista == 3:
        alpha_ = 0.55
        aa = (2.0 ** (2.0 * alpha_ - 1.0)) ** (1.0 / alpha_)
        fi = (aa * fi) ** alpha_
        for i in range(no1, nbf5):
            a = max(aa * n[i] * (1.0 - n[i]), 1e-15)
            dfi[i, :] = alpha_ * a ** (alpha_ - 1.0) * aa * (1.0 - 2.0 * n[i]) * dn_dgamma[i, :]
    elif ista == 4:
        fi = np.sqrt(fi)
        for i in range(no1, nbf5):
            a = max(fi[i], 1e-15)
            e = math.exp(-(n[i] - 0.5) ** 2)
            dfi[i, :] = 1.0 / (2.0 * a) * (1.0 - 2.0 * n[i]) * dn_dgamma[i, :] * e
            dfi[i, :] += -fi[i] * 2.0 * (n[i] - 0.5) * dn_dgamma[i, :] * e
        fi = fi * np.exp(-(n - 0.5) ** 2)
    beta = slice(no1, nbeta)
    alpha = slice(nbeta, nalpha)
    cwo = slice(nalpha, nbf5)
    Dcj = 2.0 * np.einsum("ik,j->ijk", dn_dgamma, n)
    if ista == 0:
        Dck = np.einsum("ik,j->ijk", dn_dgamma, n)
        Dck[beta, cwo, :] += np.einsum("ik,j->ijk", dfi[beta], fi[cwo])
        Dck[cwo, beta, :] += np.einsum("j,ik->ijk", fi[beta], dfi[cwo])
        Dck[cwo, cwo, :] += np.einsum("j,ik->ijk", fi[cwo], dfi[cwo])
        if nsoc > 0:
            Dck[beta, alpha, :] += (0.5 * dfi[beta] * 0.5)[:, None, :]
            Dck[cwo, alpha, :] += (dfi[cwo] * 0.5)[:, None, :]
        if nsoc > 1:
            Dck[alpha, alpha, :] = 0.0
    else:
        Dck = np.einsum("ik,j->ijk", dn_dgamma, n) + np.einsum("ik,j->ijk", dfi, fi)
        if nsoc > 1:
            Dck[alpha, alpha, :] = 0.0
    Dck[beta, cwo, :] += (np.einsum("ik,j->ijk", dnd12[beta], n_d12[cwo])
                          - np.einsum("ik,j->ijk", dnd[beta], n_d[cwo]))
    Dck[cwo, beta, :] += (np.einsum("j,ik->ijk", n_d12[beta], dnd12[cwo])
                          - np.einsum("j,ik->ijk", n_d[beta], dnd[cwo]))
    Dck[cwo, cwo, :] += (-np.einsum("j,ik->ijk", n_d12[cwo], dnd12[cwo])
                         - np.einsum("j,ik->ijk", n_d[cwo], dnd[cwo]))
    for l in range(1, ndoc + 1):
        ldx = no1 + l - 1
        cw = _cwo(no1, ndns, ndoc, ncwo, l)
        Dcj[ldx, cw, :] = 0.0
        Dcj[cw, ldx, :] = 0.0
        Dcj[np.ix_(cw, cw, np.arange(nv))] = 0.0
        a = max(n[ldx], 1e-15)
        bb = n[cw].copy()
        bb[bb < 1e-15] = 1e-15
        Dck[ldx, cw, :] = 0.5 / math.sqrt(a) * np.outer(np.sqrt(n[cw]), dn_dgamma[ldx, :])
        Dck[cw, ldx, :] = 0.5 / np.sqrt(bb)[:, None] * dn_dgamma[cw, :] * math.sqrt(n[ldx])
        Dck[np.ix_(cw, cw, np.arange(nv))] = (
            -0.5 / np.sqrt(bb)[:, None, None] * dn_dgamma[cw, None, :] * np.sqrt(n[cw])[None, :, None])
    return Dcj, Dck


def der_PNOFi_selector(n, dn_dgamma, p: Sizes):
    """src/pnof.jl:55-117 for ipnof = 8, diagonals zeroed (:109-114)."""
    Dcj, Dck = der_CJCKD8(n, dn_dgamma, p.no1, p.ndoc, p.nalpha, p.nbeta, p.nv, p.nbf5,
                          p.ndns, p.ncwo, p.MSpin, p.nsoc, p.h_cut, p.ista)
    d = np.arange(p.nbf5)
    Dcj[d, d, :] = 0.0
    Dck[d, d, :] = 0.0
    return Dcj, Dck


def calce(n, cj12, ck12, J_MO, K_MO, H_core, p: Sizes) -> float:
    """src/pnof.jl:1273-1300."""
    nb, na, n5 = p.nbeta, p.nalpha, p.nbf5
    dJ = np.diag(J_MO)
    E = np.sum(n[:nb] * (2.0 * H_core[:nb] + dJ[:nb]))
    if p.nsoc > 0:
        E += np.sum(n[nb:na] * 2.0 * H_core[nb:na])
    E += np.sum(n[na:n5] * (2.0 * H_core[na:n5] + dJ[na:n5]))
    E += np.sum(cj12 * J_MO.T)
    E += -np.sum(ck12 * K_MO.T)
    return float(E)


def calcocce(gamma, J_MO, K_MO, H_core, p: Sizes) -> float:
    """src/pnof.jl:1302-1322."""
    n, _ = ocupacion(gamma, p)
    cj12, ck12 = PNOFi_selector(n, p)
    return calce(n, cj12, ck12, J_MO, K_MO, H_core, p)


def calcoccg(gamma, J_MO, K_MO, H_core, p: Sizes) -> np.ndarray:
    """src/pnof.jl:1324-1377."""
    n, dn = ocupacion(gamma, p)
    Dcj, Dck = der_PNOFi_selector(n, dn, p)
    b = slice(p.no1, p.nbeta)
    a = slice(p.nalpha, p.nbf5)
    dJ = np.diag(J_MO)
    g = np.zeros(p.nv)
    g += dn[b].T @ (2.0 * H_core[b])
    g += dn[b].T @ dJ[b]
    g += dn[a].T @ (2.0 * H_core[a])
    g += dn[a].T @ dJ[a]
    g += 2.0 * np.einsum("ijk,ji->k", Dcj[b], J_MO[:, b])
    g += 2.0 * np.einsum("ijk,ji->k", Dcj[a], J_MO[:, a])
    g += -2.0 * np.einsum("ijk,ji->k", Dck[b], K_MO[:, b])
    g += -2.0 * np.einsum("ijk,ji->k", Dck[a], K_MO[:, a])
    return g


def computeE_elec_Hmat(Hmat, n, elag, p: Sizes) -> float:
    """computeE_elec(Hmat, n, elag, p), src/utils.jl:216-227."""
    k = p.nbf5
    return float(np.trace(elag[:k, :k]) + np.sum(n[:k] * np.diag(Hmat[:k, :k])))


def computeE_elec_HC(H, C, n, elag, p: Sizes) -> float:
    """computeE_elec(H, C, n, elag, p), src/utils.jl:191-214."""
    E = float(np.trace(elag[:p.nbf5, :p.nbf5]))
    hdiag = np.einsum("mi,mn,ni->i", C, H, C)
    E += float(np.sum(n[:p.nbeta] * hdiag[:p.nbeta]))
    if not p.HighSpin:
        E += float(np.sum(n[p.nbeta:p.nalpha] * hdiag[p.nbeta:p.nalpha]))
    else:
        E += float(np.sum(0.5 * hdiag[p.nbeta:p.nalpha]))
    E += float(np.sum(n[p.nalpha:p.nbf5] * hdiag[p.nalpha:p.nbf5]))
    return E


def computeLagrangeConvergency(elag):
    """src/utils.jl:229-236."""
    d = np.abs(elag - elag.T)
    return float(d.sum()), float(d.max())


def pack_orbital_gradient(elag, nbf5: int) -> np.ndarray:
    """grad = 4 elag - 4 elag^T packed row-wise over i < nbf5, j > i
    (src/pnof.jl:1395-1403, src/minimization.jl:365-373)."""
    nbf = elag.shape[0]
    g = 4.0 * elag - 4.0 * elag.T
    return np.concatenate([g[i, i + 1:nbf] for i in range(nbf5)])


def guess_gamma_softmax(ndoc: int, ncwo: int) -> np.ndarray:
    """src/guess.jl:200-213."""
    nv = ncwo * ndoc
    g = np.zeros(nv)
    for i in range(1, ndoc + 1):
        idx = (ndoc - i) + ndoc * np.arange(ncwo)
        g[idx] = math.log(max(0.001 / ncwo, 1e-16)) - math.log(0.999)
    return g


def guess_gamma_trigonometric(ndoc: int, ncwo: int) -> np.ndarray:
    """src/guess.jl:184-198."""
    nv = ncwo * ndoc
    g = np.zeros(nv)
    for i in range(1, ndoc + 1):
        g[i - 1] = math.acos(math.sqrt(2.0 * 0.999 - 1.0))
        ll = ndoc + (ndoc - i)
        for j in range(1, ncwo):
            g[ll + ndoc * (j - 1)] = math.asin(math.sqrt(1.0 / (ncwo - j + 1)))
    return g


def n_to_gammas_softmax(n, p: Sizes) -> np.ndarray:
    """src/utils.jl:539-561 (line by line, 0-based)."""
    gamma = np.zeros(p.nv)
    for i in range(1, p.ndoc + 1):
        n_pi = _cwo(p.no1, p.ndns, p.ndoc, p.ncwo, i)            # ll:ndoc:ul
        gamma_pi = (p.ndoc - i) + p.ndoc * np.arange(p.ncwo)    # llg:ndoc:ulg
        for j in range(p.ncwo):
            gamma[gamma_pi[j]] = math.log(max(n[n_pi[j]], 1e-16)) - math.log(n[i - 1])
    return gamma


def n_to_gammas_trigonometric(n, p: Sizes) -> np.ndarray:
    """src/utils.jl:563-584 (line by line, 0-based)."""
    gamma = np.zeros(p.nv)
    for i in range(1, p.ndoc + 1):
        idx = p.no1 + i - 1
        gamma[i - 1] = math.acos(math.sqrt(2.0 * n[idx] - 1.0))
        prefactor = max(1 - n[idx], 1e-14)
        n_pi = _cwo(p.no1, p.ndns, p.ndoc, p.ncwo, i)
        gamma_pi = p.ndoc + (p.ndoc - i) + p.ndoc * np.arange(p.ncwo - 1)
        for j in range(p.ncwo - 1):
            gamma[gamma_pi[j]] = math.asin(math.sqrt(n[n_pi[j]] / prefactor))
            prefactor = prefactor * math.cos(gamma[gamma_pi[j]]) ** 2
    return gamma


def order_occupations_softmax(old_C, old_gamma, p: Sizes):
    """src/utils.jl:586-616."""
    C = old_C.copy()
    gamma = old_gamma.copy()
    if np.any(gamma > 0):
        for i in range(1, p.ndoc + 1):
            cw = _cwo(p.no1, p.ndns, p.ndoc, p.ncwo, i)
            C_tmp = np.concatenate([old_C[:, [p.no1 + i - 1]], old_C[:, cw]], axis=1)
            gx = (p.ndoc - i) + p.ndoc * np.arange(p.ncwo)
            g_tmp = np.concatenate([[0.0], gamma[gx]])
            # Julia: sortperm(g)[end:-1:1] -- a stable ascending sort, reversed
            sort_idx = np.argsort(g_tmp, kind="stable")[::-1]
            g_tmp = g_tmp[sort_idx] - g_tmp.max()
            C_tmp = C_tmp[:, sort_idx]
            gamma[gx] = g_tmp[1:]
            C[:, p.no1 + i - 1] = C_tmp[:, 0]
            C[:, cw] = C_tmp[:, 1:]
    return C, gamma
