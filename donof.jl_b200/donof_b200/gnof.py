"""Host-side GNOF functional layer (FP64): occupation parametrisations, the
coupling coefficients cj12/ck12 and their gamma-derivatives, and the
occupation energy / gradient from cached J_MO, K_MO, H_core.

These are the O(nbf5^2 * nv) host functions that feed and consume the device
hot path; in DoNOF.jl they run on the host too, even with the GPU extension
loaded.  Reference definitions:
  ocupacion / _softmax / _trigonometric   src/pnof.jl:1024-1163
  PNOFi_selector + CJCKD8                 src/pnof.jl:1-53, 488-601
  der_PNOFi_selector + der_CJCKD8         src/pnof.jl:55-117, 603-793
  calce / calcocce / calcoccg             src/pnof.jl:1273-1377
  guess_gamma_softmax / _trigonometric    src/guess.jl:184-213
  order_occupations_softmax               src/utils.jl:586-616
"""
from __future__ import annotations

import math

import numpy as np

from .param import Param


def occupations(gamma, p: Param):
    """n (nbf5) and dn/dgamma (nbf5 x nv) for p.occ_method."""
    if p.occ_method == "Softmax":
        return _softmax(np.asarray(gamma, float), p)
    if p.occ_method == "Trigonometric":
        return _trigonometric(np.asarray(gamma, float), p)
    raise ValueError(f"occupation method {p.occ_method!r} is not supported")


ocupacion = occupations


def _fixed(p: Param) -> np.ndarray:
    n = np.zeros(p.nbf5)
    n[: p.no1] = 1.0
    n[p.no1 + p.ndoc: p.no1 + p.ndns] = 1.0 if p.HighSpin else 0.5
    return n


def _softmax(gamma, p: Param):
    n = _fixed(p)
    dn = np.zeros((p.nbf5, p.nv))
    P, G = p.pair_table(), p.gamma_table()
    e = np.exp(gamma[G])                      # (ndoc, ncwo)
    inv = 1.0 / (1.0 + e.sum(axis=1))         # strong occupations
    strong = p.no1 + np.arange(p.ndoc)
    n[strong] = inv
    w = e * inv[:, None]                      # weak occupations of each pair
    n[P] = w
    # src/pnof.jl:1152 multiplies by n[i] (1-based i, the pair index), kept as is
    dn[strong[:, None], G] = -n[: p.ndoc][:, None] * w
    eye = np.eye(p.ncwo)
    dn[P[:, :, None], G[:, None, :]] = eye[None] * w[:, :, None] - w[:, :, None] * w[:, None, :]
    return n, dn


def _trigonometric(gamma, p: Param):
    n = _fixed(p)
    nd, nc = p.ndoc, p.ncwo
    strong = p.no1 + np.arange(nd)
    n[strong] = 0.5 * (1.0 + np.cos(gamma[:nd]) ** 2)
    dstrong = -0.5 * np.sin(2.0 * gamma[:nd])
    dn = np.zeros((p.nbf5, p.nv))
    P = p.pair_table()
    for g in range(nd):
        cols = nd + (nd - (g + 1)) + nd * np.arange(nc - 1)   # angles of the weak orbitals
        th = gamma[cols]
        s2, c2 = np.sin(th) ** 2, np.cos(th) ** 2
        # n_w = h * prod_{k<w} cos^2 * (sin^2 of own angle if w < nc-1)
        h = 1.0 - n[strong[g]]
        fac = np.ones(nc)
        for k in range(nc - 1):
            fac[k] *= s2[k]
            fac[k + 1:] *= c2[k]
        n[P[g]] = h * fac
        dn[strong[g], g] = dstrong[g]
        dn[P[g], g] = -dstrong[g] * fac
        blk = np.zeros((nc, nc - 1))
        for j in range(nc - 1):
            col = np.full(nc, n[strong[g]] - 1.0)
            col[: j + 1] = 0.0
            for k in range(j):
                col[j + 1:] *= c2[k]
            col[j + 1:] *= math.sin(2.0 * th[j])
            for k in range(j + 1, nc - 1):
                col[k] *= s2[k]
                col[k + 1:] *= c2[k]
            blk[:, j] = col
        for j in range(nc - 1):
            blk[j, j] = 1.0 - n[strong[g]]
        for k in range(nc - 1):
            blk[k, k] *= math.sin(2.0 * th[k])
            for l in range(k + 1, nc - 1):
                blk[l, l] *= c2[k]
        dn[np.ix_(P[g], cols)] = blk
    return n, dn


def _phi(n, ista):
    f = np.clip(n * (1.0 - n), 0.0, None)
    if ista in (0, 1, 5):
        return np.sqrt(f)
    if ista == 2:
        return 0.9 * np.sqrt(f)
    if ista == 3:
        a = 0.55
        aa = (2.0 ** (2.0 * a - 1.0)) ** (1.0 / a)
        return (aa * f) ** a
    if ista == 4:
        return np.sqrt(f) * np.exp(-(n - 0.5) ** 2)
    raise ValueError(f"ista = {ista} is not a GNOF variant")


def _dynamic(n, p: Param):
    """n_d = n * c * exp(-((1 - n_g)/h_cut)^2) on each pair (0 elsewhere) and the
    per-pair factors needed by the derivative."""
    c = 0.8 if p.ista == 5 else 1.0
    strong = p.no1 + np.arange(p.ndoc)
    P = p.pair_table()
    coc = (1.0 - n[strong]) / p.h_cut
    F = c * np.exp(-coc * coc)
    nd = np.zeros_like(n)
    nd[strong] = n[strong] * F
    nd[P] = n[P] * F[:, None]
    return nd, F, coc


def _pairs(p: Param):
    """Index arrays of the pairs: S (ndoc, 1) strong orbitals, W (ndoc, ncwo) their weak ones."""
    return (p.no1 + np.arange(p.ndoc))[:, None], p.pair_table()


def coupling(n, p: Param):
    """cj12, ck12 of GNOF (ipnof = 8) with zeroed diagonals (PNOFi_selector)."""
    if p.ipnof != 8:
        raise ValueError("only GNOF (ipnof = 8) is on this path")
    n = np.asarray(n, float)
    nd, _, _ = _dynamic(n, p)
    nd12 = np.sqrt(nd)
    fi = _phi(n, p.ista)
    be, al, cw = slice(p.no1, p.nbeta), slice(p.nbeta, p.nalpha), slice(p.nalpha, p.nbf5)
    cj = 2.0 * np.outer(n, n)
    if p.ista == 0:
        ck = np.outer(n, n)
        ck[be, cw] += np.outer(fi[be], fi[cw])
        ck[cw, be] += np.outer(fi[cw], fi[be])
        ck[cw, cw] += np.outer(fi[cw], fi[cw])
        if p.nsoc > 0:
            ck[be, al] += 0.25 * fi[be][:, None]
            ck[al, be] += 0.25 * fi[be][None, :]
            ck[al, cw] += 0.5 * fi[cw][None, :]
            ck[cw, al] += 0.5 * fi[cw][:, None]
        if p.nsoc > 1:
            ck[al, al] = 0.5
    else:
        ck = np.outer(n, n) + np.outer(fi, fi)
    ck[be, cw] += np.outer(nd12[be], nd12[cw]) - np.outer(nd[be], nd[cw])
    ck[cw, be] += np.outer(nd12[cw], nd12[be]) - np.outer(nd[cw], nd[be])
    ck[cw, cw] -= np.outer(nd12[cw], nd12[cw]) + np.outer(nd[cw], nd[cw])
    S, W = _pairs(p)  # every pair (strong s, weak ws) at once
    cj[S, W] = 0.0
    cj[W, S] = 0.0
    cj[W[:, :, None], W[:, None, :]] = 0.0
    r = np.sqrt(n[S] * n[W])
    ck[S, W] = r
    ck[W, S] = r
    sw = np.sqrt(n[W])
    ck[W[:, :, None], W[:, None, :]] = -(sw[:, :, None] * sw[:, None, :])
    np.fill_diagonal(cj, 0.0)
    np.fill_diagonal(ck, 0.0)
    return cj, ck


PNOFi_selector = coupling


def coupling_derivatives(n, dn, p: Param):
    """Dcj12r, Dck12r (nbf5 x nbf5 x nv) with zeroed diagonals (der_PNOFi_selector)."""
    if p.ipnof != 8:
        raise ValueError("only GNOF (ipnof = 8) is on this path")
    n = np.asarray(n, float)
    nv = p.nv
    nd, F, coc = _dynamic(n, p)
    strong = p.no1 + np.arange(p.ndoc)
    P = p.pair_table()
    dnd = np.zeros((p.nbf5, nv))
    for g in range(p.ndoc):
        s, ws = strong[g], P[g]
        k = 2.0 * coc[g] / p.h_cut
        dnd[s] = F[g] * dn[s] * (1.0 + n[s] * k)
        dnd[ws] = F[g] * dn[ws] + F[g] * k * np.outer(n[ws], dn[s])
    nd12 = np.sqrt(nd)
    dnd12 = 0.5 * dnd / np.maximum(nd12, 1e-15)[:, None]
    f = np.clip(n * (1.0 - n), 0.0, None)
    dfi = np.zeros((p.nbf5, nv))
    act = slice(p.no1, p.nbf5)
    if p.ista in (0, 1, 5, 2, 4):
        fi = np.sqrt(f) * (0.9 if p.ista == 2 else 1.0)
        a = np.maximum(fi[act], 1e-15)
        scale = 0.81 if p.ista == 2 else 1.0
        dfi[act] = (scale / (2.0 * a) * (1.0 - 2.0 * n[act]))[:, None] * dn[act]
        if p.ista == 4:
            e = np.exp(-(n[act] - 0.5) ** 2)
            dfi[act] = dfi[act] * e[:, None] - (fi[act] * 2.0 * (n[act] - 0.5) * e)[:, None] * dn[act]
            fi = fi * np.exp(-(n - 0.5) ** 2)
    elif p.ista == 3:
        al_ = 0.55
        aa = (2.0 ** (2.0 * al_ - 1.0)) ** (1.0 / al_)
        fi = (aa * f) ** al_
        a = np.maximum(aa * n[act] * (1.0 - n[act]), 1e-15)
        dfi[act] = (al_ * a ** (al_ - 1.0) * aa * (1.0 - 2.0 * n[act]))[:, None] * dn[act]
    else:
        raise ValueError(f"ista = {p.ista} is not a GNOF variant")
    be, al, cw = slice(p.no1, p.nbeta), slice(p.nbeta, p.nalpha), slice(p.nalpha, p.nbf5)
    Dcj = 2.0 * dn[:, None, :] * n[None, :, None]
    Dck = dn[:, None, :] * n[None, :, None]
    if p.ista == 0:
        Dck[be, cw] += dfi[be][:, None, :] * fi[cw][None, :, None]
        Dck[cw, be] += dfi[cw][:, None, :] * fi[be][None, :, None]
        Dck[cw, cw] += dfi[cw][:, None, :] * fi[cw][None, :, None]
        if p.nsoc > 0:
            Dck[be, al] += 0.25 * dfi[be][:, None, :]
            Dck[cw, al] += 0.5 * dfi[cw][:, None, :]
    else:
        Dck += dfi[:, None, :] * fi[None, :, None]
    if p.nsoc > 1:
        Dck[al, al] = 0.0
    Dck[be, cw] += dnd12[be][:, None, :] * nd12[cw][None, :, None] - dnd[be][:, None, :] * nd[cw][None, :, None]
    Dck[cw, be] += dnd12[cw][:, None, :] * nd12[be][None, :, None] - dnd[cw][:, None, :] * nd[be][None, :, None]
    Dck[cw, cw] -= dnd12[cw][:, None, :] * nd12[cw][None, :, None] + dnd[cw][:, None, :] * nd[cw][None, :, None]
    for g in range(p.ndoc):
        s, ws = strong[g], P[g]
        Dcj[s, ws] = 0.0
        Dcj[ws, s] = 0.0
        Dcj[np.ix_(ws, ws)] = 0.0
        a = max(n[s], 1e-15)
        b = np.maximum(n[ws], 1e-15)
        Dck[s, ws] = 0.5 / math.sqrt(a) * np.sqrt(n[ws])[:, None] * dn[s][None, :]
        Dck[ws, s] = (0.5 / np.sqrt(b) * math.sqrt(n[s]))[:, None] * dn[ws]
        Dck[np.ix_(ws, ws)] = -0.5 * (dn[ws] / np.sqrt(b)[:, None])[:, None, :] * np.sqrt(n[ws])[None, :, None]
    d = np.arange(p.nbf5)
    Dcj[d, d] = 0.0
    Dck[d, d] = 0.0
    return Dcj, Dck


der_PNOFi_selector = coupling_derivatives


def _derivative_factors(n, dn, p: Param):
    """The derivatives of coupling_derivatives as sums of separable terms,
        Dcj[i, j, :] = Mcj[i, j] dn[i, :],   Dck[i, j, :] = sum_t Mck[t][i, j] A[t][i, :],
    with the per-row derivative arrays A = (dn, dfi, dnd12, dnd) (nbf5 x nv) and
    the same blocks, masks and overwrites as coupling_derivatives (and
    der_CJCKD8, src/pnof.jl:603-793) without the nv axis."""
    nd, F, coc = _dynamic(n, p)
    strong = p.no1 + np.arange(p.ndoc)
    P = p.pair_table()
    dnd = np.zeros((p.nbf5, p.nv))
    for g in range(p.ndoc):
        s, ws = strong[g], P[g]
        k = 2.0 * coc[g] / p.h_cut
        dnd[s] = F[g] * dn[s] * (1.0 + n[s] * k)
        dnd[ws] = F[g] * dn[ws] + F[g] * k * np.outer(n[ws], dn[s])
    nd12 = np.sqrt(nd)
    dnd12 = 0.5 * dnd / np.maximum(nd12, 1e-15)[:, None]
    f = np.clip(n * (1.0 - n), 0.0, None)
    dfi = np.zeros((p.nbf5, p.nv))
    act = slice(p.no1, p.nbf5)
    if p.ista in (0, 1, 5, 2, 4):
        fi = np.sqrt(f) * (0.9 if p.ista == 2 else 1.0)
        a = np.maximum(fi[act], 1e-15)
        scale = 0.81 if p.ista == 2 else 1.0
        dfi[act] = (scale / (2.0 * a) * (1.0 - 2.0 * n[act]))[:, None] * dn[act]
        if p.ista == 4:
            e = np.exp(-(n[act] - 0.5) ** 2)
            dfi[act] = dfi[act] * e[:, None] - (fi[act] * 2.0 * (n[act] - 0.5) * e)[:, None] * dn[act]
            fi = fi * np.exp(-(n - 0.5) ** 2)
    elif p.ista == 3:
        al_ = 0.55
        aa = (2.0 ** (2.0 * al_ - 1.0)) ** (1.0 / al_)
        fi = (aa * f) ** al_
        a = np.maximum(aa * n[act] * (1.0 - n[act]), 1e-15)
        dfi[act] = (al_ * a ** (al_ - 1.0) * aa * (1.0 - 2.0 * n[act]))[:, None] * dn[act]
    else:
        raise ValueError(f"ista = {p.ista} is not a GNOF variant")
    N = p.nbf5
    be, al, cw = slice(p.no1, p.nbeta), slice(p.nbeta, p.nalpha), slice(p.nalpha, p.nbf5)
    Mcj = np.tile(2.0 * n, (N, 1))
    Mdn = np.tile(n, (N, 1))
    Mdfi = np.zeros((N, N))
    Mdnd12 = np.zeros((N, N))
    Mdnd = np.zeros((N, N))
    if p.ista == 0:
        Mdfi[be, cw] += fi[cw][None, :]
        Mdfi[cw, be] += fi[be][None, :]
        Mdfi[cw, cw] += fi[cw][None, :]
        if p.nsoc > 0:
            Mdfi[be, al] += 0.25
            Mdfi[cw, al] += 0.5
    else:
        Mdfi += fi[None, :]
    Ms = (Mdn, Mdfi, Mdnd12, Mdnd)
    if p.nsoc > 1:
        for M in Ms:
            M[al, al] = 0.0
    Mdnd12[be, cw] += nd12[cw][None, :]
    Mdnd[be, cw] -= nd[cw][None, :]
    Mdnd12[cw, be] += nd12[be][None, :]
    Mdnd[cw, be] -= nd[be][None, :]
    Mdnd12[cw, cw] -= nd12[cw][None, :]
    Mdnd[cw, cw] -= nd[cw][None, :]
    S, W = _pairs(p)
    WW = (W[:, :, None], W[:, None, :])
    Mcj[S, W] = 0.0
    Mcj[W, S] = 0.0
    Mcj[WW] = 0.0
    for M in Ms:
        M[S, W] = 0.0
        M[W, S] = 0.0
        M[WW] = 0.0
    sa = np.sqrt(np.maximum(n[S], 1e-15))  # (ndoc, 1)
    sb = np.sqrt(np.maximum(n[W], 1e-15))  # (ndoc, ncwo)
    Mdn[S, W] = 0.5 / sa * np.sqrt(n[W])
    Mdn[W, S] = 0.5 / sb * np.sqrt(n[S])
    Mdn[WW] = -0.5 * (1.0 / sb)[:, :, None] * np.sqrt(n[W])[:, None, :]
    d = np.arange(N)
    Mcj[d, d] = 0.0
    for M in Ms:
        M[d, d] = 0.0
    return (dn, dfi, dnd12, dnd), Mcj, Ms


def calce(n, cj12, ck12, J_MO, K_MO, H_core, p: Param) -> float:
    """Occupation-space energy (src/pnof.jl:1273-1300)."""
    dJ = np.diag(J_MO)
    w = 2.0 * H_core + dJ
    E = float(n[: p.nbeta] @ w[: p.nbeta])
    if p.nsoc > 0:
        E += float(2.0 * n[p.nbeta: p.nalpha] @ H_core[p.nbeta: p.nalpha])
    E += float(n[p.nalpha: p.nbf5] @ w[p.nalpha: p.nbf5])
    E += float(np.sum(cj12 * J_MO.T) - np.sum(ck12 * K_MO.T))
    return E


def calcocce(gamma, J_MO, K_MO, H_core, p: Param) -> float:
    n, _ = occupations(gamma, p)
    cj, ck = coupling(n, p)
    return calce(n, cj, ck, J_MO, K_MO, H_core, p)


def calcoccg(gamma, J_MO, K_MO, H_core, p: Param) -> np.ndarray:
    """Occupation gradient (src/pnof.jl:1324-1377).  The reference contracts the
    nbf5 x nbf5 x nv derivative tensors of der_CJCKD8 with J_MO and K_MO; their
    terms are separable (_derivative_factors), so the contraction runs over
    (i, j) first and costs O(nbf5^2 + nbf5 nv) instead of O(nbf5^2 nv)."""
    n, dn = occupations(gamma, p)
    A, Mcj, Mck = _derivative_factors(n, dn, p)
    w = 2.0 * H_core + np.diag(J_MO)
    rows = np.r_[np.arange(p.no1, p.nbeta), np.arange(p.nalpha, p.nbf5)]
    g = dn[rows].T @ w[rows]
    vj = np.sum(Mcj * J_MO.T, axis=1)  # vj[i] = sum_j Mcj[i, j] J_MO[j, i]
    g += 2.0 * A[0][rows].T @ vj[rows]
    for a, M in zip(A, Mck):
        vk = np.sum(M * K_MO.T, axis=1)
        g -= 2.0 * a[rows].T @ vk[rows]
    return g


def guess_gamma(p: Param) -> np.ndarray:
    """Initial gamma (src/guess.jl:184-213)."""
    g = np.zeros(p.nv)
    if p.occ_method == "Softmax":
        g[p.gamma_table()] = math.log(max(0.001 / p.ncwo, 1e-16)) - math.log(0.999)
    elif p.occ_method == "Trigonometric":
        g[: p.ndoc] = math.acos(math.sqrt(2.0 * 0.999 - 1.0))
        for i in range(1, p.ndoc + 1):
            for j in range(1, p.ncwo):
                g[p.ndoc + (p.ndoc - i) + p.ndoc * (j - 1)] = math.asin(math.sqrt(1.0 / (p.ncwo - j + 1)))
    else:
        raise ValueError(p.occ_method)
    return g


def n_to_gammas(n, p: Param) -> np.ndarray:
    """gamma whose occupations are n: the restart path of DoNOF.energy
    (src/energy.jl:95-99), n_to_gammas_softmax (src/utils.jl:539-561) and
    n_to_gammas_trigonometric (src/utils.jl:563-584)."""
    n = np.asarray(n, dtype=np.float64)
    g = np.zeros(p.nv)
    nd, nc = p.ndoc, p.ncwo
    P = p.pair_table()
    if p.occ_method == "Softmax":
        # the reference divides by n[i] with i the pair index (1-based), kept as is
        g[p.gamma_table()] = np.log(np.maximum(n[P], 1e-16)) - np.log(n[:nd])[:, None]
    elif p.occ_method == "Trigonometric":
        strong = p.no1 + np.arange(nd)
        g[:nd] = np.arccos(np.sqrt(2.0 * n[strong] - 1.0))
        for i in range(nd):
            pref = max(1.0 - n[strong[i]], 1e-14)
            cols = nd + (nd - (i + 1)) + nd * np.arange(nc - 1)
            for j in range(nc - 1):
                g[cols[j]] = math.asin(math.sqrt(n[P[i, j]] / pref))
                pref *= math.cos(g[cols[j]]) ** 2
    else:
        raise ValueError(f"occupation method {p.occ_method!r} is not supported")
    return g


def order_occupations_softmax(C, gamma, p: Param):
    """Sort each pair's orbitals by gamma, descending (src/utils.jl:586-616)."""
    C = np.array(C, copy=True, order="F")
    gamma = np.array(gamma, copy=True)
    if not np.any(gamma > 0):
        return C, gamma
    C0 = C.copy()
    for g, (ws, gi) in enumerate(zip(p.pair_table(), p.gamma_table())):
        cols = np.r_[p.no1 + g, ws]
        vals = np.r_[0.0, gamma[gi]]
        order = np.argsort(vals, kind="stable")[::-1]
        vals = vals[order] - vals.max()
        gamma[gi] = vals[1:]
        C[:, cols] = C0[:, cols[order]]
    return C, gamma
