"""The .fchk writer (donof_b200/output.py, src/output.jl:1-283): records,
counts, values per line, the density from the occupations, the MO order and
the cartesian reordering, read back from the written file."""
import numpy as np
import pytest

from donof_b200 import Param
from donof_b200.output import BasisDescription, Shell, fchk


def _water(spherical=True):
    # O with s, s, p, d and two H with s, s, p (cc-pVDZ-like shell structure)
    shells = [Shell(0, 0, [11720.0, 1759.0, 400.8], [0.00071, 0.00547, 0.02784]),
              Shell(0, 0, [0.3023], [1.0]), Shell(1, 0, [17.7, 3.854], [0.043, 0.2289]),
              Shell(2, 0, [1.185], [1.0])]
    for a in (1, 2):
        shells += [Shell(0, a, [13.01, 1.962], [0.0197, 0.138]), Shell(0, a, [0.1220], [1.0]),
                   Shell(1, a, [0.727], [1.0])]
    xyz = np.array([[0.0, 0.0, 0.121], [0.0, 0.751, -0.485], [0.0, -0.751, -0.485]])
    return BasisDescription("cc-pVDZ", [8, 1, 1], xyz, shells, spherical)


def _nbf(basis):
    return sum((2 * s.l + 1) if basis.spherical else (s.l + 1) * (s.l + 2) // 2 for s in basis.shells)


def _read(path):
    rec, cur = {}, None
    for line in open(path).read().splitlines()[2:]:
        if line[:1] != " ":
            name = line[:43].strip()
            kind, rest = line[43], line[44:]
            if "N=" in rest:
                cur = rec[name] = {"kind": kind, "n": int(rest.split()[-1]), "vals": [], "lines": []}
            else:
                rec[name] = {"kind": kind, "value": rest.split()[0]}
                cur = None
        else:
            cur["lines"].append(line)
            cur["vals"] += [float(x) for x in line.split()]
    return rec


@pytest.mark.parametrize("spherical", [True, False])
def test_fchk_records_read_back(tmp_path, spherical):
    basis = _water(spherical)
    nbf = _nbf(basis)
    p = Param(nbf=nbf, nbfaux=4 * nbf, nalpha=5, nbeta=5, ncwo=1)
    rng = np.random.default_rng(1)
    C = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0]
    n = np.sort(rng.uniform(0, 1, p.nbf5))[::-1]
    elag = rng.standard_normal((nbf, nbf))
    path = fchk(str(tmp_path / "water"), p, basis, "Energy", -76.2, elag, n, C)
    lines = open(path).read().splitlines()
    assert lines[0] == str(tmp_path / "water") and lines[1] == "Energy PNOF8 cc-pVDZ"
    rec = _read(path)
    assert int(rec["Number of basis functions"]["value"]) == nbf
    assert int(rec["Number of independant functions"]["value"]) == p.nbf5
    assert int(rec["Charge"]["value"]) == 0 and int(rec["Multiplicity"]["value"]) == 1
    assert float(rec["Total Energy"]["value"]) == -76.2
    for name, r in rec.items():
        if "n" in r:
            assert len(r["vals"]) == r["n"], name
            per = 6 if (r["kind"] == "I" or name == "Nuclear Charges") else 5
            assert all(len(line.split()) <= per for line in r["lines"]), name
    assert rec["Shell types"]["vals"] == [0, 0, 1, -2 if spherical else 2] + [0, 0, 1] * 2
    assert rec["Shell to atom map"]["vals"] == [1] * 4 + [2] * 3 + [3] * 3
    np.testing.assert_allclose(rec["Alpha Orbital Energies"]["vals"], np.diag(elag), rtol=1e-8)
    Cf = np.array(rec["Alpha MO coefficients"]["vals"]).reshape(nbf, nbf, order="F")
    if spherical:
        np.testing.assert_allclose(Cf, C, rtol=1e-8, atol=1e-12)
    else:  # the d shell (rows 9..14, 1-based xx,xy,xz,yy,yz,zz) in the fchk order xx,yy,zz,xy/r3,xz/r3,yz/r3
        d = 5
        np.testing.assert_allclose(Cf[d + 1], C[d + 3], rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(Cf[d + 3], C[d + 1] / np.sqrt(3), rtol=1e-8, atol=1e-12)
        np.testing.assert_allclose(Cf[:d], C[:d], rtol=1e-8, atol=1e-12)
    C5 = Cf[:, :p.nbf5]
    DM = 2 * (C5 * n) @ C5.T
    tri = [DM[i, j] for i in range(nbf) for j in range(i + 1)]
    np.testing.assert_allclose(rec["Total SCF Density"]["vals"], tri, rtol=1e-7, atol=1e-8)  # 9 digits written
    np.testing.assert_allclose(rec["Natural orbital occupancies"]["vals"], n, rtol=1e-8)
    xyz = np.array(rec["Current cartesian coordinates"]["vals"]).reshape(3, 3)
    np.testing.assert_allclose(xyz, basis.xyz * 1.88973, rtol=1e-8)


def test_restart_round_trip(tmp_path):
    """save_restart / load_restart: the occupations come back through n_to_gammas."""
    from donof_b200 import gnof
    from donof_b200.output import load_restart, save_restart
    p = Param(nbf=24, nbfaux=116, nalpha=5, nbeta=5, ncwo=3)
    rng = np.random.default_rng(4)
    gamma = rng.standard_normal(p.nv)
    n, _ = gnof.occupations(gamma, p)
    C = np.linalg.qr(rng.standard_normal((24, 24)))[0]
    path = save_restart(str(tmp_path / "job"), -76.3, C, n)
    E, C2, gamma2 = load_restart(path, p)
    assert E == -76.3 and np.array_equal(C2, C)
    n2, _ = gnof.occupations(gamma2, p)
    np.testing.assert_allclose(n2, n, atol=1e-12)
