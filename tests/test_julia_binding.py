"""The Julia binding (julia/): every ccall names an entry point of
include/donof_b200.h with the same number of arguments and matching kinds
(pointer / int / double / size), the extension keeps the module name that
DoNOF.jl's compute_integrals looks up, and the Project.toml entries select it
through the DoNOFB200 package.  Julia is not installed here, so the files are
checked as text."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
JL = [ROOT / "julia" / "DoNOFB200" / "src" / "DoNOFB200.jl", ROOT / "julia" / "ext" / "DoNOFGPUExt.jl"]
HEADER = ROOT / "include" / "donof_b200.h"


def _balanced(text, start):
    """Text of the parenthesised group opening at text[start] == '('."""
    depth = 0
    for i in range(start, len(text)):
        c = text[i]
        if c in "({[":
            depth += 1
        elif c in ")}]":
            depth -= 1
            if depth == 0:
                return text[start + 1:i]
    raise ValueError("unbalanced")


def _split_top(s):
    out, depth, cur = [], 0, ""
    for c in s:
        if c in "({[":
            depth += 1
        elif c in ")}]":
            depth -= 1
        if c == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += c
    if cur.strip():
        out.append(cur.strip())
    return out


def ccalls(text):
    calls = []
    for m in re.finditer(r"ccall\(", text):
        body = _balanced(text, m.end() - 1)
        parts = _split_top(body)
        sym = re.match(r"\(:(\w+),\s*(\w+)\)", parts[0])
        assert sym, parts[0]
        types = _split_top(parts[2][1:-1]) if parts[2].startswith("(") else [parts[2]]
        calls.append((sym.group(1), sym.group(2), parts[1], types, parts[3:]))
    return calls


def header_prototypes():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    protos = {}
    for m in re.finditer(r"([\w\s\*]+?)\b(donof_\w+)\s*\(([^;{]*?)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3).strip()
        plist = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        protos[name] = (ret, plist)
    return protos


def kind_c(decl):
    d = decl.replace("const", "").strip()
    if "*" in d:
        return "ptr"
    if "unsigned long long" in d:
        return "u64"
    if "long long" in d:
        return "i64"
    if "size_t" in d:
        return "size"
    if "double" in d:
        return "f64"
    if re.match(r"int\b", d):
        return "i32"
    raise AssertionError(decl)


def kind_jl(t):
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{")) or t in ("Cstring", "Ptr"):
        return "ptr"
    return {"Cint": "i32", "Cdouble": "f64", "Float64": "f64", "Csize_t": "size", "Clonglong": "i64",
            "Culonglong": "u64", "UInt64": "u64", "Cvoid": "void"}[t]


def test_every_ccall_matches_a_declared_entry_point():
    protos = header_prototypes()
    assert len(protos) > 40
    seen = set()
    for path in JL:
        for sym, lib, ret, types, args in ccalls(path.read_text()):
            assert lib == "libdonof", (path.name, sym)
            assert sym in protos, f"{path.name}: {sym} is not declared in {HEADER.name}"
            cret, cparams = protos[sym]
            assert len(types) == len(cparams), f"{sym}: {len(types)} Julia argument types, {len(cparams)} in C"
            assert len(args) == len(types), f"{sym}: {len(args)} arguments for {len(types)} types"
            for jt, cp in zip(types, cparams):
                assert kind_jl(jt) == kind_c(cp), f"{sym}: Julia {jt} against C {cp}"
            rk = "ptr" if "*" in cret else kind_c(cret)
            assert kind_jl(ret) == rk, f"{sym}: returns {ret}, C returns {cret}"
            seen.add(sym)
    # the entry points that replace the reference extension's methods are all bound
    for need in ("donof_b_upload", "donof_iaux", "donof_lagrange2", "donof_jkh_mo", "donof_rotate",
                 "donof_orbgrad", "donof_orbopt", "donof_energy", "donof_job_free", "donof_create"):
        assert need in seen, need


def test_struct_layouts_match_the_header():
    """EnergyParams / OccParams / EnergyResult field order and kinds equal the C structs."""
    jl = JL[0].read_text()
    hdr = HEADER.read_text()

    def jl_fields(name):
        body = re.search(rf"struct {name}\n(.*?)\nend", jl, flags=re.S).group(1)
        return [(f.split("::")[0].strip(), f.split("::")[1].strip()) for f in body.strip().splitlines()]

    def c_fields(name):
        body = re.search(r"typedef struct \{([^{}]*?)\}\s*" + name + ";", hdr).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        out = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            m = re.match(r"([\w\s]+?)\s+([\w\s,]+)$", decl)
            typ, names = m.group(1), [n.strip() for n in m.group(2).split(",")]
            out += [(n, typ) for n in names]
        return out

    kinds = {"Cint": "int", "Cdouble": "double", "OccParams": "donof_occ_params"}
    for jname, cname in (("OccParams", "donof_occ_params"), ("EnergyParams", "donof_energy_params"),
                         ("EnergyResult", "donof_energy_result")):
        jf, cf = jl_fields(jname), c_fields(cname)
        assert [n for n, _ in jf] == [n for n, _ in cf], jname
        assert [kinds[t] for _, t in jf] == [t for _, t in cf], jname


def test_extension_keeps_the_name_compute_integrals_looks_up():
    ext = JL[1].read_text()
    assert re.search(r"^module DoNOFGPUExt\b", ext, flags=re.M)
    for fn in ("Iaux_gpu", "eris_to_gpu"):
        assert re.search(rf"^{fn}\(", ext, flags=re.M), fn
    for meth in ("computeJKH_MO", "JKH_MO", "compute_Lagrange2", "rotate_orbital", "calcorbg", "orbopt_adam",
                 "orbopt_adabelief", "orbopt_yogi", "orbopt_demon"):
        assert re.search(rf"DoNOF\.{meth}\(", ext), meth


def test_project_entries_select_the_extension_through_the_package():
    tomllib = pytest.importorskip("tomllib")
    pkg = tomllib.loads((ROOT / "julia" / "DoNOFB200" / "Project.toml").read_text())
    ent = tomllib.loads((ROOT / "julia" / "DoNOF.Project.extensions.toml").read_text())
    assert pkg["name"] == "DoNOFB200"
    assert ent["weakdeps"]["DoNOFB200"] == pkg["uuid"]
    assert ent["extensions"]["DoNOFGPUExt"] == "DoNOFB200"
    assert re.fullmatch(r"[0-9a-f]{8}-[0-9a-f]{4}-4[0-9a-f]{3}-[89ab][0-9a-f]{3}-[0-9a-f]{12}", pkg["uuid"])
