"""The Julia `ccall` shim against the C header, without a Julia toolchain.

Every `ccall` in stokesflow.jl_b200/julia/StokesFlowB200.jl must name an entry
point the header declares, with one Julia argument type per C parameter, in
order, of the matching kind and width, and as many values as types.  The
Julia mirrors of the result structs (SolveInfo, BatchInstance) must list the
C struct's fields in the same order and with the same types, so that `Ref{T}`
lays them out byte for byte as the library writes them.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "stokesflow_b200.h")
SHIM = os.path.join(ROOT, "stokesflow.jl_b200", "julia", "StokesFlowB200.jl")

JULIA_STRUCT_OF = {"sf_solve_info": "SolveInfo", "sf_batch_instance": "BatchInstance", "sf_deposit_grid": "DepositGrid"}


def _strip_c_comments(text):
    return re.sub(r"/\*.*?\*/", " ", text, flags=re.S)


def _strip_julia_comments(text):
    return "\n".join(re.sub(r"#.*$", "", ln) for ln in text.splitlines())


def _split_top(s):
    """Split s at the commas that sit outside (), {} and []."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur).strip())
    return out


def _closing(s, i):
    """Index of the bracket closing the one at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] in "({[":
            depth += 1
        elif s[j] in ")}]":
            depth -= 1
            if depth == 0:
                return j
    raise ValueError("unbalanced")


def c_prototypes():
    text = _strip_c_comments(open(HEADER).read())
    protos = {}
    for m in re.finditer(r"\n\s*((?:const\s+)?[A-Za-z_][\w]*\s*\**)\s*(sf_\w+)\s*\(([^;]*?)\)\s*;", text):
        ret, name, params = m.group(1).strip(), m.group(2), m.group(3)
        plist = [] if params.strip() in ("", "void") else [" ".join(p.split()) for p in params.split(",")]
        protos[name] = (ret, plist)
    return protos


def c_structs():
    text = _strip_c_comments(open(HEADER).read())
    structs = {}
    for m in re.finditer(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in m.group(1).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            dm = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)$", decl)
            base, names = dm.group(1), dm.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                stars = nm.count("*")
                nm = nm.replace("*", "").strip()
                arr = re.match(r"(\w+)\[(\d+)\]", nm)
                typ = (base.replace(" ", "") + "*" * stars)
                if arr:
                    fields.append((arr.group(1), f"{typ}[{arr.group(2)}]"))
                else:
                    fields.append((nm, typ))
        structs[m.group(2)] = fields
    return structs


def julia_ccalls():
    text = _strip_julia_comments(open(SHIM).read())
    calls = []
    for m in re.finditer(r"ccall\(", text):
        start = m.end() - 1
        body = text[start + 1:_closing(text, start)]
        items = _split_top(body)
        name = re.match(r"\(:(\w+),", items[0]).group(1)
        ret = items[1]
        types = _split_top(items[2].strip()[1:-1])
        calls.append((name, ret, types, items[3:]))
    return calls


def julia_structs():
    text = _strip_julia_comments(open(SHIM).read())
    structs = {}
    for m in re.finditer(r"^struct (\w+)\n(.*?)^end", text, flags=re.S | re.M):
        fields = []
        for part in re.split(r"[;\n]", m.group(2)):
            part = part.strip()
            if part:
                nm, typ = part.split("::")
                fields.append((nm.strip(), typ.strip()))
        structs[m.group(1)] = fields
    return structs


def c_param_kind(p):
    """The Julia ccall type a C parameter declaration binds to."""
    p = p.replace(" *", "* ").replace("  ", " ")
    typ = p.rsplit(" ", 1)[0].replace(" ", "") if " " in p else p
    simple = {"double": "Cdouble", "int64_t": "Int64", "int": "Cint", "int32_t": "Int32",
              "double*": "Ptr{Cdouble}", "constdouble*": "Ptr{Cdouble}", "void*": "Ptr{Cvoid}",
              "sf_ctx*": "Ptr{Cvoid}", "constsf_mixed_options*": "Ptr{Cvoid}", "sf_ctx**": "Ref{Ptr{Cvoid}}",
              "constchar*": "Cstring", "constsf_deposit_grid*": "Ptr{DepositGrid}"}
    if typ in simple:
        return simple[typ]
    for cname, jname in JULIA_STRUCT_OF.items():
        if typ == cname + "*":
            return f"Ref{{{jname}}}"
    raise AssertionError(f"no Julia binding rule for C parameter {p!r}")


def c_field_kind(typ):
    return {"double": "Float64", "int64_t": "Int64", "int32_t": "Int32", "double*": "Ptr{Cdouble}",
            "constdouble*": "Ptr{Cdouble}"}[typ]


def _ascii(name):
    return name.replace("ρ", "rho").replace("μ", "mu")


def test_shim_parses():
    calls = julia_ccalls()
    assert {c[0] for c in calls} >= {"sf_ctx_create", "sf_last_error", "sf_bilinear_marker_to_grid",
                                     "sf_solve_stokes", "sf_solve_stokes_mixed", "sf_move_markers_rk4"}


@pytest.mark.parametrize("call", julia_ccalls(), ids=lambda c: c[0])
def test_ccall_matches_header(call):
    name, ret, jtypes, values = call
    protos = c_prototypes()
    assert name in protos, f"{name} is not declared in the header"
    cret, cparams = protos[name]
    assert c_param_kind(cret + " r") == ret, f"{name}: return {cret} bound as {ret}"
    assert len(jtypes) == len(cparams), f"{name}: {len(jtypes)} Julia types for {len(cparams)} C parameters"
    for k, (jt, cp) in enumerate(zip(jtypes, cparams)):
        assert jt == c_param_kind(cp), f"{name}: parameter {k} ({cp}) bound as {jt}"
    assert len(values) == len(jtypes), f"{name}: {len(values)} values for {len(jtypes)} types"


@pytest.mark.parametrize("cname", sorted(JULIA_STRUCT_OF))
def test_result_structs_match_header(cname):
    cfields = c_structs()[cname]
    jfields = julia_structs()[JULIA_STRUCT_OF[cname]]
    assert [_ascii(n) for n, _ in jfields] == [n for n, _ in cfields]
    assert [t for _, t in jfields] == [c_field_kind(t) for _, t in cfields]
