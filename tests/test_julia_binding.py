"""The Julia binding (autorift.jl_b200/julia/AutoRIFTGPU.jl) against the C header.

Julia is not installed in this image, so the binding is checked by reading: every struct it
passes to the library has the header's fields in the header's order with the matching Julia
types, every `ccall` names a symbol the header declares with its number of arguments, and its
status and enum constants equal the header's.
"""

import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = (ROOT / "include" / "autorift_gpu.h").read_text()
JULIA = (ROOT / "autorift.jl_b200" / "julia" / "AutoRIFTGPU.jl").read_text()

STRUCTS = {"ar_points": "ArPoints", "ar_prepare_opts": "ArPrepareOpts",
           "ar_multichip_params": "ArMultichipParams", "ar_request": "ArRequest"}

SCALARS = {"int": "Cint", "double": "Float64", "int64_t": "Int64", "float": "Float32",
           "uint8_t": "UInt8", "uint16_t": "UInt16", "void": "Cvoid"}


def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def header_struct(name):
    blocks = {m.group(2): m.group(1) for m in
              re.finditer(r"typedef struct \{([^{}]*)\}\s*(\w+)\s*;", _strip_comments(HEADER))}
    assert name in blocks, name
    fields = []
    for decl in blocks[name].split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        decl = decl.replace("const ", "")
        m = re.match(r"([A-Za-z_0-9]+)\s*(\**)\s*(.*)", decl)
        base, stars, names = m.group(1), m.group(2), m.group(3)
        for nm in names.split(","):
            nm = nm.strip()
            extra = nm.count("*")
            nm = nm.replace("*", "").strip()
            arr = re.match(r"(\w+)\[(\d+)\]", nm)
            t = SCALARS.get(base, STRUCTS.get(base, base))
            for _ in range(len(stars) + extra):
                t = f"Ptr{{{t}}}"
            if arr:
                nm, t = arr.group(1), f"NTuple{{{arr.group(2)},{t}}}"
            fields.append((nm, t))
    return fields


def julia_struct(name):
    body = re.search(r"^struct " + name + r"\n(.*?)^end", JULIA, re.S | re.M)
    assert body, name
    fields = []
    for line in body.group(1).splitlines():
        line = line.split("#")[0].strip()
        if line:
            nm, t = line.split("::")
            fields.append((nm.strip(), t.strip().replace(" ", "")))
    return fields


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_julia_structs_match_the_header(cname):
    assert julia_struct(STRUCTS[cname]) == header_struct(cname)


def _header_functions():
    src = _strip_comments(HEADER)
    out = {}
    for m in re.finditer(r"\bint\s+(ar_\w+)\s*\(([^)]*)\)\s*;", src):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(1)] = len(args)
    return out


def _julia_ccalls():
    calls = []
    for m in re.finditer(r"ccall\(\(:(\w+),\s*LIB\),\s*\w+,\s*\(", JULIA):
        # The argument-type tuple: balance parentheses from the opening one.
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(JULIA[i], 0)
            i += 1
        types = JULIA[m.end():i - 1]
        depth, n, cur = 0, 0, ""
        for ch in types:
            if ch in "({":
                depth += 1
            elif ch in ")}":
                depth -= 1
            if ch == "," and depth == 0:
                n += 1 if cur.strip() else 0
                cur = ""
            else:
                cur += ch
        n += 1 if cur.strip() else 0
        calls.append((m.group(1), n))
    return calls


def test_every_ccall_names_a_declared_symbol_with_its_arity():
    declared = _header_functions()
    calls = _julia_ccalls()
    assert len(calls) >= 10
    for sym, n in calls:
        assert sym in declared, sym
        assert declared[sym] == n, f"{sym}: {n} argument types, header has {declared[sym]}"


def test_julia_constants_match_the_header_enums():
    enums = {}
    for m in re.finditer(r"enum\s*\{([^}]*)\}", _strip_comments(HEADER)):
        for item in m.group(1).split(","):
            if "=" in item:
                k, v = item.split("=")
                enums[k.strip()] = int(v.strip())
    found = 0
    for m in re.finditer(r"^const ((?:AR_\w+,?\s*)+)=\s*(.+)$", JULIA, re.M):
        names = [x.strip() for x in m.group(1).split(",") if x.strip()]
        vals = [int(v) for v in re.findall(r"Cint\((\d+)\)", m.group(2))]
        assert len(names) == len(vals)
        for k, v in zip(names, vals):
            assert enums[k] == v, k
            found += 1
    assert found >= 10


def test_binding_keeps_no_global_pair_cache_and_passes_both_masks():
    # Device pairs are owned by a Cache or freed by the call that made them.
    assert "IdDict" not in JULIA
    for fn in ("init", "reinit!", "autorift!", "imagepair"):
        assert re.search(r"^function " + re.escape(fn) + r"\(|^" + re.escape(fn) + r"\(",
                         JULIA, re.M), fn
    assert "Base.close(cache::Cache)" in JULIA
    sub = JULIA[JULIA.index("function submit("):JULIA.index("function Base.fetch")]
    assert "reference_valid" in sub and "C_NULL, \n" not in sub
