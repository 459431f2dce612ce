"""The Fortran ISO_C_BINDING module (bgk_pcm_b200/fortran/bgk_c.f90) checked
mechanically against the C header (include/bgk_pcm.h).

No Fortran compiler exists on either machine, so nothing else would notice a
binding that disagrees with the library: a missing `value` attribute makes
Fortran pass the address of an integer where C reads the integer itself, and
a struct with a field out of order shifts every later field.  The reference
binds its one C helper the same way (STEP_7/get_mem_mod.f90:7 to
STEP_7/get_mem.c:23).  Checked here, for every bind(c) interface:

* the bound name exists in the header, with the same number of arguments;
* each argument's kind (c_int, c_double, c_size_t, c_char, c_ptr, or one of
  the bind(c) types) and passing: `value` where C takes a scalar or a handle
  by value, by reference where C takes a pointer or an array; array extents
  where C states one (double out[4]);
* the result kind;
* every bind(c) derived type has the C struct's fields, in order, with
  matching kinds;
* every named constant equals the header's #define of the same name;
* every function the header declares is bound.
"""
from __future__ import annotations

import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "bgk_pcm.h"
F90 = ROOT / "bgk_pcm_b200" / "fortran" / "bgk_c.f90"

STRUCTS = ("bgk_params", "bgk_options", "bgk_adjoint_spec")


# ------------------------------------------------------------------ C side
def _strip_c_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def _c_arg(decl: str):
    """(base type, pointer depth, array extent or None, name) of one C parameter."""
    decl = decl.strip()
    m = re.match(r"^(.*?)([A-Za-z_]\w*)\s*(\[\s*(\d*)\s*\])?$", decl)
    assert m, decl
    typ, name, arr, ext = m.group(1), m.group(2), m.group(3), m.group(4)
    depth = typ.count("*")
    base = " ".join(t for t in typ.replace("*", " ").split() if t != "const")
    return base, depth, (int(ext) if ext else (0 if arr else None)), name


def parse_header(text: str):
    body = re.sub(r"(?m)^\s*#.*$", " ", _strip_c_comments(text))
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(BGK_\w+)\s+(-?\d+)\b", text)}
    structs = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", body, flags=re.S):
        fields = []
        for stmt in m.group(2).split(";"):
            stmt = " ".join(stmt.split())
            if not stmt:
                continue
            first, *rest = stmt.split(",")
            base, depth, _, name = _c_arg(first)
            fields.append((base, depth, name))
            for r in rest:
                r = r.strip()
                d = r.count("*")
                fields.append((base, d if d else depth, r.replace("*", "").strip()))
        structs[m.group(3)] = fields
    funcs = {}
    for stmt in re.split(r"[;{}]", body):
        m = re.match(r"^\s*((?:const\s+)?\w+\s*\**)\s*(bgk_\w+)\s*\(([^)]*)\)\s*$", stmt, flags=re.S)
        if not m:
            continue
        ret, name, args = m.group(1), m.group(2), " ".join(m.group(3).split())
        params = [] if args in ("", "void") else [_c_arg(a) for a in args.split(",")]
        funcs[name] = (" ".join(ret.replace("*", " * ").split()), params)
    return defines, structs, funcs


# ------------------------------------------------------------ Fortran side
def _join_continuations(text: str) -> list[str]:
    lines, cur = [], ""
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        if cur:
            line = line.lstrip()
            if line.startswith("&"):
                line = line[1:]
        cur += line
        if cur.endswith("&"):
            cur = cur[:-1]
            continue
        lines.append(cur.strip())
        cur = ""
    return lines


def _split_top(s: str) -> list[str]:
    """Split at commas outside parentheses."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _decl(line: str):
    """(type spec, attributes, [(name, init or None)]) of a declaration line."""
    spec, names = line.split("::", 1)
    parts = _split_top(spec)
    typ = parts[0].replace(" ", "").lower()
    attrs = [a.replace(" ", "").lower() for a in parts[1:]]
    ents = []
    for n in _split_top(names):
        if "=" in n:
            k, v = n.split("=", 1)
            ents.append((k.strip(), v.strip()))
        else:
            ents.append((n.strip(), None))
    return typ, attrs, ents


def parse_f90(text: str):
    lines = _join_continuations(text)
    params, types, funcs = {}, {}, {}
    i = 0
    while i < len(lines):
        ln = lines[i]
        low = ln.lower()
        m = re.match(r"type\s*,\s*bind\(c\)\s*::\s*(\w+)", low)
        if m:
            tname, fields = m.group(1), []
            i += 1
            while not lines[i].lower().startswith("end type"):
                typ, _, ents = _decl(lines[i])
                fields += [(typ, n.lower()) for n, _ in ents]
                i += 1
            types[tname] = fields
        elif "parameter" in low and "::" in low and not low.startswith("function"):
            typ, attrs, ents = _decl(ln)
            if "parameter" in attrs:
                for n, v in ents:
                    params[n] = (typ, int(v))
        m = re.match(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\(\s*c\s*,\s*name\s*=\s*\"(\w+)\"\s*\)\s*result\((\w+)\)",
                     ln, flags=re.I)
        if m:
            args = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
            bind_name, res = m.group(3), m.group(4).lower()
            decls = {}
            i += 1
            while not lines[i].lower().startswith("end function"):
                if "::" in lines[i] and not lines[i].lower().startswith("import"):
                    typ, attrs, ents = _decl(lines[i])
                    for n, _ in ents:
                        decls[n.lower()] = (typ, attrs)
                i += 1
            funcs[bind_name] = {"args": [(a, *decls[a]) for a in args], "result": decls[res][0]}
        i += 1
    return params, types, funcs


# ------------------------------------------------------------- the mapping
def expected_fortran(base: str, depth: int, extent):
    """(type spec, passed by value, array extent: None scalar, '*' any, n) a
    C parameter needs on the Fortran side."""
    if base in ("bgk_ctx", "void"):
        return "type(c_ptr)", depth == 1, None
    if base in STRUCTS:
        assert depth == 1
        return f"type({base})", False, None
    kind = {"int": "integer(c_int)", "double": "real(c_double)", "size_t": "integer(c_size_t)",
            "char": "character(kind=c_char)"}[base]
    if extent is not None:
        return kind, False, extent if extent else "*"
    if depth == 0:
        return kind, True, None
    return kind, False, "*" if base == "char" else "scalar-or-array"


def expected_field(base: str, depth: int) -> str:
    if depth:
        return "type(c_ptr)"
    return {"int": "integer(c_int)", "double": "real(c_double)"}[base]


def check_binding(header_text: str, f90_text: str) -> list[str]:
    defines, structs, cfuncs = parse_header(header_text)
    params, types, ffuncs = parse_f90(f90_text)
    errs = []
    for name, (typ, val) in params.items():
        if name not in defines:
            errs.append(f"constant {name} has no #define in the header")
        elif defines[name] != val:
            errs.append(f"constant {name} = {val}, header {defines[name]}")
    for tname in STRUCTS:
        if tname not in types:
            errs.append(f"type {tname} is not bound")
            continue
        want = [(expected_field(b, d), n.lower()) for b, d, n in structs[tname]]
        if types[tname] != want:
            errs.append(f"type {tname}: fields {types[tname]} != header {want}")
    for name in cfuncs:
        if name not in ffuncs:
            errs.append(f"{name} is declared in the header but not bound")
    for name, f in ffuncs.items():
        if name not in cfuncs:
            errs.append(f"{name} is bound but not declared in the header")
            continue
        ret, cargs = cfuncs[name]
        if len(cargs) != len(f["args"]):
            errs.append(f"{name}: {len(f['args'])} arguments, header {len(cargs)}")
            continue
        want_res = "integer(c_int)" if ret == "int" else ("type(c_ptr)" if ret.endswith("*") else ret)
        if f["result"] != want_res:
            errs.append(f"{name}: result {f['result']}, header {ret}")
        for (fname, ftyp, attrs), (base, depth, extent, cname) in zip(f["args"], cargs):
            kind, by_value, ext = expected_fortran(base, depth, extent)
            has_value = "value" in attrs
            dims = [a[len("dimension("):-1] for a in attrs if a.startswith("dimension(")]
            where = f"{name}({cname})"
            if (depth == 1 or extent is not None) and ftyp == "type(c_ptr)" and has_value and not dims:
                continue    # an address passed as a c_ptr by value: the same C pointer (device memory)
            if ftyp != kind:
                errs.append(f"{where}: {ftyp}, header needs {kind}")
            if has_value != by_value:
                errs.append(f"{where}: {'value' if has_value else 'by reference'}, header passes it "
                            f"{'by value' if by_value else 'as a pointer'}")
            if ext == "*" and dims != ["*"]:
                errs.append(f"{where}: dimension {dims}, header needs an assumed-size array")
            if isinstance(ext, int) and dims != [str(ext)]:
                errs.append(f"{where}: dimension {dims}, header needs dimension({ext})")
            if ext is None and dims:
                errs.append(f"{where}: an array, header takes a scalar")
    return errs


# ------------------------------------------------------------------- tests
def test_fortran_module_matches_header():
    errs = check_binding(HEADER.read_text(), F90.read_text())
    assert errs == [], "\n".join(errs)
    _, _, cfuncs = parse_header(HEADER.read_text())
    _, _, ffuncs = parse_f90(F90.read_text())
    assert len(ffuncs) == len(cfuncs) >= 32


def test_header_parser_sees_every_declaration():
    """The prototype parser above finds every bgk_ function the header names
    (so no declaration escapes the binding check)."""
    text = HEADER.read_text()
    _, _, cfuncs = parse_header(text)
    named = set(re.findall(r"\b(bgk_[a-z_0-9]+)\s*\(", _strip_c_comments(text)))
    assert set(cfuncs) == named


@pytest.mark.parametrize("mutate,expect", [
    # an integer passed by value loses its `value`: Fortran would pass its address
    (lambda s: s.replace("integer(c_int), value :: nsteps", "integer(c_int) :: nsteps", 1), "by reference"),
    # a context handle passed by reference
    (lambda s: s.replace("""function bgk_sync(ctx) bind(c, name="bgk_sync") result(rc)
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx""", """function bgk_sync(ctx) bind(c, name="bgk_sync") result(rc)
       import :: c_int, c_ptr
       type(c_ptr) :: ctx"""), "bgk_sync(ctx)"),
    # two struct fields swapped
    (lambda s: s.replace("integer(c_int) :: precision, tanh_mode, fma", "integer(c_int) :: tanh_mode, precision, fma"),
     "type bgk_options"),
    # a wrong kind
    (lambda s: s.replace("integer(c_size_t), intent(out) :: bytes", "integer(c_int), intent(out) :: bytes"),
     "bgk_rows_bytes(bytes)"),
    # a wrong extent
    (lambda s: s.replace("real(c_double), dimension(4), intent(out) :: out", "real(c_double), dimension(3), intent(out) :: out"),
     "dimension(4)"),
    # a constant that drifted
    (lambda s: s.replace("BGK_FIELD_PHI = 22", "BGK_FIELD_PHI = 23"), "BGK_FIELD_PHI"),
])
def test_checker_finds_planted_mistakes(mutate, expect):
    """Each planted mistake (in a copy of the module text, in memory) is reported."""
    text = F90.read_text()
    bad = mutate(text)
    assert bad != text
    errs = check_binding(HEADER.read_text(), bad)
    assert any(expect in e for e in errs), errs
