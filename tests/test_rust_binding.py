"""The Rust binding shown in INTEGRATION.md (the `extern "C"` block a
maintainer adds to the reference crate) against include/rh3t.h and the
ctypes mirror the tests use (3t_rh_b200/_lib.py): every #[repr(C)] struct
has the header's fields in the header's order with the same C layout
(offsets and size), and every declared function has the header's
parameter list. No Rust toolchain is needed: both texts are parsed."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# scalar types: (size, alignment, class)
C_SCALARS = {"int32_t": (4, 4, "i32"), "int64_t": (8, 8, "i64"), "uint32_t": (4, 4, "u32"), "uint8_t": (1, 1, "u8"),
             "double": (8, 8, "f64"), "char": (1, 1, "c_char"), "int": (4, 4, "c_int")}
RUST_SCALARS = {"i32": (4, 4, "i32"), "i64": (8, 8, "i64"), "u32": (4, 4, "u32"), "u8": (1, 1, "u8"),
                "f64": (8, 8, "f64"), "c_char": (1, 1, "c_char"), "c_int": (4, 4, "c_int")}
SAME_CLASS = {("c_int", "i32"), ("i32", "c_int")}


def _header():
    src = open(os.path.join(ROOT, "include", "rh3t.h")).read()
    return re.sub(r"/\*.*?\*/", "", src, flags=re.S)


def _rust():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```rust\n(.*?)```", text, flags=re.S)
    return "\n".join(b for b in blocks if 'extern "C"' in b)


def _c_field_type(t):
    t = t.replace("const ", "").strip()
    if t.endswith("*"):
        return ("ptr", 8, 8)
    return (C_SCALARS[t][2],) + C_SCALARS[t][:2]


def header_structs():
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", _header(), flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            m = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)", decl)
            base, names = m.group(1), m.group(2)
            for nm in names.split(","):
                nm = nm.strip()
                stars = len(nm) - len(nm.lstrip("*"))
                nm = nm.lstrip("*").strip()
                count = 1
                am = re.match(r"(\w+)\[(\w+)\]", nm)
                if am:
                    nm, count = am.group(1), int(am.group(2))
                cls, size, align = _c_field_type(base + "*" * stars)
                fields.append((nm, cls, size, align, count))
        out[name] = fields
    return out


def _rust_type(t):
    t = t.strip()
    am = re.match(r"\[(.+);\s*(\d+)\]$", t)
    if am:
        cls, size, align, _ = _rust_type(am.group(1))
        return cls, size, align, int(am.group(2))
    if t.startswith("*const") or t.startswith("*mut"):
        return "ptr", 8, 8, 1
    size, align, cls = RUST_SCALARS[t]
    return cls, size, align, 1


def rust_structs():
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\]\s*pub struct (\w+)\s*\{(.*?)\}", _rust(), flags=re.S):
        fields = []
        for nm, ty in re.findall(r"pub (\w+):\s*((?:\[[^\]]*\])|(?:\*(?:const|mut) [\w:]+)|\w+)", body):
            cls, size, align, count = _rust_type(ty)
            fields.append((nm, cls, size, align, count))
        out[name] = fields
    return out


def layout(fields):
    off, offsets, maxa = 0, [], 1
    for _, _, size, align, count in fields:
        off = (off + align - 1) // align * align
        offsets.append(off)
        off += size * count
        maxa = max(maxa, align)
    return offsets, (off + maxa - 1) // maxa * maxa


def _norm_name(n):
    return {"lambda_": "lambda"}.get(n, n)


def test_rust_structs_match_header():
    hs, rs = header_structs(), rust_structs()
    assert set(rs) >= {"rh3t_grid", "rh3t_params", "rh3t_bc", "rh3t_ghost_table", "rh3t_error"}
    for name, rf in rs.items():
        assert name in hs, f"{name} is not declared in rh3t.h"
        hf = hs[name]
        assert [f[0] for f in rf] == [f[0] for f in hf], f"{name}: field names/order differ"
        for a, b in zip(rf, hf):
            assert a[4] == b[4] and a[2] == b[2] and (a[1] == b[1] or (a[1], b[1]) in SAME_CLASS), \
                f"{name}.{a[0]}: {a} vs {b}"
        assert layout(rf) == layout(hf), f"{name}: layout differs"


def test_ctypes_mirror_matches_header(rh):
    from importlib import import_module
    lib = import_module("3t_rh_b200._lib")
    hs = header_structs()
    mirror = {"rh3t_grid": lib.Grid, "rh3t_params": lib.Params, "rh3t_bc": lib.BC, "rh3t_arc": lib.Arc,
              "rh3t_ghost_table": lib.GhostTable, "rh3t_error": lib.Error, "rh3t_instance": lib.Instance,
              "rh3t_tune_entry": lib.TuneEntry}
    assert set(mirror) == set(hs)
    for name, cls in mirror.items():
        offsets, size = layout(hs[name])
        names = [_norm_name(f[0]) for f in cls._fields_]
        assert names == [f[0] for f in hs[name]], name
        assert [getattr(cls, f[0]).offset for f in cls._fields_] == offsets, name
        assert C.sizeof(cls) == size, name


def header_functions():
    out = {}
    for ret, name, args in re.findall(r"(?:^|\n)\s*((?:const\s+)?[\w]+\s*\**)\s*(rh3t_\w+)\s*\(([^)]*)\)\s*;",
                                      _header()):
        params = []
        for a in args.split(","):
            a = a.strip()
            if not a or a == "void":
                continue
            m = re.match(r"(.*?)(\w+)$", a)
            params.append(m.group(1).strip())
        out[name] = (ret.strip(), params)
    return out


RUST_POINTEES = {"c_void": "void", "f64": "double", "u8": "uint8_t", "u32": "uint32_t", "i32": "int32_t",
                 "i64": "int64_t", "c_char": "char"}


def _c_class(t):
    """'ptr:<pointee>' with one 'ptr:' per level of indirection, else the scalar class."""
    t = re.sub(r"\s+", " ", t.strip())
    stars = t.count("*")
    base = t.replace("*", " ").replace("const", " ").split()
    base = base[0] if base else ""
    if stars:
        return "ptr:" * stars + base
    return C_SCALARS[base][2] if base in C_SCALARS else base


def _rust_class(t):
    t = t.strip()
    stars = 0
    while True:
        m = re.match(r"\*(?:const|mut)\s+(.*)$", t)
        if not m:
            break
        stars, t = stars + 1, m.group(1).strip()
    if stars:
        return "ptr:" * stars + RUST_POINTEES.get(t, t)
    return RUST_SCALARS[t][2] if t in RUST_SCALARS else t


def _split_params(args):
    params, depth, cur = [], 0, ""
    for ch in args:
        if ch == "," and depth == 0:
            params.append(cur)
            cur = ""
            continue
        depth += 1 if ch in "[(" else (-1 if ch in "])" else 0)
        cur += ch
    if cur.strip():
        params.append(cur)
    return [p.split(":", 1)[1].strip() for p in params]


def rust_functions():
    block = re.search(r'extern "C"\s*\{(.*?)\n\}', _rust(), flags=re.S).group(1)
    block = re.sub(r"//[^\n]*", "", block)
    out = {}
    for name, args, ret in re.findall(r"pub fn (\w+)\s*\((.*?)\)\s*(?:->\s*([\w:]+))?\s*;", block, flags=re.S):
        out[name] = (ret or "", _split_params(args))
    return out


def test_rust_functions_match_header():
    hf, rf = header_functions(), rust_functions()
    assert len(rf) >= 15
    for name, (rret, rparams) in rf.items():
        assert name in hf, f"{name} is not declared in rh3t.h"
        hret, hparams = hf[name]
        assert len(rparams) == len(hparams), f"{name}: {len(rparams)} parameters vs {len(hparams)}"
        for k, (a, b) in enumerate(zip(rparams, hparams)):
            ca, cb = _rust_class(a), _c_class(b)
            ok = ca == cb or (ca, cb) in SAME_CLASS
            assert ok, f"{name} parameter {k}: rust {a} ({ca}) vs C {b} ({cb})"
        hret_c = "" if hret == "void" else _c_class(hret)
        rret_c = _rust_class(rret) if rret else ""
        assert hret_c == rret_c or (hret_c, rret_c) in SAME_CLASS, f"{name}: returns {rret} vs {hret}"


@pytest.mark.parametrize("name", ["rh3t_error"])
def test_error_message_offset(name):
    """The field the Rust wrapper turns into the panic text sits where the
    header puts it."""
    hs, rs = header_structs(), rust_structs()
    ho, _ = layout(hs[name])
    ro, _ = layout(rs[name])
    hi = [f[0] for f in hs[name]].index("message")
    ri = [f[0] for f in rs[name]].index("message")
    assert ho[hi] == ro[ri] == 32
