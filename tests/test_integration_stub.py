"""The Rust binding shown in INTEGRATION.md against the C header.

The reference's host is Rust and cannot be compiled here, so the FFI stub a
maintainer would paste into the reference is checked as text: its two
#[repr(C)] structs must list the header's fields in the header's order with
the same types, and every function its extern "C" block declares must exist
in the header with the same parameter and return types.
"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fluid_step.h")
DOC = os.path.join(ROOT, "INTEGRATION.md")

C_SCALAR = {"float": "f32", "double": "f64", "uint32_t": "u32", "int32_t": "i32",
            "uint64_t": "u64", "int": "c_int", "size_t": "usize", "char": "c_char",
            "void": "c_void", "fe_ctx": "c_void", "fe_params": "FeParams",
            "fe_stats": "FeStats", "fe_status": "c_int", "fe_field": "c_int"}


def _strip_c_comments(text):
    return re.sub(r"/\*.*?\*/", "", text, flags=re.S)


def _rust_block():
    text = open(DOC).read()
    blocks = re.findall(r"```rust\n(.*?)```", text, flags=re.S)
    assert blocks, "no rust block in INTEGRATION.md"
    return blocks[0]


def c_struct_fields(name):
    text = _strip_c_comments(open(HEADER).read())
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S)
    assert m, name
    out = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        mm = re.fullmatch(r"(\w+)\s+(\w+)(?:\[(\d+)\])?", decl)
        assert mm, decl
        ty = C_SCALAR[mm.group(1)]
        out.append((mm.group(2), f"[{ty}; {mm.group(3)}]" if mm.group(3) else ty))
    return out


def rust_struct_fields(name):
    m = re.search(r"pub struct %s \{(.*?)\}" % name, _rust_block(), flags=re.S)
    assert m, name
    out = []
    for item in re.findall(r"pub (\w+): ([^,]+?)\s*(?:,|$)", m.group(1).strip()):
        out.append((item[0], re.sub(r"\s+", " ", item[1]).strip()))
    return out


def c_type_to_rust(decl):
    """'const fe_params* p' -> '*const FeParams' (the parameter name dropped)."""
    decl = decl.strip()
    const = decl.startswith("const ")
    if const:
        decl = decl[len("const "):]
    m = re.fullmatch(r"(\w+)\s*(\**)\s*\w*", decl)
    assert m, decl
    base, stars = C_SCALAR.get(m.group(1), m.group(1)), len(m.group(2))
    if stars == 0:
        return base
    ty = ("*const " if const else "*mut ") + base
    for _ in range(stars - 1):
        ty = "*mut " + ty
    return ty


def c_functions():
    text = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"FE_API\s+([\w\s\*]+?)\s*(\bfe_\w+)\s*\(([^)]*)\)\s*;", text):
        ret = m.group(1).strip()
        args = [a for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        out[m.group(2)] = (c_type_to_rust(ret + " r") if ret != "void" else None,
                           [c_type_to_rust(a) for a in args])
    return out


def rust_functions():
    m = re.search(r'extern "C" \{(.*?)\n\}', _rust_block(), flags=re.S)
    assert m
    out = {}
    for f in re.finditer(r"pub fn (\w+)\((.*?)\)\s*(?:->\s*([^;]+))?;", m.group(1), flags=re.S):
        args = []
        for a in f.group(2).split(","):
            if a.strip():
                args.append(re.sub(r"\s+", " ", a.split(":", 1)[1]).strip())
        out[f.group(1)] = (f.group(3).strip() if f.group(3) else None, args)
    return out


def test_rust_structs_match_the_header():
    for c_name, r_name in (("fe_params", "FeParams"), ("fe_stats", "FeStats")):
        assert rust_struct_fields(r_name) == c_struct_fields(c_name), r_name


def test_rust_extern_block_matches_the_header():
    header = c_functions()
    rust = rust_functions()
    assert len(rust) >= 10
    for name, (ret, args) in rust.items():
        assert name in header, f"{name} is not in include/fluid_step.h"
        assert (ret, args) == header[name], (name, (ret, args), header[name])
