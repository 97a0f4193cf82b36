"""The Rust FFI module include/hydroflux_gpu.rs against include/hydroflux_gpu.h.

The .rs file holds the FFI declarations a maintainer adds to the Rust crate
to call this library. There is no Rust toolchain here, so it is not
compiled. This test stands in for the compile-time half of that: every C
function of the header is declared in the module, every `extern "C"`
function of the module exists in the header with the same return and
parameter types, and every `#[repr(C)]` struct lists the header struct's
fields in the same order with the same types."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hydroflux_gpu.h")
RUST = os.path.join(ROOT, "include", "hydroflux_gpu.rs")

RUST_SCALARS = {"f64": "double", "i64": "int64_t", "u64": "uint64_t", "i32": "int32_t",
                "c_int": "int", "c_char": "char", "c_void": "void"}


def rust_type(t):
    """Rust FFI type -> normalised C spelling ('const double*', 'hf_sim**')."""
    t = t.strip()
    stars = []
    while t.startswith("*"):
        m = re.match(r"\*(const|mut)\s+(.*)", t)
        stars.append(m.group(1))
        t = m.group(2).strip()
    if t in RUST_SCALARS:
        base = RUST_SCALARS[t]
    else:  # HfMeshDesc -> hf_mesh_desc
        assert t.startswith("Hf"), t
        base = "hf" + re.sub(r"([A-Z])", lambda m: "_" + m.group(1).lower(), t[2:])
    # the pointer next to the base carries the base's constness
    if stars and stars[-1] == "const":
        base = "const " + base
    return base + "*" * len(stars)


def c_type(t):
    t = re.sub(r"\s+", " ", t.strip())
    t = re.sub(r"\s*\*\s*", "*", t)
    return t


def strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def header():
    src = strip_c_comments(open(HEADER).read())
    structs = {}
    for m in re.finditer(r"typedef struct (\w+) \{(.*?)\} (\w+);", src, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            fm = re.match(r"(.*?)(\w+)\s*$", decl, flags=re.S)
            fields.append((fm.group(2), c_type(fm.group(1))))
        structs[m.group(3)] = fields
    funcs = {}
    for m in re.finditer(r"([\w\s\*]+?)\b(hf_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        ret = c_type(ret.replace("extern", "").replace("HF_API", ""))
        params = []
        if args and args != "void":
            for a in args.split(","):
                am = re.match(r"(.*?)(\w+)\s*$", a.strip(), flags=re.S)
                params.append(c_type(am.group(1)))
        funcs[name] = (ret, params)
    return structs, funcs


def shim():
    structs, funcs = {}, {}
    for block in [open(RUST).read()]:
        code = re.sub(r"//[^\n]*", " ", block)
        for m in re.finditer(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}",
                             code, flags=re.S):
            fields = []
            for f in m.group(2).split(","):
                f = f.strip()
                if f:
                    fm = re.match(r"pub (\w+)\s*:\s*(.+)$", f, flags=re.S)
                    fields.append((fm.group(1), rust_type(fm.group(2))))
            structs[m.group(1)] = fields
        for ext in re.findall(r'extern "C" \{(.*?)\n\}', code, flags=re.S):
            for m in re.finditer(r"pub fn (\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", ext, flags=re.S):
                params = []
                for a in m.group(2).split(","):
                    a = a.strip()
                    if a:
                        params.append(rust_type(a.split(":", 1)[1]))
                ret = rust_type(m.group(3)) if m.group(3) else "void"
                funcs[m.group(1)] = (ret, params)
    return structs, funcs


def test_parsers_see_the_shim():
    s_structs, s_funcs = shim()
    h_structs, h_funcs = header()
    assert len(s_funcs) >= 60 and len(s_structs) >= 7
    assert "hf_sim_create_aos" in h_funcs and "hf_config" in h_structs


def test_module_declares_every_header_function_and_struct():
    s_structs, s_funcs = shim()
    h_structs, h_funcs = header()
    assert sorted(h_funcs) == sorted(s_funcs)
    assert sorted(h_structs) == sorted(rust_type(r) for r in s_structs)


def test_shim_functions_match_the_header():
    _, s_funcs = shim()
    _, h_funcs = header()
    for name, (ret, params) in sorted(s_funcs.items()):
        assert name in h_funcs, f"{name} is not declared in the header"
        assert h_funcs[name] == (ret, params), (name, h_funcs[name], (ret, params))


def test_shim_structs_match_the_header():
    s_structs, _ = shim()
    h_structs, _ = header()
    for rname, fields in sorted(s_structs.items()):
        cname = rust_type(rname)
        assert cname in h_structs, f"{cname} is not a header struct"
        assert fields == h_structs[cname], (rname, fields, h_structs[cname])


@pytest.mark.parametrize("t,want", [("*const f64", "const double*"),
                                    ("*mut *mut HfSim", "hf_sim**"),
                                    ("*const HfScenarioDesc", "const hf_scenario_desc*"),
                                    ("c_int", "int"), ("*const c_char", "const char*")])
def test_rust_type_mapping(t, want):
    assert rust_type(t) == want
