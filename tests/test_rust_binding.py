"""The Rust crate's raw bindings (spectral-cuda/src/ffi.rs) against the C ABI,
checked on CPU (there is no Rust toolchain here to compile the crate): every
`extern "C"` function of the header is declared in ffi.rs and nothing else
is, with the same number of arguments; every one is exported by the built
library; and every `#[repr(C)]` record has the header struct's fields in the
header's order."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "spectral_cuda.h")
FFI = os.path.join(ROOT, "spectral-cuda", "src", "ffi.rs")


def _split_top(args):
    """Split an argument list at top-level commas (Rust array types hold ';', not ',')."""
    out, depth, cur = [], 0, ""
    for ch in args:
        if ch in "([<":
            depth += 1
        elif ch in ")]>":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [a.strip() for a in out if a.strip()]


def header_functions():
    s = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for _, name, args in re.findall(r"\n\s*((?:const\s+)?\w+\s*\*?)\s*(sc_\w+)\s*\(([^;]*?)\)\s*;", s):
        args = " ".join(args.split())
        out[name] = 0 if args == "void" else len(_split_top(args))
    return out


def rust_functions():
    s = open(FFI).read()
    block = s[s.index('extern "C" {'):]
    out = {}
    for name, args in re.findall(r"pub fn (\w+)\((.*?)\)\s*(?:->\s*[^;]+)?;", block, flags=re.S):
        out[name] = len(_split_top(args))
    return out


def header_structs():
    s = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(sc_\w+)\s*;", s, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            names = decl.split(",")
            first = names[0].split()
            fields.append(re.sub(r"\[.*", "", first[-1]).lstrip("*"))
            fields += [re.sub(r"\[.*", "", n.strip()).lstrip("*") for n in names[1:]]
        out[name] = fields
    return out


def rust_structs():
    s = open(FFI).read()
    out = {}
    for name, body in re.findall(r"pub struct (Sc\w+)\s*\{(.*?)\}", s, flags=re.S):
        out[name] = re.findall(r"pub (\w+):", body)
    return out


def test_every_function_declared_with_its_arity():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 90
    assert sorted(h) == sorted(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    bad = {n: (h[n], r[n]) for n in h if h[n] != r[n]}
    assert not bad, bad


def test_every_declared_function_is_exported():
    from spectral_b200._lib import LIB_PATH
    lib = C.CDLL(LIB_PATH)
    missing = [n for n in rust_functions() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("c_name", ["sc_primitive", "sc_material", "sc_plane", "sc_beam", "sc_camera",
                                    "sc_vol_weights", "sc_debug_photon", "sc_film_options", "sc_tracer_options",
                                    "sc_screen", "sc_trace_desc", "sc_scene_job", "sc_batch_tuning",
                                    "sc_server_config", "sc_request"])
def test_records_have_the_header_fields_in_order(c_name):
    rs_name = "".join(w.capitalize() for w in c_name.split("_"))
    assert header_structs()[c_name] == rust_structs()[rs_name]
