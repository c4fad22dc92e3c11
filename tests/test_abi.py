"""The C ABI library loads and exports every entry point include/gpl.h declares (no GPU)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "gpl.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gpl_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_command_and_kernels():
    names = declared()
    for n in ["gpl_create", "gpl_destroy", "gpl_global_placement", "gpl_result_free", "gpl_set_option",
              "gpl_kernel_density_scatter", "gpl_kernel_poisson", "gpl_kernel_wa", "gpl_kernel_bicgstab", "gpl_kernel_rudy"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from gpl_b200 import build
    so = build.build()
    lib = C.CDLL(so)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from gpl_b200 import engine, synth
    with pytest.raises(engine.EngineUnavailable):
        engine.global_placement(synth.generate("cfg1"), [])


def _c_fields(src, name):
    body = re.search(r"typedef struct %s \{(.*?)\} %s_t;" % (name, name), src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        if "(*" in decl:
            out.append(re.search(r"\(\*\s*(\w+)\)", decl).group(1))
            continue
        for part in decl.split(","):
            out.append(re.search(r"(\w+)\s*(\[\d+\])?\s*$", part.strip()).group(1))
    return out


def _rust_fields(md, name):
    body = re.search(r"pub struct %s \{(.*?)\n\}" % name, md, re.S).group(1)
    return re.findall(r"pub (\w+):", body)


@pytest.mark.parametrize("c_name,rust_name", [("gpl_design", "GplDesign"), ("gpl_router", "GplRouter"), ("gpl_result", "GplResult")])
def test_rust_binding_fields_follow_the_header(c_name, rust_name):
    """The Rust structs INTEGRATION.md gives name every field of the C structs, in their order
    (a layout check by name; no Rust compiler is available to check types)."""
    src = open(os.path.join(ROOT, "include", "gpl.h")).read()
    md = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    assert _rust_fields(md, rust_name) == _c_fields(src, c_name)
