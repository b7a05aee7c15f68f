"""The C-ABI library loads and exports every entry point include/pawsim_b200.h declares,
and the ctypes mirror of the config struct has the header's fields in order (no GPU work)."""
import ctypes
import os
import re

import pawsim_b200

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pawsim_b200.h")


def declared():
    src = open(HDR).read()
    return re.findall(r"PAWSIM_API\s+[\w\s\*]+?\b(pawsim_\w+)\s*\(", src)


def test_every_declared_symbol_is_exported():
    lib = pawsim_b200.load_library()
    names = declared()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n


def test_config_struct_matches_header():
    src = open(HDR).read()
    body = re.search(r"typedef struct pawsim_gpu_config\s*\{(.*?)\}\s*pawsim_gpu_config;", src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, rest = decl.split(None, 1)
        fields += [(n.strip(), typ) for n in rest.split(",")]
    got = [(n, "int" if t is ctypes.c_int else "double") for n, t in pawsim_b200.GpuConfig._fields_]
    assert got == fields
