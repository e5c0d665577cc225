"""The ctypes binding (master_b200/capi.py) against the C headers: every
entry point of include/*.h has a ctypes signature with the header's number
of parameters, the same scalar type in every scalar position, a pointer in
every pointer position and the header's return type, so no call through the
binding passes, say, a 32-bit int where the library reads an int64_t."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from master_b200 import capi

ROOT = Path(__file__).resolve().parents[1]

SCALARS = {"int": C.c_int, "int64_t": C.c_int64, "uint64_t": C.c_uint64, "uint32_t": C.c_uint32,
           "double": C.c_double, "float": C.c_float, "unsigned": C.c_uint}
RETURNS = {"int": C.c_int, "void": None, "const char *": C.c_char_p, "void *": C.c_void_p}
PROTOTYPE = re.compile(r"^(int|void|const char|void)\s*(\*?)\s*(dsmc_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", re.M)


def prototypes(header: str) -> dict[str, tuple[str, list[str]]]:
    """name -> (return type, parameters) of every function the header declares."""
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for ret, star, name, params in PROTOTYPE.findall(text):
        ps = [" ".join(p.split()) for p in params.split(",")]
        out[name] = (ret + (" *" if star else ""), [] if ps in (["void"], [""]) else ps)
    return out


def is_pointer_type(t) -> bool:
    return t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, C._Pointer))


@pytest.mark.parametrize("header", ["dsmc_b200.h", "dsmc_surrogate.h"])
def test_every_binding_matches_its_prototype(header):
    lib = capi.load()
    protos = prototypes(header)
    declared = capi.EXPORTED if header == "dsmc_b200.h" else capi.EXPORTED_SURROGATE
    assert set(protos) == set(declared), "the parser must find every declared entry point"
    for name, (ret, params) in protos.items():
        fn = getattr(lib, name)
        assert fn.restype is RETURNS[ret], f"{name} returns {ret}, ctypes has {fn.restype}"
        args = fn.argtypes
        assert args is not None, f"{name}: no ctypes signature"
        assert len(args) == len(params), f"{name}: {len(args)} ctypes arguments for {len(params)} parameters"
        for i, (p, t) in enumerate(zip(params, args)):
            if "*" in p or "[" in p:
                assert is_pointer_type(t), f"{name} argument {i} ({p}) is a pointer, ctypes has {t}"
            else:
                ctype = " ".join(w for w in p.split()[:-1] if w != "const")
                assert ctype in SCALARS, f"{name} argument {i}: unknown type {ctype}"
                assert t is SCALARS[ctype], f"{name} argument {i} ({p}): ctypes has {t}"
