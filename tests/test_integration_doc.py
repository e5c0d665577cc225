"""The C++ bindings shown in INTEGRATION.md compile against the public header.

Each ```cpp block of the document is wrapped in a function of its own (in an
inner block, so that the names it declares may shadow the caller's), with
the variables the blocks take from their surroundings as parameters and a
stand-in for the two MPI names one block calls, and the whole file is
compiled by g++ with warnings as errors for argument conversions."""
from __future__ import annotations

import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

PRELUDE = """\
#include <cstdint>
#include <cstdio>
#include <vector>
#include "dsmc_b200.h"
// the caller's MPI, for the block that reduces profile sums across ranks
enum { MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD };
static int MPI_Reduce(const void *, void *, int, int, int, int, int) { return 0; }
"""
# what the blocks take from the code around them
PARAMS = ("dsmc_ctx *ctx, int sys, dsmc_settings s, const float *weight, const float *drift, "
          "int64_t n_in, std::vector<uint32_t> in")


def cpp_blocks() -> list[str]:
    text = (ROOT / "INTEGRATION.md").read_text()
    return re.findall(r"```cpp\n(.*?)```", text, flags=re.S)


def test_document_has_cpp_bindings():
    assert len(cpp_blocks()) >= 5


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_bindings_compile_against_the_header(tmp_path):
    parts = [PRELUDE]
    for i, block in enumerate(cpp_blocks()):
        body = "\n".join(line for line in block.splitlines() if not line.startswith("#include"))
        parts.append(f"void binding_{i}({PARAMS}) {{\n  {{\n{body}\n  }}\n}}\n")
    src = tmp_path / "bindings.cpp"
    src.write_text("\n".join(parts))
    res = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                          "-Wno-unused-but-set-variable", "-Wno-unused-parameter", "-Werror=conversion-null",
                          "-Werror=narrowing", f"-I{ROOT / 'include'}", str(src)], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
