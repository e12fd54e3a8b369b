"""The reference-side code of INTEGRATION.md compiles.

Each ```cpp / ```c block is compiled (syntax only) against include/pcg.h and,
for the C++ ones, the reference's own headers with the shim defines of
oracle/ref_shim, so that the GpuDomain / GpuSpecieP bindings name members
the reference's classes really have.  Fragments are wrapped in a function
that has a handle `h` (and a `slot`); the GpuSpecieP method gets a class
declaration around it.  Skipped where the reference's headers are absent
($PICOPIC_REFERENCE, or the checkout the last
oracle build compiled) or no compiler is installed.
"""
import os
import re
import shutil
import subprocess

import pytest

from oracle.harness import reference_root

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = reference_root()


def blocks():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as f:
        text = f.read()
    return [(lang, body) for lang, body in re.findall(r"```(\w+)\n(.*?)```", text, re.S) if lang in ("c", "cpp")]


def wrap(lang: str, body: str) -> str:
    if "#include" in body:  # a whole translation unit
        extra = "\nvoid GpuDomain::upload(std::vector<SpecieP*>&) {}\n" if "class GpuDomain" in body else ""
        return body + extra
    if lang == "c":
        return '#include <stddef.h>\n#include "pcg.h"\nvoid snippet(void) {\n' + body + "\n}\n"
    head = '#include "pcg.h"\n#include "domain.hpp"\nusing namespace constant;\n'
    if "GpuSpecieP::" in body:
        return (head + "struct GpuSpecieP : SpecieP {\n  pcg_handle* h;\n  int slot;\n"
                "  void calc_temperature();\n};\n" + body)
    return head + "void snippet(pcg_handle* h, int slot) {\n(void)slot;\n" + body + "\n}\n"


def test_integration_snippets_compile(tmp_path):
    if not REF or not os.path.isdir(os.path.join(REF, "include")):
        pytest.skip("the reference's headers are not here")
    if not shutil.which("g++") or not shutil.which("gcc"):
        pytest.skip("no host compiler")
    found = blocks()
    assert len(found) >= 4
    for k, (lang, body) in enumerate(found):
        src = tmp_path / f"snippet{k}.{'c' if lang == 'c' else 'cpp'}"
        src.write_text(wrap(lang, body))
        if lang == "c":
            cmd = ["gcc", "-std=c11", "-fsyntax-only", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src)]
        else:
            cmd = ["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "oracle", "ref_shim"),
                   "-I", os.path.join(REF, "include"), "-I", os.path.join(ROOT, "include"), str(src)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, f"block {k} ({lang}):\n{body}\n{r.stderr[-2000:]}"
