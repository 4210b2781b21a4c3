"""The Python mirror's ctypes structures have the C ABI's layout: a small C
program compiled against include/dycg.h prints sizeof and offsetof of every
field the mirror declares, and they must agree byte for byte (a drift would
make every call through the mirror read or write the wrong fields)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from dycgraph_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = {
    "dycg_edge": engine.Edge,
    "dycg_options": engine.Options,
    "dycg_batch_stats": engine.BatchStats,
    "dycg_graph_info": engine.GraphInfo,
    "dycg_query_mapping": engine.QueryMapping,
    "dycg_policy_report": engine.PolicyReport,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_c_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "dycg.h"', "int main(void) {"]
    for cname, cls in MIRRORS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname} {f} %zu %zu\\n", offsetof({cname}, {f}), '
                         f"sizeof((({cname} *)0)->{f}));")
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        parts = ln.split()
        if parts[1] == "size":
            got[(parts[0], None)] = (int(parts[2]),)
        else:
            got[(parts[0], parts[1])] = (int(parts[2]), int(parts[3]))
    for cname, cls in MIRRORS.items():
        assert got[(cname, None)] == (ctypes.sizeof(cls),), cname
        for f, _ in cls._fields_:
            d = getattr(cls, f)
            assert got[(cname, f)] == (d.offset, d.size), (cname, f)


def _code_blocks(path, lang):
    import re
    text = open(os.path.join(ROOT, path)).read()
    return re.findall(r"```" + lang + r"\n(.*?)```", text, re.S)


@pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                    reason="no C/C++ compiler")
def test_documented_examples_compile_against_the_header(tmp_path):
    """The README's C example and INTEGRATION.md's C++ shim use only names and
    signatures that include/dycg.h declares (syntax and type check, no link)."""
    (c_example,) = _code_blocks("README.md", "c")
    src = tmp_path / "readme.c"
    src.write_text('#include "dycg.h"\n'
                   "int example(const dycg_edge *dels, size_t nd, const dycg_edge *adds, size_t na,\n"
                   "            uint32_t *dist, uint32_t *parent) {\n" + c_example + "  return 0;\n}\n")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-fsyntax-only", "-I",
                    os.path.join(ROOT, "include"), str(src)], check=True, capture_output=True)
    (shim,) = _code_blocks("INTEGRATION.md", "cpp")
    src = tmp_path / "shim.cpp"
    src.write_text(shim)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I",
                    os.path.join(ROOT, "include"), str(src)], check=True, capture_output=True)
