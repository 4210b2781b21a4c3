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


@pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None,
                    reason="no C/C++ compiler")
def test_examples_compile_against_the_header():
    """The C usage example and the reference-side C++ shim (tests/examples/,
    the code the README and the integration guide show) use only names and
    signatures that include/dycg.h declares (syntax and type check, no link)."""
    ex = os.path.join(ROOT, "tests", "examples")
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-fsyntax-only", "-I", inc,
                    os.path.join(ex, "readme_example.c")], check=True, capture_output=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", inc,
                    os.path.join(ex, "integration_shim.cpp")], check=True, capture_output=True)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_operator_structs_state_the_python_operators(tmp_path):
    """include/dycg_operators.h (the kernels' edge-weight rule) and
    dycgraph_b200/operators.py state the same traits and rules."""
    import numpy as np
    from dycgraph_b200 import operators
    rng = np.random.default_rng(5)
    pts = [(int(a), int(b)) for a, b in rng.integers(0, 1 << 32, (40, 2))] + [(0, 0), (7, 7), (1, 2)]
    src = ['#include <cstdio>', '#include "dycg_operators.h"', "using namespace dycg_ops;",
           "template <class O> void dump(const char *n, unsigned long long u, unsigned long long v) {",
           '  std::printf("%s %llu %llu %u %u %u %u %d %d %d %d %d\\n", n, u, v,',
           "    O::TraversalEdgeWeight(u, v), O::DeletionEdgeWeight(u, v),",
           "    O::GetInitBuffer(u, v), O::GetInitValue(u, v),",
           "    (int)O::kSupportsGpuDeletionRepair, (int)O::kVertexSeeds,",
           "    (int)O::kRootedDeletionWitness, (int)O::kSignedResidual,",
           "    (int)O::IsDeletionDependency(u, v, u % 5, v % 5, v % 5, u, false));", "}",
           "int main() {"]
    for u, v in pts:
        for name in ("SSSP", "BFS", "CC", "PR"):
            src.append(f'  dump<{name}>("{name}", {u}ull, {v}ull);')
    src += ["  return 0;", "}"]
    (tmp_path / "ops.cpp").write_text("\n".join(src) + "\n")
    exe = tmp_path / "ops"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    str(tmp_path / "ops.cpp"), "-o", str(exe)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        name, u, v, tw, dw, ib, iv, gpu, seeds, witness, signed, dep = line.split()
        u, v = int(u), int(v)
        O = operators.BY_NAME[name.lower()]
        assert int(tw) == O.TraversalEdgeWeight(u, v) % (1 << 32), line
        assert int(dw) == O.DeletionEdgeWeight(u, v) % (1 << 32), line
        want_ib = O.GetInitBuffer(u, v) if hasattr(O, "GetInitBuffer") else operators.INF
        assert int(ib) == want_ib and int(iv) == O.GetInitValue(u, v), line
        assert (int(gpu), int(seeds), int(witness), int(signed)) == (
            O.kSupportsGpuDeletionRepair, O.kVertexSeeds, O.kRootedDeletionWitness,
            O.kSignedResidual), line
        assert bool(int(dep)) == bool(O.IsDeletionDependency(u, v, u % 5, v % 5, v % 5, u, False)), line
