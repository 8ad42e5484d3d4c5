"""The C-ABI library loads without a GPU and exports every declared symbol;
the C++ drop-in headers compile."""
import os
import re
import subprocess

import pytest

import mpir_b200 as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "mpir_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mpir_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_all_declared_symbols():
    L = mp.lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name


def test_version_and_errors_without_gpu():
    L = mp.lib()
    assert L.mpir_version() >= 10000
    # host-only entry points work without a device
    assert mp.QDLDL_etree(2, [0, 1, 3], [0, 0, 1])[0] == 1


def test_cpp_dropin_headers_compile(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(
        '#include "MPIR/gmres_ir.hpp"\n#include "MPIR/qdldl.hpp"\n'
        "int main() { GmresLDLIR<float, double, double> s; s.SetTolerance(1e-12);\n"
        "  s.SetMaxIRIterations(5); s.SetMaxGmresIterations(20); return 0; }\n")
    r = subprocess.run(["g++", "-std=c++20", "-fsyntax-only", f"-I{ROOT}/include", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_luir_header_compiles(tmp_path):
    src = tmp_path / "l.cpp"
    src.write_text(
        '#include "qdldl-luir/luir.hpp"\n'
        "int main() { Stats st; long n = 1; long Ap[2] = {0, 1}; long Ai[1] = {0};\n"
        "  double Ax[1] = {2.0}, b[1] = {1.0}, x[1];\n"
        "  if (false) LUIR_QDLDL<float, double, double, double>(n, Ap, Ai, Ax, b, x, &st, 10);\n"
        "  return st.get_num_refinement_steps(); }\n")
    r = subprocess.run(["g++", "-std=c++23", "-fsyntax-only", f"-I{ROOT}/include", str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
