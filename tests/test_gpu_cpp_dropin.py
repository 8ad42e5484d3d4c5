"""The C++ drop-in executed: a caller written against the reference's headers
(include/MPIR/gmres_ir.hpp and include/MPIR/qdldl.hpp of this project, which
keep the reference's templates) is compiled with g++, linked against
libmpir_b200.so and run on the GPU.

It follows the reference's example driver (examples/example.cpp:140-174:
GmresLDLIR<double, double, dd_real> with tolerance 1e-15, 200 refinement
steps of 50 GMRES iterations, Compute then Solve, errors printed), then the
float factor instantiation GmresLDLIR<float, double, double>, then the
QDLDL usage of LUIR_QDLDL (qdldl-luir/luir.hpp:79-177: QDLDL_etree,
QDLDL_factor<long, float>, QDLDL_solve<long, float, double>).  Each result
must reach backward error <= 1e-14 (the plain LDL^T solve: the float factor's
accuracy, <= 1e-5 relative residual)."""
import os
import subprocess

import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CALLER = r'''
#include <cmath>
#include <cstdio>
#include <fstream>
#include <vector>
#include "MPIR/gmres_ir.hpp"
#include "MPIR/qdldl.hpp"

template <class T> static std::vector<T> rd(std::ifstream &f, size_t k) {
  std::vector<T> v(k); f.read(reinterpret_cast<char *>(v.data()), k * sizeof(T)); return v;
}
static double berr(const std::vector<size_t> &Ap, const std::vector<size_t> &Ai,
                   const std::vector<double> &Ax, const std::vector<double> &x,
                   const std::vector<double> &b) {
  std::vector<double> r = MatrixMultiply<double>(Ap, Ai, Ax, x), rowsum(x.size(), 0.0);
  double rn = 0, xn = 0, bn = 0, an = 0;
  const size_t n = x.size();
  for (size_t j = 0; j < n; j++)
    for (size_t p = Ap[j]; p < Ap[j + 1]; p++) {
      rowsum[j] += std::fabs(Ax[p]);
      if (Ai[p] != j) rowsum[Ai[p]] += std::fabs(Ax[p]);
    }
  for (size_t i = 0; i < n; i++) {
    rn = std::fmax(rn, std::fabs(b[i] - r[i])); xn = std::fmax(xn, std::fabs(x[i]));
    bn = std::fmax(bn, std::fabs(b[i])); an = std::fmax(an, rowsum[i]);
  }
  return rn / (an * xn + bn);
}
int main(int argc, char **argv) {
  std::ifstream f(argv[1], std::ios::binary);
  long n, nnz;
  f.read(reinterpret_cast<char *>(&n), 8); f.read(reinterpret_cast<char *>(&nnz), 8);
  auto ap = rd<long>(f, n + 1); auto ai = rd<long>(f, nnz); auto Ax = rd<double>(f, nnz);
  auto b = rd<double>(f, n); auto xt = rd<double>(f, n);
  std::vector<size_t> Ap(ap.begin(), ap.end()), Ai(ai.begin(), ai.end());
  auto ferr = [&](const std::vector<double> &x) {
    double d = 0, m = 0;
    for (long i = 0; i < n; i++) { d = std::fmax(d, std::fabs(x[i] - xt[i])); m = std::fmax(m, std::fabs(xt[i])); }
    return d / m;
  };
  {
    GmresLDLIR<double, double, mpir::double_double> solver;
    solver.SetTolerance(1e-15);
    solver.SetMaxIRIterations(200);
    solver.SetMaxGmresIterations(50);
    solver.Compute<double, 1 << 21, 5, 2048>(Ap, Ai, Ax, 0);
    std::vector<double> x = solver.Solve(b);
    std::printf("gmres_double_dd %.3e %.3e %d\n", berr(Ap, Ai, Ax, x, b), ferr(x),
                solver.LastReport().factor_prec);
  }
  {
    GmresLDLIR<float, double, double> solver;
    solver.Compute<double>(Ap, Ai, Ax, 0);
    std::vector<double> x = solver.Solve(b);
    std::printf("gmres_float %.3e %.3e %zu\n", berr(Ap, Ai, Ax, x, b), ferr(x),
                solver.Solve(std::vector<double>(n - 1)).size());
  }
  {
    std::vector<long> work(n), Lnz(n), etree(n);
    long sum = QDLDL_etree<long>(n, ap.data(), ai.data(), work.data(), Lnz.data(), etree.data());
    std::vector<long> Lp(n + 1), Li(sum), iwork(3 * n);
    std::vector<float> Axf(Ax.begin(), Ax.end()), Lx(sum), D(n), Dinv(n), fwork(n);
    std::vector<char> bw(n);
    long pos = QDLDL_factor<long, float>(n, ap.data(), ai.data(), Axf.data(), Lp.data(), Li.data(),
                                         Lx.data(), D.data(), Dinv.data(), Lnz.data(), etree.data(),
                                         reinterpret_cast<bool *>(bw.data()), iwork.data(), fwork.data());
    std::vector<double> x(b);
    QDLDL_solve<long, float, double>(n, Lp.data(), Li.data(), Lx.data(), Dinv.data(), x.data());
    std::printf("qdldl_float %.3e %.3e %ld\n", berr(Ap, Ai, Ax, x, b), ferr(x), pos);
    long r64 = QDLDL_factor<long, double>(n, ap.data(), ai.data(), Ax.data(), Lp.data(), Li.data(),
                                          nullptr, nullptr, nullptr, Lnz.data(), etree.data(),
                                          nullptr, nullptr, nullptr);
    std::printf("qdldl_double_status %ld\n", r64);
  }
  return 0;
}
'''


def test_cpp_caller_links_and_solves(tmp_path):
    s = kkt.small2d(seed=3)
    path = tmp_path / "sys.bin"
    with open(path, "wb") as f:
        np.array([s.n, s.nnz], np.int64).tofile(f)
        s.Ap.astype(np.int64).tofile(f)
        s.Ai.astype(np.int64).tofile(f)
        s.Ax.tofile(f)
        s.b.tofile(f)
        s.x_true.tofile(f)
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "mpir_b200")
    mp.lib()  # the library is built
    r = subprocess.run(["g++", "-std=c++23", "-O1", f"-I{ROOT}/include", str(src), "-o", str(exe),
                        f"-L{libdir}", "-lmpir_b200", f"-Wl,-rpath,{libdir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    out = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines() if ln.strip()}
    be, fe, fprec = out["gmres_double_dd"]
    assert float(be) <= 1e-14 and int(fprec) == mp.F32
    be, fe, empty = out["gmres_float"]
    assert float(be) <= 1e-14 and int(empty) == 0  # size mismatch: empty vector
    be, fe, pos = out["qdldl_float"]
    assert float(be) <= 1e-5 and int(pos) == int(np.sum(s.Ax[np.diff(s.Ap).cumsum() - 1] > 0))
    assert int(out["qdldl_double_status"][0]) == -7
