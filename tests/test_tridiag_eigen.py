"""The library's host eigensolver for the duct's z operator (csrc/tridiag_eigen.h; the reference calls LAPACK dstev at
src/initialization.f90:605): compiled here with g++ and checked against numpy's symmetric eigensolver on random and
Neumann-type tridiagonal matrices up to the 512-cell limit of the duct path."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dopamine-fdm_b200", "csrc")

HARNESS = r"""
#include "tridiag_eigen.h"
#include <cstdio>
int main() {
    int n;
    if (std::scanf("%d", &n) != 1) return 2;
    std::vector<double> d(n), e(n > 0 ? n - 1 : 0), q;
    for (auto &x : d) if (std::scanf("%lf", &x) != 1) return 2;
    for (auto &x : e) if (std::scanf("%lf", &x) != 1) return 2;
    if (!dfdm::tridiag_eigen(d, e, q)) return 1;
    for (int m = 0; m < n; ++m) std::printf("%.17g\n", d[m]);
    for (size_t i = 0; i < q.size(); ++i) std::printf("%.17g\n", q[i]);
    return 0;
}
"""


@pytest.fixture(scope="module")
def solver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    d = tmp_path_factory.mktemp("eig")
    src = d / "eig.cpp"
    src.write_text(HARNESS)
    exe = d / "eig"
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True)

    def run(diag, off):
        n = len(diag)
        text = f"{n}\n" + "\n".join(repr(float(x)) for x in list(diag) + list(off)) + "\n"
        out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True).stdout.split()
        vals = np.array([float(x) for x in out])
        return vals[:n], vals[n:].reshape(n, n)
    return run


def neumann_operator(n, rng):
    """The symmetrised second difference with Neumann end rows on a stretched grid, as the duct builds it."""
    f = np.cumsum(0.5 + rng.random(n + 1))                  # faces
    w = np.diff(f)                                          # cell widths
    c = 0.5 * (f[1:] + f[:-1])                              # centres
    h = np.diff(c)                                          # centre spacings
    diag = np.zeros(n)
    diag[1:] -= 1.0 / (w[1:] * h)
    diag[:-1] -= 1.0 / (w[:-1] * h)
    off = 1.0 / (h * np.sqrt(w[:-1] * w[1:]))
    return diag, off


@pytest.mark.parametrize("n,kind", [(1, "random"), (2, "random"), (17, "random"), (129, "random"), (511, "random"),
                                    (17, "neumann"), (129, "neumann"), (512, "neumann")])
def test_tridiag_eigen_matches_numpy(solver, n, kind):
    rng = np.random.default_rng(n)
    if kind == "random":
        diag, off = rng.standard_normal(n) * 5.0, rng.standard_normal(max(n - 1, 0)) * 2.0
    else:
        diag, off = neumann_operator(n, rng)
    lam, q = solver(diag, off)
    T = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    want = np.linalg.eigvalsh(T)
    scale = max(np.max(np.abs(want)), 1e-300)
    assert np.all(np.diff(lam) >= 0.0)                                  # ascending, as dstev returns them
    assert np.max(np.abs(lam - want)) <= 1e-13 * scale
    assert np.max(np.abs(T @ q - q * lam[None, :])) <= 1e-13 * scale   # eigenpairs
    assert np.max(np.abs(q.T @ q - np.eye(n))) <= 1e-12                 # orthonormal
    if kind == "neumann":   # the constant null vector of Dzz: the smallest eigenvalue in magnitude vanishes
        assert np.min(np.abs(lam)) <= 1e-12 * scale
