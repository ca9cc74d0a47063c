"""The reference-side binding of the GPU Krylov solvers (tests/cpp/
reference_binding.cpp): numeric::GpuCGSolver derives from the reference's own
EMLinearSolverBase and takes its CsrMatrix<double> and CGConfig.

* CPU: it compiles against the reference's headers (oracle/Makefile.ref,
  where the reference checkout is present).
* GPU: solving through the reference's interface gives the reference
  CGSolver's results (both built from the same CsrMatrix): status SUCCESS,
  solutions within 1e-8 relative, iteration counts within the usual margin
  for NONE and JACOBI (ILU0 differs by design: ILU(0) against the
  reference's IncompleteLUT).
"""
import os
import subprocess

import numpy as np
import pytest

from emagddm_b200 import mesh
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "reference_binding")
REF = os.environ.get("EMG_REFERENCE_DIR", "/root/reference")


def test_binding_compiles_against_the_reference_headers():
    if not os.path.isdir(os.path.join(REF, "include", "numeric")):
        pytest.skip("reference checkout not present")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "-f", "Makefile.ref",
                           f"REF={REF}", "../tests/cpp/reference_binding"])
    assert os.access(BIN, os.X_OK)


@pytest.mark.gpu
def test_binding_solves_like_the_reference(tmp_path):
    if not os.access(BIN, os.X_OK):
        pytest.skip("binding not built (needs the reference headers at build time)")
    m = mesh.plain_scale(6)
    l2g = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    rp, col, kv, _, rhs = O.assemble(m, l2g, int(l2g.max()) + 1)
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    path = tmp_path / "system.txt"
    with open(path, "w") as f:
        f.write(f"{n} {kv.size}\n")
        for i, j, v in zip(rows, col, kv):
            f.write(f"{i} {j} {v!r}\n")
        for v in rhs:
            f.write(f"{v!r}\n")
    out = subprocess.run([BIN, str(path)], capture_output=True, text=True, timeout=300, check=True).stdout
    res = {}
    for line in out.splitlines():
        p = line.split()
        if len(p) == 6 and p[0] in ("GpuCG", "CGSolver"):
            res[(p[0], p[1])] = (int(p[2]), int(p[3]), float(p[4]), float(p[5]))
    for pc in ("none", "jacobi", "ilu0"):
        g, r = res[("GpuCG", pc)], res[("CGSolver", pc)]
        assert g[0] == r[0] == 0, (pc, g, r)
        assert g[2] < 1e-10
        assert g[3] <= 1e-8, (pc, g)
        if pc != "ilu0":
            assert abs(g[1] - r[1]) <= max(3, 0.15 * r[1]), (pc, g, r)
