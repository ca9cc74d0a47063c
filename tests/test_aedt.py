"""Ansys Maxwell project input (emg_aedt_*, emagddm_b200.aedt): the
materials, objects and boundaries of an .aedt text project, and their
mapping onto a Gmsh mesh whose physical volumes carry the objects' names.

Known answers: the reference's own AEDT tests on its project file
(test/test_aedt_parsing.cpp:48-164: at least 8 materials, copper
sigma = 5.8e7 and mu_r = 0.999991, B27AV1400 nonlinear with a BH curve from
(0, 0), the N45UH magnet mu_r = 1.0739096, at least 20 boundaries,
VectorPotential1 a 'Vector Potential' of value 0), read where the reference
checkout is present; a small project written here pins every field."""
import os

import numpy as np
import pytest

from emagddm_b200 import _abi, aedt, mesh

REF = os.environ.get("EMG_REFERENCE_DIR", "/root/reference")
MU0 = 4e-7 * np.pi

PROJECT = """$begin 'AnsoftProject'
\t$begin 'Definitions'
\t\t$begin 'Materials'
\t\t\t$begin 'iron_lin'
\t\t\t\tpermeability='1000'
\t\t\t\tconductivity='2000000'
\t\t\t$end 'iron_lin'
\t\t\t$begin 'steel_bh'
\t\t\t\t$begin 'permeability'
\t\t\t\t\tproperty_type='nonlinear'
\t\t\t\t\t$begin 'BHCoordinates'
\t\t\t\t\t\tDimUnits[2: '', '']
\t\t\t\t\t\tPoints[6: 0, 0, 100, 0.5, 1000, 1.5]
\t\t\t\t\t$end 'BHCoordinates'
\t\t\t\t$end 'permeability'
\t\t\t$end 'steel_bh'
\t\t\t$begin 'air'
\t\t\t\tpermittivity='1'
\t\t\t$end 'air'
\t\t\t$begin 'odd'
\t\t\t\tpermeability='mu_core'
\t\t\t$end 'odd'
\t\t$end 'Materials'
\t$end 'Definitions'
\t$begin 'Maxwell3DModel'
\t\t$begin 'GeometryPart'
\t\t\t$begin 'Attributes'
\t\t\t\tName='Core'
\t\t\t\tMaterialValue='"iron_lin"'
\t\t\t\tSolveInside=true
\t\t\t$end 'Attributes'
\t\t$end 'GeometryPart'
\t\t$begin 'GeometryPart'
\t\t\t$begin 'Attributes'
\t\t\t\tName='Air'
\t\t\t\tMaterialValue='"air"'
\t\t\t\tSolveInside=false
\t\t\t$end 'Attributes'
\t\t$end 'GeometryPart'
\t$end 'Maxwell3DModel'
\t$begin 'BoundarySetup'
\t\t$begin 'Boundaries'
\t\t\t$begin 'Outer'
\t\t\t\tBoundType='Vector Potential'
\t\t\t\tEdges(18)
\t\t\t\tValue='0'
\t\t\t$end 'Outer'
\t\t\t$begin 'Coil1'
\t\t\t\tBoundType='Coil'
\t\t\t\tObjects(7)
\t\t\t$end 'Coil1'
\t\t$end 'Boundaries'
\t$end 'BoundarySetup'
$end 'AnsoftProject'
"""


def test_small_project_fields(tmp_path):
    p = tmp_path / "small.aedt"
    p.write_text(PROJECT)
    pr = aedt.AedtProject(str(p))
    assert [m.name for m in pr.materials] == ["iron_lin", "steel_bh", "air", "odd"]
    iron, steel, air, odd = pr.materials
    assert (iron.mu_r, iron.sigma, iron.flags) == (1000.0, 2e6, 0)
    assert steel.flags == aedt.FLAG_NONLINEAR
    np.testing.assert_array_equal(steel.bh, [[0, 0], [100, 0.5], [1000, 1.5]])
    assert steel.mu_r == pytest.approx(0.5 / (MU0 * 100), rel=1e-14)   # initial permeability
    assert (air.mu_r, air.sigma, air.flags) == (1.0, 0.0, 0)
    assert odd.flags == aedt.FLAG_MU_NOT_NUMBER
    assert [(o.name, o.material, o.solve_inside) for o in pr.objects] == [("Core", "iron_lin", True),
                                                                          ("Air", "air", False)]
    assert [(b.name, b.type, b.value) for b in pr.boundaries] == [("Outer", "Vector Potential", "0"),
                                                                  ("Coil1", "Coil", "")]
    nu, sigma = pr.material_arrays(["Air", "Core"])
    np.testing.assert_array_equal(nu, [1.0, 1e-3])
    np.testing.assert_array_equal(sigma, [0.0, 2e6])
    with pytest.raises(KeyError):
        pr.material_arrays(["Shaft"])


def test_malformed_project_is_rejected(tmp_path):
    p = tmp_path / "bad.aedt"
    p.write_text("$begin 'A'\n$begin 'B'\n$end 'A'\n")
    with pytest.raises(_abi.EmgError) as e:
        aedt.AedtProject(str(p))
    assert e.value.code == _abi.EMG_INVALID_INPUT and "unbalanced" in str(e.value)


def test_reference_project_known_answers():
    path = os.path.join(REF, "docs", "project", "Temp.aedt")
    if not os.path.exists(path):
        pytest.skip("reference checkout not present")
    pr = aedt.AedtProject(path)
    assert len(pr.materials) >= 8
    cu = pr.material("copper")
    assert cu.sigma == pytest.approx(58e6, abs=1000) and cu.mu_r == pytest.approx(0.999991, abs=1e-4)
    bh = pr.material("B27AV1400")
    assert bh.flags & aedt.FLAG_NONLINEAR and len(bh.bh) > 0
    assert bh.bh[0, 0] == pytest.approx(0.0, abs=1e-3) and bh.bh[0, 1] == pytest.approx(0.0, abs=1e-3)
    pm = next(m for m in pr.materials if "N45UH" in m.name)
    assert pm.mu_r == pytest.approx(1.0739096, abs=1e-3)
    assert len(pr.boundaries) >= 20
    vp = next(b for b in pr.boundaries if b.name == "VectorPotential1")
    assert (vp.type, vp.value) == ("Vector Potential", "0")


@pytest.mark.parametrize("version", ["2.2", "4.1"])
def test_gmsh_volumes_take_their_materials_from_the_project(tmp_path, version):
    m = mesh.plain_scale(4)
    mp = tmp_path / f"cube{version}.msh"
    mesh.write_gmsh(m, str(mp), version=version, volume_tags=(1, 2), names={1: "Air", 2: "Core", 100: "Outer"})
    r = mesh.read_gmsh(str(mp))
    assert r.material_names == ["Air", "Core"]
    # (the 4.1 writer groups the elements by volume, so compare counts)
    np.testing.assert_array_equal(np.bincount(r.material), np.bincount(m.material))
    p = tmp_path / "small.aedt"
    p.write_text(PROJECT)
    nu, sigma = aedt.AedtProject(str(p)).material_arrays(r.material_names)
    np.testing.assert_array_equal(nu, m.nu)          # the benchmark's own mu_r = 1000 block


@pytest.mark.gpu
def test_project_materials_drive_the_gpu_solve(tmp_path):
    """A perturbed mesh written with named volumes, read back, its nu / sigma
    taken from the project by object name; GPU assembly and Jacobi-PCG agree
    with the oracle's solve of the same system to 1e-8."""
    from oracle import oracle as O
    from tests.helpers import System, oracle_system, solve
    base = mesh.perturbed(mesh.plain_scale(8), amplitude=0.2, seed=3)
    mp = tmp_path / "cube.msh"
    mesh.write_gmsh(base, str(mp), names={1: "Air", 2: "Core"})
    p = tmp_path / "small.aedt"
    p.write_text(PROJECT)
    r = mesh.read_gmsh(str(mp), sources=base.sources)
    r.nu, r.sigma = aedt.AedtProject(str(p)).material_arrays(r.material_names)
    l2g = O.dof_build(r.tets, r.dirichlet, gauge=O.GAUGE_REF)["l2g"]
    s = System(r, l2g)
    rp, col, kv, _, rhs = oracle_system(r, l2g)
    x, out = solve(s.matrix(0), rhs, "cg", tol=1e-12, max_iter=50000, precond=1)
    xo, st, _, res = O.pcg(rp, col, kv, rhs, tol=1e-12, max_iter=50000, precond=1)
    assert out.status == 0 and (st == 0 or res < 1e-11)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
