"""Synthetic structured tetrahedral and hexahedral meshes of the unit cube.

The reference solve path consumes an ``fe_em::EMMeshData`` (nodes, TET4_EDGE
elements with a material id, and a DIRICHLET / VECTOR_EDGE_ONLY boundary
marker holding edge node pairs; ``include/fe_em/em_mesh_data.hpp:90-230``).
This module builds the same data as flat numpy arrays for an n^3 hex grid with
every hex split into 6 tetrahedra (Kuhn split), the layout every test and the
benchmark use:

* node gid = i + (n+1) * (j + (n+1) * k), coordinates (i, j, k) / n;
* hexes in k -> j -> i order; hex vertices v0..v7 = (i,j,k), (i+1,j,k),
  (i+1,j+1,k), (i,j+1,k) and the same at k+1;
* tets per hex {0,1,2,6}, {0,2,3,6}, {0,3,7,6}, {0,7,4,6}, {0,4,5,6}, {0,5,1,6};
* Dirichlet edges: every mesh edge lying in a boundary face (n x A = 0).

The ``hex_*`` variants keep the hexes themselves as HEX8_EDGE elements
(vertex order v0..v7 above, ElementGeometry's HEX8 order); a ``CubeMesh``
whose ``tets`` array has 8 columns is a hex mesh.  The ``prism_*`` variants
split every hex into two PRISM6_EDGE elements (triangles (v0, v1, v2) and
(v0, v2, v3) extruded along z; nodes bottom 0-2, top 3-5), the ``pyramid_*``
variants into six PYRAMID5_EDGE elements, one per hex face, with the apex at
an added node in the hex centre (gid (n+1)^3 + hex index).  The element
type follows the number of columns of ``tets``: 4, 8, 6 or 5.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from functools import lru_cache

import numpy as np

KUHN = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6],
                 [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]], dtype=np.int64)
# TET4 local edges, ElementGeometry::get_local_edges(TET4)
GEO_EDGES = np.array([[0, 1], [1, 2], [0, 2], [0, 3], [1, 3], [2, 3]], dtype=np.int64)
# HEX8 local edges, ElementGeometry::get_local_edges(HEX8)
HEX_EDGES = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6], [6, 7], [7, 4],
                      [0, 4], [1, 5], [2, 6], [3, 7]], dtype=np.int64)
# PRISM6 and PYRAMID5 local edges, ElementGeometry::get_local_edges
PRISM_EDGES = np.array([[0, 1], [1, 2], [0, 2], [3, 4], [4, 5], [3, 5], [0, 3], [1, 4], [2, 5]], dtype=np.int64)
PYRAMID_EDGES = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [0, 4], [1, 4], [2, 4], [3, 4]], dtype=np.int64)
# Element types (same values as the C ABI's EMG_ELEM_*).
ELEM_TET4_EDGE = 0
ELEM_HEX8_EDGE = 1
ELEM_PRISM6_EDGE = 2
ELEM_PYRAMID5_EDGE = 3
# mixed mesh: rows of 9 ints (8 node slots, -1 past the element's nodes, then
# its type), 12 edge slots per element in l2g (-1 past the element's edges)
ELEM_MIXED = 4
TYPE_OF_NODES = {4: ELEM_TET4_EDGE, 8: ELEM_HEX8_EDGE, 6: ELEM_PRISM6_EDGE, 5: ELEM_PYRAMID5_EDGE,
                 9: ELEM_MIXED}
EDGES_OF_TYPE = {ELEM_TET4_EDGE: 6, ELEM_HEX8_EDGE: 12, ELEM_PRISM6_EDGE: 9, ELEM_PYRAMID5_EDGE: 8,
                 ELEM_MIXED: 12}
NODES_OF_TYPE = {ELEM_TET4_EDGE: 4, ELEM_HEX8_EDGE: 8, ELEM_PRISM6_EDGE: 6, ELEM_PYRAMID5_EDGE: 5}
LOCAL_EDGES = {ELEM_TET4_EDGE: GEO_EDGES, ELEM_HEX8_EDGE: HEX_EDGES, ELEM_PRISM6_EDGE: PRISM_EDGES,
               ELEM_PYRAMID5_EDGE: PYRAMID_EDGES}

# Source region kinds (same values as the C ABI's EMG_SRC_*).
SRC_BOX = 1
SRC_ANNULUS_Z = 2


@dataclass
class Source:
    """Uniform current density ``j`` inside an open region evaluated at
    quadrature points: BOX p = (xmin, xmax, ymin, ymax, zmin, zmax);
    ANNULUS_Z p = (cx, cy, rmin, rmax, zmin, zmax)."""
    kind: int
    j: tuple
    p: tuple


@dataclass
class CubeMesh:
    n: int
    xyz: np.ndarray          # (V, 3) float64
    tets: np.ndarray         # (T, 4) int32
    material: np.ndarray     # (T,) int32
    dirichlet: np.ndarray    # (D, 2) int32 node pairs
    nu: np.ndarray           # per-material reluctivity 1/mu
    sigma: np.ndarray        # per-material conductivity
    sources: list = field(default_factory=list)
    name: str = ""

    @property
    def n_nodes(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_tets(self) -> int:
        """Number of elements (tets, or hexes for a hex mesh)."""
        return int(self.tets.shape[0])

    @property
    def elem_type(self) -> int:
        return TYPE_OF_NODES[self.tets.shape[1]]


def cube_topology(n: int):
    """Nodes, tets and boundary-face edge pairs of the n^3 Kuhn-split cube
    (fresh copies of a cached topology)."""
    xyz, tets, dirichlet = _cube_topology(n)
    return xyz.copy(), tets.copy(), dirichlet.copy()


@lru_cache(maxsize=64)
def _cube_topology(n: int):
    n1 = n + 1
    g = np.arange(n1, dtype=np.float64) / n
    kk, jj, ii = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    xyz = np.stack([g[ii.ravel()], g[jj.ravel()], g[kk.ravel()]], axis=1)
    hk, hj, hi = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    verts = np.stack([(hi + a) + n1 * ((hj + b) + n1 * (hk + c)) for a, b, c in off], axis=1)
    tets = verts[:, KUHN].reshape(-1, 4).astype(np.int32)
    return xyz, tets, _boundary_pairs(tets, GEO_EDGES, n)


@lru_cache(maxsize=64)
def _hex_topology(n: int):
    xyz, tets, dirichlet = _cube_topology(n)
    n1 = n + 1
    hk, hj, hi = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    hexes = np.stack([(hi + a) + n1 * ((hj + b) + n1 * (hk + c)) for a, b, c in off], axis=1).astype(np.int32)
    return xyz, hexes, _boundary_pairs(hexes, HEX_EDGES, n)


def hex_topology(n: int):
    """Nodes, HEX8 elements and boundary-face edge pairs of the n^3 cube."""
    xyz, hexes, dirichlet = _hex_topology(n)
    return xyz.copy(), hexes.copy(), dirichlet.copy()


def prism_topology(n: int):
    """Nodes, PRISM6 elements (two per grid cell) and boundary-face edge pairs
    of the n^3 cube."""
    xyz, hexes, _ = _hex_topology(n)
    # ElementGeometry's PRISM6 order with the reference's PRISM6 map (node 0 at
    # area coordinate xi, node 1 at eta, node 2 at the right angle) gives a
    # positive Jacobian for these triangles
    a = hexes[:, [0, 1, 2, 4, 5, 6]]
    b = hexes[:, [0, 2, 3, 4, 6, 7]]
    prisms = np.stack([a, b], axis=1).reshape(-1, 6).astype(np.int32)
    return xyz.copy(), prisms, _boundary_pairs(prisms, PRISM_EDGES, n)


def pyramid_topology(n: int):
    """Nodes (the grid plus one centre node per cell), PYRAMID5 elements (six
    per cell, base = a cell face ordered so that the apex lies on the side the
    reference map puts it) and boundary-face edge pairs of the n^3 cube."""
    xyz, hexes, _ = _hex_topology(n)
    n1 = n + 1
    centres = xyz[hexes].mean(axis=1)
    cid = (n1 ** 3 + np.arange(len(hexes))).astype(np.int32)
    faces = [[0, 1, 2, 3], [4, 7, 6, 5], [0, 4, 5, 1], [3, 2, 6, 7], [0, 3, 7, 4], [1, 5, 6, 2]]
    pyr = np.stack([np.concatenate([hexes[:, f], cid[:, None]], axis=1) for f in faces], axis=1)
    return np.vstack([xyz, centres]), pyr.reshape(-1, 5).astype(np.int32), _boundary_pairs(pyr.reshape(-1, 5),
                                                                                           PYRAMID_EDGES, n)


def _boundary_pairs(elems, local_edges, n):
    """Unique element edges whose two nodes share a coordinate plane at 0 or
    n (grid indices), as sorted node pairs (nodes beyond the grid, such as
    cell centres, lie on no boundary)."""
    n1 = n + 1
    e = elems[:, local_edges].reshape(-1, 2).astype(np.int64)
    e = e[(e < n1 ** 3).all(axis=1)]
    e.sort(axis=1)
    e = np.unique(e[:, 0] * (n1 ** 3) + e[:, 1])
    a, b = e // (n1 ** 3), e % (n1 ** 3)
    ia, ja, ka = a % n1, (a // n1) % n1, a // (n1 * n1)
    ib, jb, kb = b % n1, (b // n1) % n1, b // (n1 * n1)
    on = np.zeros(a.shape, dtype=bool)
    for ca, cb in ((ia, ib), (ja, jb), (ka, kb)):
        on |= (ca == cb) & ((ca == 0) | (ca == n))
    return np.stack([a[on], b[on]], axis=1).astype(np.int32)


def centroids(xyz: np.ndarray, tets: np.ndarray) -> np.ndarray:
    return xyz[tets].mean(axis=1)


def plain_small(n: int = 16) -> CubeMesh:
    """Plain method, small: nu = 1 everywhere, J = (0,0,1) inside the central
    box [0.375, 0.625]^3 (grid-aligned at n = 16)."""
    xyz, tets, dirichlet = cube_topology(n)
    return CubeMesh(n=n, xyz=xyz, tets=tets, material=np.zeros(len(tets), np.int32),
                    dirichlet=dirichlet, nu=np.array([1.0]), sigma=np.array([0.0]),
                    sources=[Source(SRC_BOX, (0.0, 0.0, 1.0),
                                    (0.375, 0.625, 0.375, 0.625, 0.375, 0.625))],
                    name=f"cube{n}_box")


def plain_scale(n: int = 64, mu_iron: float = 1000.0) -> CubeMesh:
    """Plain method at scale: iron block [0.25,0.75]^2 x [0.4,0.6] (mu_r =
    1000, by tet centroid), mu_r = 1 elsewhere; z-directed coil current on the
    annulus 0.3 < r < 0.45 (axis x = y = 0.5), 0.2 < z < 0.8."""
    xyz, tets, dirichlet = cube_topology(n)
    c = centroids(xyz, tets)
    iron = ((c[:, 0] > 0.25) & (c[:, 0] < 0.75) & (c[:, 1] > 0.25) & (c[:, 1] < 0.75)
            & (c[:, 2] > 0.4) & (c[:, 2] < 0.6))
    return CubeMesh(n=n, xyz=xyz, tets=tets, material=iron.astype(np.int32),
                    dirichlet=dirichlet, nu=np.array([1.0, 1.0 / mu_iron]),
                    sigma=np.array([0.0, 0.0]),
                    sources=[Source(SRC_ANNULUS_Z, (0.0, 0.0, 1.0),
                                    (0.5, 0.5, 0.3, 0.45, 0.2, 0.8))],
                    name=f"cube{n}_iron_coil")


def hex_small(n: int = 16) -> CubeMesh:
    """plain_small on HEX8_EDGE elements (the n^3 grid cells themselves)."""
    xyz, hexes, dirichlet = hex_topology(n)
    m = plain_small(1)
    return CubeMesh(n=n, xyz=xyz, tets=hexes, material=np.zeros(len(hexes), np.int32),
                    dirichlet=dirichlet, nu=m.nu, sigma=m.sigma, sources=m.sources, name=f"hex{n}_box")


def hex_scale(n: int = 64, mu_iron: float = 1000.0) -> CubeMesh:
    """plain_scale on HEX8_EDGE elements: iron block by cell centroid, the
    same coil source."""
    xyz, hexes, dirichlet = hex_topology(n)
    c = centroids(xyz, hexes)
    iron = ((c[:, 0] > 0.25) & (c[:, 0] < 0.75) & (c[:, 1] > 0.25) & (c[:, 1] < 0.75)
            & (c[:, 2] > 0.4) & (c[:, 2] < 0.6))
    m = plain_scale(1, mu_iron)
    return CubeMesh(n=n, xyz=xyz, tets=hexes, material=iron.astype(np.int32), dirichlet=dirichlet,
                    nu=m.nu, sigma=m.sigma, sources=m.sources, name=f"hex{n}_iron_coil")


def mixed_rows(types, elems) -> np.ndarray:
    """Padded mixed-mesh rows from per-element types and node lists."""
    rows = -np.ones((len(types), 9), np.int32)
    for r, (t, e) in enumerate(zip(types, elems)):
        rows[r, : len(e)] = e
        rows[r, 8] = t
    return rows


def element_edges(rows: np.ndarray) -> np.ndarray:
    """(E, 2) node pairs of every element edge of a one-type or mixed
    element array, elements in order, local edges in order."""
    et = TYPE_OF_NODES[rows.shape[1]]
    if et != ELEM_MIXED:
        return rows[:, LOCAL_EDGES[et]].reshape(-1, 2)
    out = [rows[rows[:, 8] == t][:, LOCAL_EDGES[t]].reshape(-1, 2) for t in range(4)]
    return np.vstack([o for o in out if len(o)])


def mixed_cells(n: int, kind_of_cell, small: bool = True, mu_iron: float = 1000.0) -> CubeMesh:
    """Mixed mesh of the n^3 grid: every cell becomes the elements kind_of_cell
    (i, j, k) names -- "hex" (one HEX8), "prism" (two PRISM6, as prism_topology),
    "tet" (six Kuhn TET4) or "pyramid" (six PYRAMID5 around an added centre
    node, as pyramid_topology) -- cells in k -> j -> i order.  Neighbouring
    cells must share faces of one shape (quadrilaterals between hex, pyramid
    and prism side faces; triangles between prisms' z-faces and tets)."""
    xyz, hexes, _ = _hex_topology(n)
    n1 = n + 1
    faces = [[0, 1, 2, 3], [4, 7, 6, 5], [0, 4, 5, 1], [3, 2, 6, 7], [0, 3, 7, 4], [1, 5, 6, 2]]
    types, elems, centres = [], [], []
    for c, h in enumerate(hexes):
        i, j, k = c % n, (c // n) % n, c // (n * n)
        kind = kind_of_cell(i, j, k)
        if kind == "hex":
            types.append(ELEM_HEX8_EDGE); elems.append(h)
        elif kind == "prism":
            for sel in ([0, 1, 2, 4, 5, 6], [0, 2, 3, 4, 6, 7]):
                types.append(ELEM_PRISM6_EDGE); elems.append(h[sel])
        elif kind == "tet":
            for tet in KUHN:
                types.append(ELEM_TET4_EDGE); elems.append(h[tet])
        else:
            cid = n1 ** 3 + len(centres)
            centres.append(xyz[h].mean(axis=0))
            for f in faces:
                types.append(ELEM_PYRAMID5_EDGE); elems.append(np.r_[h[f], cid])
    rows = mixed_rows(types, elems)
    allxyz = np.vstack([xyz] + ([np.array(centres)] if centres else []))
    edges = element_edges(rows)
    d = _boundary_pairs(np.asarray(edges, np.int64), np.array([[0, 1]]), n)
    m = plain_small(1) if small else plain_scale(1, mu_iron)
    c = np.array([allxyz[e[:NODES_OF_TYPE[t]]].mean(axis=0) for t, e in zip(types, elems)])
    mat = np.zeros(len(types), np.int32) if small else (
        (c[:, 0] > 0.25) & (c[:, 0] < 0.75) & (c[:, 1] > 0.25) & (c[:, 1] < 0.75)
        & (c[:, 2] > 0.4) & (c[:, 2] < 0.6)).astype(np.int32)
    return CubeMesh(n=n, xyz=allxyz, tets=rows, material=mat, dirichlet=d, nu=m.nu, sigma=m.sigma,
                    sources=m.sources, name=f"mixed{n}")


def mixed_hex_prism(n: int, small: bool = True) -> CubeMesh:
    """Hexahedra for x < 1/2, prisms beyond (shared x-faces are quadrilaterals)."""
    return mixed_cells(n, lambda i, j, k: "hex" if 2 * i < n else "prism", small)


def mixed_prism_tet(n: int, small: bool = True) -> CubeMesh:
    """Prisms for z < 1/2, Kuhn tetrahedra above (shared z-faces are triangles)."""
    return mixed_cells(n, lambda i, j, k: "prism" if 2 * k < n else "tet", small)


def mixed_hex_pyramid_prism(n: int, small: bool = True) -> CubeMesh:
    """Hexahedra (x < 1/2, z < 1/2), pyramid cells (x < 1/2, z >= 1/2), prisms
    (x >= 1/2): every shared face a quadrilateral."""
    return mixed_cells(n, lambda i, j, k: "prism" if 2 * i >= n else ("hex" if 2 * k < n else "pyramid"), small)


def _on_cells(kind: str, n: int, mu_iron: float, small: bool) -> CubeMesh:
    xyz, elems, dirichlet = prism_topology(n) if kind == "prism" else pyramid_topology(n)
    if small:
        m = plain_small(1)
        mat = np.zeros(len(elems), np.int32)
    else:
        m = plain_scale(1, mu_iron)
        c = centroids(xyz, elems)
        mat = ((c[:, 0] > 0.25) & (c[:, 0] < 0.75) & (c[:, 1] > 0.25) & (c[:, 1] < 0.75)
               & (c[:, 2] > 0.4) & (c[:, 2] < 0.6)).astype(np.int32)
    return CubeMesh(n=n, xyz=xyz, tets=elems, material=mat, dirichlet=dirichlet, nu=m.nu, sigma=m.sigma,
                    sources=m.sources, name=f"{kind}{n}_{'box' if small else 'iron_coil'}")


def prism_small(n: int = 16) -> CubeMesh:
    """plain_small on PRISM6_EDGE elements."""
    return _on_cells("prism", n, 1.0, True)


def prism_scale(n: int = 64, mu_iron: float = 1000.0) -> CubeMesh:
    """plain_scale on PRISM6_EDGE elements (iron block by element centroid)."""
    return _on_cells("prism", n, mu_iron, False)


def pyramid_small(n: int = 16) -> CubeMesh:
    """plain_small on PYRAMID5_EDGE elements."""
    return _on_cells("pyramid", n, 1.0, True)


def pyramid_scale(n: int = 64, mu_iron: float = 1000.0) -> CubeMesh:
    """plain_scale on PYRAMID5_EDGE elements (iron block by element centroid)."""
    return _on_cells("pyramid", n, mu_iron, False)


def jittered_cuts(n: int, parts: int = 4, seed: int = 20261203, jitter: int | None = None):
    """Cut positions (in cells) per axis: ``parts - 1`` planes at multiples of
    n / parts, each moved by an integer in [-jitter, jitter] (default
    n / parts / 8, i.e. slab widths 12..20 cells for n = 64, 4 parts), so
    subdomain volumes vary about 0.4-2x."""
    if n % parts:
        raise ValueError("n must be a multiple of parts")
    w = n // parts
    j = max(w // 8, 1 if w >= 3 else 0) if jitter is None else jitter
    rng = np.random.default_rng(seed)
    return [np.array([k * w + int(rng.integers(-j, j + 1)) for k in range(1, parts)], np.int64)
            for _ in range(3)]


def jittered_partition(m: CubeMesh, parts: int = 4, seed: int = 20261203, jitter: int | None = None):
    """Tet -> subdomain by centroid for a parts^3 box partition of the cube
    with jittered cut planes; subdomain id = ix + parts * (iy + parts * iz)."""
    cuts = jittered_cuts(m.n, parts, seed, jitter)
    c = centroids(m.xyz, m.tets) * m.n
    idx = [np.searchsorted(cuts[a], c[:, a], side="right") for a in range(3)]
    return (idx[0] + parts * (idx[1] + parts * idx[2])).astype(np.int32)


def random_instance(n: int, seed: int) -> CubeMesh:
    """One many-instance case: a random axis-aligned box with mu_r in
    [1, 1000] (1 elsewhere) and a uniform J_z in a random sub-box."""
    rng = np.random.default_rng(seed)
    xyz, tets, dirichlet = cube_topology(n)
    lo = rng.uniform(0.05, 0.5, 3)
    hi = lo + rng.uniform(0.2, 0.45, 3)
    mu = rng.uniform(1.0, 1000.0)
    c = centroids(xyz, tets)
    inside = np.all((c > lo) & (c < np.minimum(hi, 0.95)), axis=1)
    slo = rng.uniform(0.1, 0.5, 3)
    shi = slo + rng.uniform(0.15, 0.4, 3)
    return CubeMesh(n=n, xyz=xyz, tets=tets, material=inside.astype(np.int32),
                    dirichlet=dirichlet, nu=np.array([1.0, 1.0 / mu]),
                    sigma=np.array([0.0, 0.0]),
                    sources=[Source(SRC_BOX, (0.0, 0.0, 1.0),
                                    (slo[0], min(shi[0], 0.9), slo[1], min(shi[1], 0.9),
                                     slo[2], min(shi[2], 0.9)))],
                    name=f"cube{n}_rand{seed}")


def perturbed(m: CubeMesh, amplitude: float = 0.2, seed: int = 0) -> CubeMesh:
    """The same mesh with every interior node moved by up to `amplitude` cell
    widths per coordinate (uniform random, seeded): unstructured geometry on
    the same topology; boundary nodes stay on the faces."""
    rng = np.random.default_rng(seed)
    xyz = m.xyz.copy()
    interior = np.all((xyz > 1e-12) & (xyz < 1.0 - 1e-12), axis=1)
    h = 1.0 / m.n
    xyz[interior] += rng.uniform(-amplitude * h, amplitude * h, (int(interior.sum()), 3))
    return CubeMesh(**{**m.__dict__, "xyz": xyz, "name": m.name + f"_perturbed{seed}"})


HEX_FACES = np.array([[0, 1, 2, 3], [4, 5, 6, 7], [0, 1, 5, 4], [2, 3, 7, 6], [0, 3, 7, 4], [1, 2, 6, 5]])


def write_gmsh(m: CubeMesh, path: str, version: str = "2.2", volume_tags=(1, 2), boundary_tag: int = 100,
               names=None):
    """Write the mesh as an ASCII Gmsh file (2.2 or 4.1): node tags 1..V,
    the tetrahedra (type 4) or hexahedra (type 5) with physical tag
    volume_tags[material], and every boundary face as a triangle (type 2) or
    a quadrangle (type 3, corners in cyclic order) with physical tag
    `boundary_tag`.  `names` ({physical tag: name}) adds a $PhysicalNames
    section (dimension 3 for the volume tags, 2 for the boundary tag)."""
    tets = np.asarray(m.tets, np.int64)
    hexa = tets.shape[1] == 8
    if hexa:
        cyc = tets[:, HEX_FACES].reshape(-1, 4)
        _, first, cnt = np.unique(np.sort(cyc, axis=1), axis=0, return_index=True, return_counts=True)
        bfaces = cyc[np.sort(first[cnt == 1])]
    else:
        faces = np.sort(tets[:, [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]].reshape(-1, 3), axis=1)
        uf, cnt = np.unique(faces, axis=0, return_counts=True)
        bfaces = uf[cnt == 1]
    ftype, vtype = (3, 5) if hexa else (2, 4)
    vt = np.asarray(volume_tags)[np.asarray(m.material)]
    nodes = lambda row: " ".join(str(int(v) + 1) for v in row)
    pn = ""
    if names:
        rows = [f'{2 if int(t) == boundary_tag else 3} {int(t)} "{n}"' for t, n in sorted(names.items())]
        pn = "$PhysicalNames\n%d\n%s\n$EndPhysicalNames\n" % (len(rows), "\n".join(rows))
    with open(path, "w") as f:
        if version.startswith("2"):
            f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n" + pn + "$Nodes\n%d\n" % m.n_nodes)
            for i, (x, y, z) in enumerate(m.xyz):
                f.write(f"{i + 1} {float(x)!r} {float(y)!r} {float(z)!r}\n")
            f.write("$EndNodes\n$Elements\n%d\n" % (len(bfaces) + len(tets)))
            eid = 1
            for fc in bfaces:
                f.write(f"{eid} {ftype} 2 {boundary_tag} 1 {nodes(fc)}\n")
                eid += 1
            for t, tag in zip(tets, vt):
                f.write(f"{eid} {vtype} 2 {int(tag)} {int(tag)} {nodes(t)}\n")
                eid += 1
            f.write("$EndElements\n")
        else:
            vols = sorted(set(int(v) for v in vt))
            f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n" + pn + "$Entities\n0 0 1 %d\n" % len(vols))
            f.write(f"1 0 0 0 1 1 1 1 {boundary_tag} 0\n")
            for v in vols:
                f.write(f"{v} 0 0 0 1 1 1 1 {v} 0\n")
            f.write("$EndEntities\n$Nodes\n1 %d 1 %d\n3 1 0 %d\n" % (m.n_nodes, m.n_nodes, m.n_nodes))
            f.write("".join(f"{i + 1}\n" for i in range(m.n_nodes)))
            f.write("".join(f"{float(x)!r} {float(y)!r} {float(z)!r}\n" for x, y, z in m.xyz))
            f.write("$EndNodes\n$Elements\n%d %d 1 %d\n" % (1 + len(vols), len(bfaces) + len(tets),
                                                           len(bfaces) + len(tets)))
            eid = 1
            f.write(f"2 1 {ftype} {len(bfaces)}\n")
            for fc in bfaces:
                f.write(f"{eid} {nodes(fc)}\n")
                eid += 1
            for v in vols:
                sel = tets[vt == v]
                f.write(f"3 {v} {vtype} {len(sel)}\n")
                for t in sel:
                    f.write(f"{eid} {nodes(t)}\n")
                    eid += 1
            f.write("$EndElements\n")


def read_gmsh(path: str, dirichlet_tags=None, nu=None, sigma=None, sources=None) -> CubeMesh:
    """Read an ASCII Gmsh file through the library (emg_mesh_read_gmsh).
    Materials: one per physical volume tag (ascending); nu / sigma per
    material (default 1 / 0)."""
    import ctypes as C

    from . import _abi
    L = _abi.lib()
    tags = None if not dirichlet_tags else np.ascontiguousarray(dirichlet_tags, np.int32)
    h = C.c_void_p()
    _abi.check(L.emg_mesh_read_gmsh(path.encode(), _abi.ptr(tags), 0 if tags is None else len(tags),
                                    C.byref(h)), "emg_mesh_read_gmsh")
    try:
        nn, nt, nd, nm = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        L.emg_mesh_info(h, C.byref(nn), C.byref(nt), C.byref(nd), C.byref(nm))
        npe = C.c_int32()
        L.emg_mesh_elem_type(h, None, C.byref(npe), None)
        xyz = np.empty((nn.value, 3))
        tets = np.empty((nt.value, npe.value), np.int32)
        mat = np.empty(nt.value, np.int32)
        dp = np.empty((nd.value, 2), np.int32)
        L.emg_mesh_export(h, _abi.ptr(xyz), _abi.ptr(tets), _abi.ptr(mat), _abi.ptr(dp))
        mtags = np.empty(max(nm.value, 1), np.int32)
        L.emg_mesh_material_tags(h, _abi.ptr(mtags))
    finally:
        L.emg_mesh_destroy(h)
    k = nm.value
    m = CubeMesh(n=0, xyz=xyz, tets=tets, material=mat, dirichlet=dp,
                 nu=np.ones(k) if nu is None else np.asarray(nu, np.float64),
                 sigma=np.zeros(k) if sigma is None else np.asarray(sigma, np.float64),
                 sources=list(sources or []), name=path)
    m.material_tags = mtags[:k]
    names = physical_names(path)
    m.physical_names = names
    # the name of every material (physical volume), in material-id order
    m.material_names = [names.get((3, int(t))) for t in m.material_tags]
    return m


def physical_names(path: str) -> dict:
    """{(dimension, physical tag): name} from a Gmsh file's $PhysicalNames
    section (empty without one)."""
    out = {}
    with open(path) as f:
        for line in f:
            if line.strip() == "$PhysicalNames":
                n = int(f.readline())
                for _ in range(n):
                    dim, tag, rest = f.readline().split(None, 2)
                    out[(int(dim), int(tag))] = rest.strip().strip('"')
                break
            if line.strip() == "$Nodes":
                break
    return out
