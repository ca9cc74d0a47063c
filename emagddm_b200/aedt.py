"""Ansys Maxwell project input: the materials, objects and boundaries of an
.aedt text project (the data the reference's AedtProjectLoader takes from
MaxwellParserImpl, src/tool/aedt_project_loader.cpp:60-130), read by the
library (emg_aedt_*), and their mapping onto a mesh read from Gmsh whose
physical volumes carry the objects' names.

Units: relative permeability and conductivity [S/m] as in the project; a
nonlinear (BH-curve) material stands in with its initial permeability.  The
solver's nu per material is 1 / (mu0 mu_r) with the caller's mu0 (the
benchmark meshes use mu0 = 1).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi

FLAG_NONLINEAR, FLAG_MU_NOT_NUMBER, FLAG_SIGMA_NOT_NUMBER = 1, 2, 4
_NAME = 512


@dataclass
class Material:
    name: str
    mu_r: float
    sigma: float
    flags: int
    bh: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))  # (H, B) pairs of a nonlinear material


@dataclass
class Object:
    name: str
    material: str
    solve_inside: bool


@dataclass
class Boundary:
    name: str
    type: str
    value: str


class AedtProject:
    def __init__(self, path: str):
        L = _abi.lib()
        h = C.c_void_p()
        _abi.check(L.emg_aedt_read(path.encode(), C.byref(h)), "emg_aedt_read")
        try:
            nm, no, nb = C.c_int32(), C.c_int32(), C.c_int32()
            L.emg_aedt_info(h, C.byref(nm), C.byref(no), C.byref(nb))
            self.materials, self.objects, self.boundaries = [], [], []
            for k in range(nm.value):
                name = C.create_string_buffer(_NAME)
                mu, sg, fl, nbh = C.c_double(), C.c_double(), C.c_int32(), C.c_int32()
                L.emg_aedt_material(h, k, name, _NAME, C.byref(mu), C.byref(sg), C.byref(fl), C.byref(nbh))
                bh = np.zeros((nbh.value, 2))
                if nbh.value:
                    hh, bb = np.empty(nbh.value), np.empty(nbh.value)
                    L.emg_aedt_bh_curve(h, k, _abi.ptr(hh), _abi.ptr(bb), nbh.value)
                    bh = np.stack([hh, bb], axis=1)
                self.materials.append(Material(name.value.decode(), mu.value, sg.value, fl.value, bh))
            for k in range(no.value):
                name, mat, si = C.create_string_buffer(_NAME), C.create_string_buffer(_NAME), C.c_int32()
                L.emg_aedt_object(h, k, name, _NAME, mat, _NAME, C.byref(si))
                self.objects.append(Object(name.value.decode(), mat.value.decode(), bool(si.value)))
            for k in range(nb.value):
                name, typ, val = (C.create_string_buffer(_NAME) for _ in range(3))
                L.emg_aedt_boundary(h, k, name, _NAME, typ, _NAME, val, _NAME)
                self.boundaries.append(Boundary(name.value.decode(), typ.value.decode(), val.value.decode()))
        finally:
            L.emg_aedt_destroy(h)

    def material(self, name: str) -> Material:
        key = name.lower()
        for m in self.materials:
            if m.name.lower() == key:
                return m
        raise KeyError(f"material {name!r} is not defined in the project")

    def object(self, name: str) -> Object:
        for o in self.objects:
            if o.name == name:
                return o
        raise KeyError(f"object {name!r} is not in the project")

    def material_arrays(self, volume_names, mu0: float = 1.0):
        """nu = 1 / (mu0 mu_r) and sigma per mesh material, the mesh materials
        named by the objects they were meshed from (Gmsh physical volume names,
        in material-id order)."""
        nu, sigma = [], []
        for v in volume_names:
            m = self.material(self.object(v).material)
            if m.flags & (FLAG_MU_NOT_NUMBER | FLAG_SIGMA_NOT_NUMBER):
                raise ValueError(f"material {m.name!r} of {v!r} has a property that is not a number")
            nu.append(1.0 / (mu0 * m.mu_r))
            sigma.append(m.sigma)
        return np.asarray(nu), np.asarray(sigma)
