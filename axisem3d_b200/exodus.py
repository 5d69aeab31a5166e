"""Exodus meshes of the salvus mesher, read as the reference's ExodusMesh does
(SOLVER/src/preloop/exodus/ExodusMesh.cpp). Mesh reading runs once before the time loop,
on the host.

Both container formats the NetCDF library reads are accepted: NetCDF-4 (HDF5; the
reference's example meshes) through this package's own HDF5 reader, and NetCDF-3 classic
through `scipy.io.netcdf_file`.

What is read, and the order and rules applied (all from ExodusMesh.cpp):
  - global variables `name_glo_var` / `vals_glo_var` with the renames of
    readBcastGlobal (:198-241); the records `crdsys` and `model` from `info_records`;
  - connectivity `connect1` (0-based), coordinates `coordx`, `coordy` (:244-285);
  - side sets `ss_names`, `elem_ss<i>`, `side_ss<i>` (0-based), the side-set keys
    (x0/x1/y0/y1 Cartesian, t0/t1/r0/r1 spherical), and `min_edge_length` and
    `dist_tolerance` from the edges of the axial quads (:288-350);
  - element variables `element_type` and `fluid` (:353-392);
  - the radial profile: the depth profile along the axis and the radial variables on it,
    with the discontinuity check and the averaging of fake gaps (:395-562), then the
    rotation of the axial quads so that side 3 lies on the axis (:583-610);
  - the ellipticity curve (:614-632).
"""
from __future__ import annotations

import bisect
import os

import numpy as np

from . import hdf5

EPS = np.finfo(np.float64).eps


class ExodusError(RuntimeError):
    """An Exodus file this reader cannot use; messages follow "Class::method || text"."""


def cycle4(p: int) -> int:
    """Mapping::cycle4."""
    return p - 4 if p > 3 else (p + 4 if p < 0 else p)


class _Nc:
    """The variables of a NetCDF-3 or NetCDF-4 file by name."""

    def __init__(self, path: str):
        with open(path, "rb") as f:
            magic = f.read(4)
        if magic[:3] == b"CDF":
            from scipy.io import netcdf_file
            nc = netcdf_file(path, "r", mmap=False)
            self._vars = {k: np.array(v.data) for k, v in nc.variables.items()}
            nc.close()
        elif magic == b"\x89HDF":
            h = hdf5.File(path)
            self._h = h
            self._vars = None
        else:
            raise ExodusError("NetCDF_Reader::open || Not a NetCDF file: %s" % path)

    def has(self, name: str) -> bool:
        return name in self._vars if self._vars is not None else name in self._h.datasets

    def read(self, name: str) -> np.ndarray:
        if not self.has(name):
            raise ExodusError("NetCDF_Reader::readMatrix || Variable not found: %s" % name)
        if self._vars is not None:
            return self._vars[name]
        return self._h.datasets[name].read()

    def strings(self, name: str) -> list:
        a = self.read(name)
        if a.ndim == 1:
            a = a[None, :]
        out = []
        for row in a:
            b = b"".join(x if isinstance(x, bytes) else bytes([x]) for x in row.tolist())
            out.append(b.split(b"\0")[0].decode("utf-8", "replace").strip())
        return out


class ExodusMesh:
    """A salvus-mesher Exodus mesh: the data ExodusMesh keeps after its constructor."""

    def __init__(self, path: str):
        self.path = path
        nc = _Nc(path)
        self._read_global(nc)
        self.connectivity = nc.read("connect1").astype(np.int64) - 1
        self.coords = np.stack([nc.read("coordx").astype(np.float64),
                                nc.read("coordy").astype(np.float64)], axis=1)
        self._read_side_sets(nc)
        self._read_elemental(nc)
        self._read_radial(nc)
        self._rotate_axial()
        if not self.is_cartesian:
            self.ellipticity = nc.read("ellipticity").astype(np.float64).copy()
        else:
            self.ellipticity = np.array([[0.0, 1.0], [1.0, 1.0]])
        self.ellipticity[0] *= self.mesh_surface

    # ---------------- reading ----------------
    def _read_global(self, nc):
        names = nc.strings("name_glo_var")
        vals = np.asarray(nc.read("vals_glo_var"), dtype=np.float64).reshape(-1)
        self.global_variables = {}
        for name, v in zip(names, vals):
            if name == "dt":
                name = "dt (nPol = 1)"
            if name.startswith(("w_", "y_", "f_")):
                name = "attenuation_" + name
            self.global_variables[name] = float(v)
        self.records = {}
        self.cmd_mesh_gen = ""
        for rec in nc.strings("info_records"):
            parts = rec.split("=")
            key = parts[0].strip()
            if key in ("crdsys", "model") and len(parts) > 1:
                self.records[key] = parts[1].strip()
            if "cmdl" in key and len(parts) > 1:
                self.cmd_mesh_gen += "=".join(parts[1:]).strip() + "\n"
        if "crdsys" not in self.records:
            raise ExodusError("ExodusMesh::readBcastGlobal || Record crdsys not found.")

    def _read_side_sets(self, nc):
        names = nc.strings("ss_names") if nc.has("ss_names") else []
        self.side_sets = {}
        for i, name in enumerate(names):
            elems = np.asarray(nc.read("elem_ss%d" % (i + 1))).astype(np.int64) - 1
            sides = np.asarray(nc.read("side_ss%d" % (i + 1))).astype(np.int64) - 1
            m = {}
            for e, s in zip(elems.tolist(), sides.tolist()):
                m.setdefault(e, s)                        # std::map::insert keeps the first
            self.side_sets[name] = m
        c = self.is_cartesian
        self.key_left = "x0" if c else "t0"
        self.key_right = "x1" if c else "t1"
        self.key_bottom = "y0" if c else "r0"
        self.key_top = "y1" if c else "r1"
        min_edge = np.finfo(np.float64).max
        for q in self.side_sets.get(self.key_left, {}):
            for a in range(4):
                b = 0 if a == 3 else a + 1
                d = self.coords[self.connectivity[q, a]] - self.coords[self.connectivity[q, b]]
                min_edge = min(min_edge, float(np.hypot(d[0], d[1])))
        self.global_variables["min_edge_length"] = min_edge
        self.global_variables["dist_tolerance"] = min_edge / 1000.

    def _elem_var_keys(self, nc):
        names = nc.strings("name_elem_var")
        return {n: "vals_elem_var%deb1" % (i + 1) for i, n in enumerate(names)}

    def _read_elemental(self, nc):
        keys = self._elem_var_keys(nc)
        for need in ("element_type", "fluid"):
            if need not in keys:
                raise ExodusError("ExodusMesh::readBcastElemental || Element variable %s not found." % need)
        self.geometry_type = np.rint(np.asarray(nc.read(keys["element_type"])).reshape(-1)).astype(np.int64)
        self.is_fluid = np.rint(np.asarray(nc.read(keys["fluid"])).reshape(-1)).astype(np.int64)

    def _read_radial(self, nc):
        keys = self._elem_var_keys(nc)
        self.element_nodes_storage = "RHO_0" in keys
        isotropic = "ETA_0" not in keys and "ETA" not in keys
        names = ["RHO", "VP", "VS"] if isotropic else ["RHO", "VPV", "VPH", "VSV", "VSH", "ETA"]
        if self.has_attenuation:
            names += ["QMU", "QKAPPA"]
        tol = self.global_variables["dist_tolerance"]
        coords: list = []
        quad_nodes: list = []
        for q in range(self.num_quads):
            side = self.side_sets.get(self.key_left, {}).get(q, -1)
            if side < 0:
                continue
            other = 0 if side == 3 else side + 1
            z1 = self.coords[self.connectivity[q, side], 1]
            z2 = self.coords[self.connectivity[q, other], 1]
            if min(z1, z2) < 0.:
                continue
            d = (z2 - z1) / abs(z2 - z1) * tol
            z1 += d
            z2 -= (z2 - z1) / abs(z2 - z1) * tol
            i1 = bisect.bisect_right(coords, z1)
            coords.insert(i1, z1)
            quad_nodes.insert(i1, (q, side))
            i2 = bisect.bisect_right(coords, z2)
            coords.insert(i2, z2)
            quad_nodes.insert(i2, (q, other))
        if len(coords) < 2:
            raise ExodusError("ExodusMesh::readBcastRadial || No axial elements found.")
        vals = np.zeros((len(coords), len(names)))
        for j, name in enumerate(names):
            if self.element_nodes_storage:
                buf = [np.asarray(nc.read(keys[name + "_%d" % k])).reshape(-1) for k in range(4)]
                for i, (q, node) in enumerate(quad_nodes):
                    vals[i, j] = buf[node][q]
            else:
                if name not in keys:
                    raise ExodusError("ExodusMesh::readBcastRadial || Element variable %s not found." % name)
                buf = np.asarray(nc.read(keys[name])).reshape(-1)
                for i, (q, _) in enumerate(quad_nodes):
                    vals[i, j] = buf[q]
        all_discs = np.asarray(nc.read("discontinuities"), dtype=np.float64).reshape(-1)
        discs = [d for d in all_discs.tolist() if coords[0] - 2. * tol < d < coords[-1] + 2. * tol]
        found = 0
        for i in range(len(coords) - 1):
            if coords[i + 1] - coords[i] > tol * 4:
                continue
            is_disc = False
            for d in discs:
                if coords[i] < d < coords[i + 1]:
                    is_disc = True
                    found += 1
                    break
            if not is_disc:
                vals[i] = (vals[i] + vals[i + 1]) * .5
                vals[i + 1] = vals[i]
        if found != len(discs) - 2:
            raise ExodusError("ExodusMesh::readBcastRadial || Error verifying mesh discontinuities.")
        self.discontinuities = np.array(discs)
        self.radial_coords = np.array(coords)
        self.radial_variables = {n: vals[:, j].copy() for j, n in enumerate(names)}

    def _rotate_axial(self):
        """Rotate the nodes of axial quads so that side 3 lies on the axis (:583-610)."""
        for q, side in list(self.side_sets.get(self.key_left, {}).items()):
            row = self.connectivity[q].copy()
            for v in range(4):
                self.connectivity[q, v] = row[cycle4(v + side - 3)]
            for name, m in self.side_sets.items():
                if q in m:
                    m[q] = cycle4(m[q] - side + 3)

    # ---------------- accessors (ExodusMesh.hpp) ----------------
    @property
    def num_quads(self) -> int:
        return int(self.connectivity.shape[0])

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def is_cartesian(self) -> bool:
        return self.records.get("crdsys") != "spherical"

    @property
    def has_attenuation(self) -> bool:
        return "nr_lin_solids" in self.global_variables

    @property
    def is_isotropic(self) -> bool:
        return "VP" in self.radial_variables

    def side(self, name: str, quad: int) -> int:
        return self.side_sets.get(name, {}).get(quad, -1)

    def left_side(self, q):
        return self.side(self.key_left, q)

    def right_side(self, q):
        return self.side(self.key_right, q)

    def bottom_side(self, q):
        return self.side(self.key_bottom, q)

    def top_side(self, q):
        return self.side(self.key_top, q)

    @property
    def mesh_surface(self) -> float:
        return float(self.radial_coords[-1] + self.global_variables["dist_tolerance"])

    @property
    def mesh_bottom(self) -> float:
        return float(self.radial_coords[0] - self.global_variables["dist_tolerance"])

    @property
    def solid_surface(self) -> float:
        vs = self.radial_variables["VS" if self.is_isotropic else "VSV"]
        tol = self.global_variables["dist_tolerance"]
        for i in range(len(self.radial_coords) - 1, 0, -1):
            if vs[i] > EPS:
                return float(self.radial_coords[i] + tol)
        return self.mesh_bottom - tol * 1000.

    def boundary_info_abc(self, key: str):
        """ExodusMesh::boundaryInfoABC: (present, outer, span) of RIGHT, BOTTOM or TOP."""
        ss = {"RIGHT": self.key_right, "BOTTOM": self.key_bottom, "TOP": self.key_top}.get(key)
        if ss is None:
            raise ExodusError("ExodusMesh::boundaryInfoABC || Invalid boundary key: " + key)
        if ss not in self.side_sets:
            return False, 0.0, 0.0
        inner, outer_r = self.inner_radius, self.outer_radius
        if key == "BOTTOM":
            return True, inner, inner - outer_r
        if key == "TOP":
            return True, outer_r, outer_r - inner
        if self.is_cartesian:
            outer = float(self.coords[:, 0].max())
        else:
            outer = float(np.max(np.arctan2(self.coords[:, 0], self.coords[:, 1])))
        return True, outer, outer

    # geodesy::getInnerRadius / getOuterRadius: the mesh bottom and surface
    @property
    def inner_radius(self) -> float:
        return self.mesh_bottom

    @property
    def outer_radius(self) -> float:
        return self.mesh_surface

    def summary(self) -> dict:
        """The figures of ExodusMesh::verbose."""
        gt = self.geometry_type
        return {"file": os.path.basename(self.path), "crdsys": self.records.get("crdsys"),
                "model": self.records.get("model"), "isotropic": self.is_isotropic,
                "attenuation": self.has_attenuation, "elements": self.num_quads,
                "nodes": self.num_nodes,
                "geometry": {"spherical": int(np.sum(gt == 0)), "linear": int(np.sum(gt == 1)),
                             "semi-spherical": int(np.sum(gt == 2))},
                "fluid": int(self.is_fluid.sum()), "solid": int(self.num_quads - self.is_fluid.sum()),
                "side_sets": {k: len(v) for k, v in self.side_sets.items()},
                "discontinuities": len(self.discontinuities)}
