"""Volumetric 3-D models on structured grids (the reference's StructuredGridV3D), for the
preloop.

Follows SOLVER/src/models3D: Model3D::buildInparam and computeElemSPZ (Model3D.cpp),
Volumetric3D::buildInparam (volumetric/Volumetric3D.cpp:135-200), StructuredGridV3D
(volumetric/StructuredGridV3D.cpp: constructor, getProperties), sg_tools.hpp (inparam
parsing, units, longitude range), Model3D.hpp (inplaneScope, coordsFromMeshToModel) and
StructuredGrid.hpp (reading with the data-rank shuffle; multilinear interpolation with
vector_tools::linearInterpSorted factors). The properties a grid returns are applied to
the quads by preloop.py as Material::addProperty3D does.

Supported: horizontal LATITUDE_LONGITUDE / DISTANCE_AZIMUTH / XY_CARTESIAN, vertical DEPTH /
RADIUS, length and angle units, whole_element_inplane, reference kinds ABS / REF1D / REF3D /
REF_PERTURB, properties RHO, VP, VS, VPV, VPH, VSV, VSH, ETA, QMU, QKAPPA. Cij properties,
geometric and ocean-load 3-D models raise `Model3DError`.
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps


class Model3DError(RuntimeError):
    """A 3-D model input the preloop cannot use ("Class::method || text")."""


def _read_nc(path):
    """{name: array} of a NetCDF-3 (scipy) or NetCDF-4 (this package's HDF5 reader) file."""
    with open(path, "rb") as f:
        magic = f.read(4)
    if magic[:3] == b"CDF":
        from scipy.io import netcdf_file
        nc = netcdf_file(path, "r", mmap=False)
        out = {k: np.array(v.data) for k, v in nc.variables.items()}
        nc.close()
        return out
    if magic == b"\x89HDF":
        from . import hdf5
        h = hdf5.File(path)
        return _LazyH5(h)
    raise Model3DError("NetCDF_Reader::open || Not a NetCDF file: %s" % path)


class _LazyH5(dict):
    def __init__(self, h):
        super().__init__()
        self._h = h

    def __contains__(self, k):
        return k in self._h.datasets

    def __getitem__(self, k):
        if k not in self._h.datasets:
            raise KeyError(k)
        return self._h.datasets[k].read()


class StructuredGrid:
    """StructuredGrid<D, double>: coordinates, data [nvar, n0, n1, ...] and multilinear
    interpolation; a coordinate outside its axis (beyond the end by more than the range
    times machine epsilon) is out of range."""

    def __init__(self, path, coord_vars, data_info, shuffle):
        if sorted(shuffle) != list(range(len(coord_vars))):
            raise Model3DError("StructuredGrid::StructuredGrid || Invalid data ranks to shuffle.")
        nc = _read_nc(path)
        self.coords = []
        for name in coord_vars:
            if name not in nc:
                raise Model3DError("NetCDF_Reader::readVectorDouble || Variable not found: %s || "
                                   "NetCDF file: %s" % (name, path))
            self.coords.append(np.asarray(nc[name], dtype=np.float64).reshape(-1).copy())
        unique = sorted({v for v, _ in data_info})
        self.rank_factor = [(unique.index(v), f) for v, f in data_info]
        data = []
        for v in unique:
            if v not in nc:
                raise Model3DError("NetCDF_Reader::readTensorDouble || Variable not found: %s || "
                                   "NetCDF file: %s" % (v, path))
            data.append(np.transpose(np.asarray(nc[v], dtype=np.float64), axes=shuffle))
        self.data = np.stack(data, axis=0)
        for d, c in enumerate(self.coords):
            if len(c) != self.data.shape[d + 1]:
                raise Model3DError("StructuredGrid::StructuredGrid || Incompatible grid sizes in "
                                   "coordinates and data. || Dimension: %s || NetCDF file: %s"
                                   % (coord_vars[d], path))
            if len(c) < 2:
                raise Model3DError("StructuredGrid::StructuredGrid || Too few grid points; at least "
                                   "two are required. || Dimension: %s" % coord_vars[d])
            if np.any(np.diff(c) <= 0):
                raise Model3DError("StructuredGrid::StructuredGrid || Coordinates are not ascendingly "
                                   "sorted. || Dimension: %s" % coord_vars[d])

    def compute(self, crd):
        """crd [n, D] -> (values [n, nvar] with the factors applied, in-range mask [n],
        first out-of-range dimension [n] or -1)."""
        crd = np.atleast_2d(np.asarray(crd, dtype=np.float64))
        n, D = crd.shape
        ok = np.ones(n, bool)
        dim_out = np.full(n, -1, np.int64)
        i0s, f1s = [], []
        for d in range(D):
            c = self.coords[d]
            tol = (c[-1] - c[0]) * EPS
            x = crd[:, d]
            bad = (x < c[0] - tol) | (x > c[-1] + tol)
            dim_out = np.where(ok & bad, d, dim_out)
            ok &= ~bad
            i1 = np.searchsorted(c, x, side="right")
            i1 = np.where(i1 == 0, 1, np.where(i1 == len(c), len(c) - 1, i1))
            i0 = i1 - 1
            f1 = (x - c[i0]) / (c[i1] - c[i0])
            i0s.append(i0)
            f1s.append(f1)
        nu = self.data.shape[0]
        u = np.zeros((n, nu))
        for corner in range(2 ** D):
            idx = [slice(None)]
            w = np.ones(n)
            left = corner
            for d in range(D):
                b = left % 2
                left //= 2
                idx.append(i0s[d] + b)
                w = w * (f1s[d] if b else 1. - f1s[d])
            vals = self.data[tuple(idx)]                                   # [nu, n]
            u += (w[:, None] * vals.T)
        out = np.stack([u[:, r] * f for r, f in self.rank_factor], axis=1)
        return out, ok, dim_out


class StructuredGridV3D:
    """One `list_of_3D_models` entry of class StructuredGridV3D."""

    REF_KINDS = ("ABS", "REF1D", "REF3D", "REF_PERTURB")
    PROPERTIES = ("RHO", "VP", "VS", "VPV", "VPH", "VSV", "VSH", "ETA", "QMU", "QKAPPA")

    def __init__(self, name, gm, root, inp_path, cartesian):
        self.name = name
        rc = root + ":coordinates"
        h = gm.get(rc + ":horizontal")
        if h == "DISTANCE_AZIMUTH":
            self.source_centered, self.xy, self.ellipticity = True, False, False
        elif h == "XY_CARTESIAN":
            if not cartesian:
                raise Model3DError("sg_tools::inparamHorizontal || XY_CARTESIAN is incompatible with a "
                                   "spherical mesh.")
            self.source_centered, self.xy, self.ellipticity = True, True, False
        elif h == "LATITUDE_LONGITUDE":
            self.source_centered, self.xy = False, False
            self.ellipticity = gm.get(rc + ":ellipticity", bool)
        else:
            raise Model3DError("sg_tools::inparamHorizontal || Parameter coordinates:horizontal must be "
                               "DISTANCE_AZIMUTH, || XY_CARTESIAN or LATITUDE_LONGITUDE. || Model name: "
                               + name)
        v = gm.get(rc + ":vertical")
        if v == "DEPTH":
            self.use_depth = True
            self.depth_solid = gm.get(rc + ":depth_below_solid_surface", bool)
        elif v == "RADIUS":
            self.use_depth, self.depth_solid = False, False
        else:
            raise Model3DError("sg_tools::inparamVertical || Parameter coordinates:vertical must be either "
                               "RADIUS or DEPTH. || Model name: " + name)
        vars_ = gm.get_vector(rc + ":nc_variables")
        rank = gm.get_vector(rc + ":data_rank", int)
        if len(vars_) != 3 or len(rank) != 3:
            raise Model3DError("sg_tools::inparamVarRank || The size of coordinates:nc_variables and "
                               "coordinates:data_rank must be 3. || Model name: " + name)
        lu = gm.get(rc + ":length_unit")
        length = {"m": 1., "km": 1e3}[lu] if lu in ("m", "km") else gm.get(rc + ":length_unit", float)
        angle = 1.0
        if not self.xy:
            angle = gm.get_options(rc + ":angle_unit", {"degree": math.pi / 180., "radian": 1.})
        undulated = gm.get(rc + ":undulated_geometry", bool)
        if undulated and self.use_depth:
            raise Model3DError("StructuredGridV3D::StructuredGridV3D || Cannot use depth as vertical "
                               "coordinate in undulated geometry. || Model name = " + name)
        self.center = gm.get(rc + ":whole_element_inplane", bool)
        rp = root + ":properties"
        self.props = []
        for i in range(gm.get(rp + ":[?]", int)):
            key = gm.get(rp + ":{%d}" % i)
            rpi = rp + ":[%d]:%s" % (i, key)
            if key.startswith("C"):
                raise Model3DError("StructuredGridV3D::StructuredGridV3D || Cij properties are not "
                                   "supported by this build. || Model name = " + name)
            if key not in self.PROPERTIES:
                raise Model3DError("Material::addProperty3D || Unacceptable property key: %s || Model "
                                   "name = %s" % (key, name))
            ref = gm.get_options(rpi + ":reference_kind", {k: k for k in self.REF_KINDS})
            self.props.append((key, gm.get(rpi + ":nc_var"), gm.get(rpi + ":factor", float), ref))
        fname = gm.get(root + ":nc_data_file")
        self.grid = StructuredGrid(inp_path(fname), vars_, [(p[1], p[2]) for p in self.props], rank)
        # sg_tools::constructUnits
        g = self.grid.coords
        if self.source_centered:
            if cartesian:
                g[0] *= length
                g[1] *= (length if self.xy else angle)
            else:
                g[0] *= angle
                g[1] *= angle
        else:
            g[0] *= angle / (math.pi / 180.)
            g[1] *= angle / (math.pi / 180.)
        g[2] *= length
        self.lon360 = False
        if not self.source_centered:
            lon = g[1]
            if lon[0] < 0. - EPS and lon[-1] > 180. + EPS:
                raise Model3DError("sg_tools::constructLon360 || Longitude range must be either "
                                   "[-180, 180] or [0, 360]. || Model name = " + name)
            self.lon360 = bool(lon[-1] > 180. + EPS)

    # Model3D::inplaneScope on (s, z) columns
    def _inplane_scope(self, sz, geo):
        check_r = self.source_centered and not self.xy
        g = self.grid.coords
        if geo.cartesian:
            a, b = sz[:, 0], sz[:, 1]
        else:
            r = np.hypot(sz[:, 0], sz[:, 1])
            t = np.where(r < EPS, 0., np.arccos(np.clip(sz[:, 1] / np.maximum(r, EPS), -1., 1.)))
            a, b = t, r
        if check_r and (a.max() < g[0][0] or a.min() > g[0][-1]):
            return False
        if self.use_depth:
            R = geo.outer_solid_radius if self.depth_solid else geo.outer_radius
            b = R - b
        if b.max() < g[2][0] or b.min() > g[2][-1]:
            return False
        return True

    # Model3D::coordsFromMeshToModel
    def _to_model(self, spz, geo):
        if self.source_centered:
            if geo.cartesian:
                crd = spz.copy()
                if self.xy:
                    crd[:, 0] = spz[:, 0] * np.cos(spz[:, 1])
                    crd[:, 1] = spz[:, 0] * np.sin(spz[:, 1])
            else:
                r = np.hypot(spz[:, 0], spz[:, 2])
                t = np.where(r < EPS, 0., np.arccos(np.clip(spz[:, 2] / np.maximum(r, EPS), -1., 1.)))
                crd = np.stack([t, spz[:, 1], r], axis=1)
        else:
            if geo.cartesian:
                if np.any(spz[:, 2] < spz[:, 0] * 10.):
                    raise Model3DError("Model3D::coordsFromMeshToModel || Invalid geographic location in "
                                       "Cartesian mesh. || Model name = " + self.name)
                t = spz[:, 0] / spz[:, 2]
                bend = np.stack([spz[:, 2] * np.sin(t), spz[:, 1], spz[:, 2] * np.cos(t)], axis=1)
                crd = geo.spz2llr(bend, self.ellipticity, self.lon360)
            else:
                crd = geo.spz2llr(spz, self.ellipticity, self.lon360)
        if self.use_depth:
            R = geo.outer_solid_radius if self.depth_solid else geo.outer_radius
            crd = crd.copy()
            crd[:, 2] = R - crd[:, 2]
        return crd

    def properties(self, nodal_sz, point_sz, point_nr, geo):
        """StructuredGridV3D::getProperties for one quad: (in_scope [25][nr_p] bool,
        values [25][nr_p][nprop]) per point, or None when the quad is out of the model."""
        if self.center and not self._inplane_scope(nodal_sz.mean(axis=0)[None, :], geo):
            return None
        if not self._inplane_scope(nodal_sz, geo):
            return None
        rows = []
        for p in range(25):
            nr = int(point_nr[p])
            phi = np.linspace(0., 2. * np.pi / nr * (nr - 1), nr) if nr > 1 else np.zeros(1)
            rows.append(np.stack([np.full(nr, point_sz[0, p]), phi, np.full(nr, point_sz[1, p])], axis=1))
        spz = np.concatenate(rows, axis=0)
        crd = self._to_model(spz, geo)
        vals, ok, dim_out = self.grid.compute(crd)
        if self.center:
            bad = (~ok) & (((self.source_centered and not self.xy) & (dim_out == 0)) | (dim_out == 2))
            if np.any(bad):
                k = int(np.nonzero(bad)[0][0])
                raise Model3DError("StructuredGridV3D::getProperties || A GLL point of an element is out of "
                                   "inplane model range,|| but coordinates:whole_element_inplane is set to "
                                   "true.|| Out-of_range coordinate = %g|| Out-of-range dimension = %d|| "
                                   "Model name = %s" % (crd[k, dim_out[k]], dim_out[k], self.name))
        if not ok.any():
            return None
        out_ok, out_v, r0 = [], [], 0
        for p in range(25):
            nr = int(point_nr[p])
            out_ok.append(ok[r0:r0 + nr])
            out_v.append(vals[r0:r0 + nr])
            r0 += nr
        return out_ok, out_v


def build_models(inp, cartesian):
    """Model3D::buildInparam: the activated entries of list_of_3D_models, in order."""
    gm = inp.model
    if not gm.contains("list_of_3D_models") or not gm._walk("list_of_3D_models"):
        return []
    models = []
    for i in range(gm.get("list_of_3D_models:[?]", int)):
        name = gm.get("list_of_3D_models:{%d}" % i)
        root = "list_of_3D_models:[%d]:%s" % (i, name)
        if not gm.get(root + ":activated", bool):
            continue
        cls = gm.get(root + ":class_name")
        if cls != "StructuredGridV3D":
            raise Model3DError("Model3D::buildInparam || 3-D model class %s is not supported by this "
                               "build (StructuredGridV3D only). || Model name: %s" % (cls, name))
        models.append(StructuredGridV3D(name, gm, root, inp.path, cartesian))
    return models


def lin_interp_phi(vals, nr_out):
    """PhysicalProperty::linInterpPhi: values on nr_in equal phi slices -> nr_out slices."""
    vals = np.asarray(vals, dtype=np.float64)
    nr_in = len(vals)
    if nr_in == nr_out:
        return vals.copy()
    d_in, d_out = 1. / nr_in, 1. / nr_out
    out = np.empty(nr_out)
    for a in range(nr_out):
        phi = a * d_out
        l0 = int(phi / d_in)
        l1 = 0 if l0 == nr_in - 1 else l0 + 1
        out[a] = vals[l0] + (vals[l1] - vals[l0]) / d_in * (phi - l0 * d_in)
    return out


def try_reduce_1d(arrs):
    """PhysicalProperty::tryReduceTo1D on the 25 per-point arrays: 1-D if every point is
    constant in phi (relative to its norm)."""
    for a in arrs:
        if np.linalg.norm(a - a[0]) > np.linalg.norm(a) * EPS:
            return False
    return True

