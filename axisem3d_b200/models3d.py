"""3-D models on structured grids for the preloop: volumetric (StructuredGridV3D), geometric
(StructuredGridG3D, Ellipticity) and ocean-load (StructuredGridO3D) models of the reference.

Follows SOLVER/src/models3D: Model3D::buildInparam and computeElemSPZ (Model3D.cpp),
Volumetric3D::buildInparam (volumetric/Volumetric3D.cpp:135-200), StructuredGridV3D
(volumetric/StructuredGridV3D.cpp: constructor, getProperties), Geometric3D::buildInparam
(geometric/Geometric3D.cpp:115-190), StructuredGridG3D::getUndulation, Ellipticity::
getUndulation, OceanLoad3D::buildInparam and StructuredGridO3D::getSumRhoDepth, sg_tools.hpp
(inparam parsing, units, longitude range), Model3D.hpp (inplaneScope, coordsFromMeshToModel)
and StructuredGrid.hpp (reading with the data-rank shuffle; multilinear interpolation with
vector_tools::linearInterpSorted factors). What a model returns is applied to the quads by
preloop.py: properties as Material::addProperty3D does, undulation as Undulation::
addUndulation, sum(rho * depth) as OceanLoad::addSumRhoDepth.

Supported: horizontal LATITUDE_LONGITUDE / DISTANCE_AZIMUTH / XY_CARTESIAN, vertical DEPTH /
RADIUS, length and angle units, whole_element_inplane, undulated_geometry, reference kinds
ABS / REF1D / REF3D / REF_PERTURB, properties RHO, VP, VS, VPV, VPH, VSV, VSH, ETA, QMU,
QKAPPA. Cij properties raise `Model3DError`.
"""
from __future__ import annotations

import math

import numpy as np

EPS = np.finfo(np.float64).eps
DEPS = 1e-12                  # numerical::dEpsilon, the reference's tolerance for 1-D / zero tests


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
    times 1e-12, as vector_tools::linearInterpSorted allows) is out of range."""

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
            tol = (c[-1] - c[0]) * DEPS                # vector_tools::linearInterpSorted
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


# ------------------------------------------------ sg_tools and Model3D helpers ---
def _horizontal(gm, rc, name, cartesian):
    """sg_tools::inparamHorizontal: (source_centered, xy, ellipticity)."""
    h = gm.get(rc + ":horizontal")
    if h == "DISTANCE_AZIMUTH":
        return True, False, False
    if h == "XY_CARTESIAN":
        if not cartesian:
            raise Model3DError("sg_tools::inparamHorizontal || XY_CARTESIAN is incompatible with a "
                               "spherical mesh.")
        return True, True, False
    if h == "LATITUDE_LONGITUDE":
        return False, False, gm.get(rc + ":ellipticity", bool)
    raise Model3DError("sg_tools::inparamHorizontal || Parameter coordinates:horizontal must be "
                       "DISTANCE_AZIMUTH, || XY_CARTESIAN or LATITUDE_LONGITUDE. || Model name: " + name)


def _vertical(gm, rc, name):
    """sg_tools::inparamVertical: (use_depth, depth_below_solid_surface)."""
    v = gm.get(rc + ":vertical")
    if v == "DEPTH":
        return True, gm.get(rc + ":depth_below_solid_surface", bool)
    if v == "RADIUS":
        return False, False
    raise Model3DError("sg_tools::inparamVertical || Parameter coordinates:vertical must be either "
                       "RADIUS or DEPTH. || Model name: " + name)


def _var_rank(gm, rc, name, n):
    """sg_tools::inparamVarRank<n>: coordinate variable names and the data rank."""
    vars_ = gm.get_vector(rc + ":nc_variables")
    rank = gm.get_vector(rc + ":data_rank", int)
    if len(vars_) != n or len(rank) != n:
        raise Model3DError("sg_tools::inparamVarRank || The size of coordinates:nc_variables and "
                           "coordinates:data_rank must be %d. || Model name: %s" % (n, name))
    return vars_, rank


def _units(gm, rc, xy):
    """sg_tools::inparamUnits: (length unit, angle unit)."""
    lu = gm.get(rc + ":length_unit")
    length = {"m": 1., "km": 1e3}[lu] if lu in ("m", "km") else gm.get(rc + ":length_unit", float)
    angle = 1.0
    if not xy:
        angle = gm.get_options(rc + ":angle_unit", {"degree": math.pi / 180., "radian": 1.})
    return length, angle


def _construct_units(g, source_centered, xy, vertical, length, angle, cartesian):
    """sg_tools::constructUnits on the grid coordinates g (in place): horizontal axes to
    metres / radians (source-centred) or degrees (geographic), the vertical axis to metres."""
    if source_centered:
        if cartesian:
            g[0] *= length
            g[1] *= (length if xy else angle)
        else:
            g[0] *= angle
            g[1] *= angle
    else:
        g[0] *= angle / (math.pi / 180.)
        g[1] *= angle / (math.pi / 180.)
    if vertical:
        g[2] *= length


def _lon360(g, name):
    """sg_tools::constructLon360: longitudes in [0, 360] rather than [-180, 180]."""
    lon = g[1]
    if lon[0] < 0. - DEPS and lon[-1] > 180. + DEPS:
        raise Model3DError("sg_tools::constructLon360 || Longitude range must be either "
                           "[-180, 180] or [0, 360]. || Model name = " + name)
    return bool(lon[-1] > 180. + DEPS)


def inplane_scope(sz, geo, check_r, rmin, rmax, check_z, zmin, zmax, use_depth, depth_solid):
    """Model3D::inplaneScope (models3D/Model3D.hpp:69-109) on (s, z) rows: the quad may touch
    the model's horizontal (theta or s) and vertical (r / z or depth) ranges."""
    if not check_r and not check_z:
        return True
    sz = np.atleast_2d(sz)
    if geo.cartesian:
        a, b = sz[:, 0], sz[:, 1]
    else:
        r = np.hypot(sz[:, 0], sz[:, 1])
        t = np.where(r < DEPS, 0., np.arccos(np.clip(sz[:, 1] / np.maximum(r, DEPS), -1., 1.)))
        a, b = t, r
    if check_r and (a.max() < rmin or a.min() > rmax):
        return False
    if check_z:
        if use_depth:
            R = geo.outer_solid_radius if depth_solid else geo.outer_radius
            b = R - b
        if b.max() < zmin or b.min() > zmax:
            return False
    return True


def to_model(spz, geo, source_centered, xy, ellipticity, lon360, use_depth, depth_solid, name):
    """Model3D::coordsFromMeshToModel (Model3D.hpp:111-175): mesh (s, phi, z) rows to the
    model's coordinates (theta, phi, r), (x, y, z), (s, phi, z) or (lat, lon, r), with depth
    for r when the model uses depth."""
    spz = np.atleast_2d(spz)
    if source_centered:
        if geo.cartesian:
            crd = spz.copy()
            if xy:
                crd[:, 0] = spz[:, 0] * np.cos(spz[:, 1])
                crd[:, 1] = spz[:, 0] * np.sin(spz[:, 1])
        else:
            r = np.hypot(spz[:, 0], spz[:, 2])
            t = np.where(r < DEPS, 0., np.arccos(np.clip(spz[:, 2] / np.maximum(r, DEPS), -1., 1.)))
            crd = np.stack([t, spz[:, 1], r], axis=1)
    else:
        if geo.cartesian:
            if np.any(spz[:, 2] < spz[:, 0] * 10.):
                raise Model3DError("Model3D::coordsFromMeshToModel || Invalid geographic location in "
                                   "Cartesian mesh. || Model name = " + name)
            t = spz[:, 0] / spz[:, 2]
            bend = np.stack([spz[:, 2] * np.sin(t), spz[:, 1], spz[:, 2] * np.cos(t)], axis=1)
            crd = geo.spz2llr(bend, ellipticity, lon360)
        else:
            crd = geo.spz2llr(spz, ellipticity, lon360)
    if use_depth:
        R = geo.outer_solid_radius if depth_solid else geo.outer_radius
        crd = crd.copy()
        crd[:, 2] = R - crd[:, 2]
    return crd


def element_spz(point_sz, point_nr, und=None, cartesian=True):
    """Model3D::computeElemSPZ (Model3D.cpp:16-66): the (s, phi, z) of every (point, slice)
    of a quad, slices at phi = 2 pi k / nr of each point; with `und` (per-point undulation,
    1 or nr values) the points move by it along z (Cartesian) or along r (spherical)."""
    rows = []
    for p in range(25):
        nr = int(point_nr[p])
        phi = np.linspace(0., 2. * np.pi / nr * (nr - 1), nr) if nr > 1 else np.zeros(1)
        s0, z0 = point_sz[0, p], point_sz[1, p]
        s, z = np.full(nr, s0), np.full(nr, z0)
        if und is not None:
            u = np.broadcast_to(np.asarray(und[p], np.float64), (nr,))
            if cartesian:
                z = z + u
            else:
                r = math.hypot(s0, z0)
                th = 0. if r < DEPS else math.acos(z0 / r)
                s = s + u * math.sin(th)
                z = z + u * math.cos(th)
        rows.append(np.stack([s, phi, z], axis=1))
    return np.concatenate(rows, axis=0)


def _split(vals, point_nr, npts=25):
    out, r0 = [], 0
    for p in range(npts):
        nr = int(point_nr[p])
        out.append(vals[r0:r0 + nr])
        r0 += nr
    return out


class StructuredGridV3D:
    """One `list_of_3D_models` entry of class StructuredGridV3D."""
    kind = "volumetric"

    REF_KINDS = ("ABS", "REF1D", "REF3D", "REF_PERTURB")
    PROPERTIES = ("RHO", "VP", "VS", "VPV", "VPH", "VSV", "VSH", "ETA", "QMU", "QKAPPA")

    def __init__(self, name, gm, root, inp_path, cartesian):
        self.name = name
        rc = root + ":coordinates"
        self.source_centered, self.xy, self.ellipticity = _horizontal(gm, rc, name, cartesian)
        self.use_depth, self.depth_solid = _vertical(gm, rc, name)
        vars_, rank = _var_rank(gm, rc, name, 3)
        length, angle = _units(gm, rc, self.xy)
        undulated = gm.get(rc + ":undulated_geometry", bool)
        self.undulated = undulated
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
                                   "supported by this engine. || Model name = " + name)
            if key not in self.PROPERTIES:
                raise Model3DError("Material::addProperty3D || Unacceptable property key: %s || Model "
                                   "name = %s" % (key, name))
            ref = gm.get_options(rpi + ":reference_kind", {k: k for k in self.REF_KINDS})
            self.props.append((key, gm.get(rpi + ":nc_var"), gm.get(rpi + ":factor", float), ref))
        fname = gm.get(root + ":nc_data_file")
        self.grid = StructuredGrid(inp_path(fname), vars_, [(p[1], p[2]) for p in self.props], rank)
        _construct_units(self.grid.coords, self.source_centered, self.xy, True, length, angle, cartesian)
        self.lon360 = False if self.source_centered else _lon360(self.grid.coords, name)

    def _inplane_scope(self, sz, geo):
        g = self.grid.coords
        return inplane_scope(sz, geo, self.source_centered and not self.xy, g[0][0], g[0][-1], True, g[2][0],
                             g[2][-1], self.use_depth, self.depth_solid)

    def _to_model(self, spz, geo):
        return to_model(spz, geo, self.source_centered, self.xy, self.ellipticity, self.lon360, self.use_depth,
                        self.depth_solid, self.name)

    def properties(self, nodal_sz, point_sz, point_nr, geo, und=None):
        """StructuredGridV3D::getProperties for one quad: (in_scope [25][nr_p] bool,
        values [25][nr_p][nprop]) per point, or None when the quad is out of the model.
        `und`: the quad's undulation per point, used when the model asks for the
        undulated geometry."""
        if self.center and not self._inplane_scope(nodal_sz.mean(axis=0)[None, :], geo):
            return None
        if not self._inplane_scope(nodal_sz, geo):
            return None
        spz = element_spz(point_sz, point_nr, und if self.undulated else None, geo.cartesian)
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


class StructuredGridG3D:
    """A geometric 3-D model (models3D/geometric/StructuredGridG3D.cpp): an undulation
    map on a 2-D grid applied between two radii (or depths) min < interface < max, ramped
    linearly from 0 at min and max to the map's value at the interface."""
    kind = "geometric"

    def __init__(self, name, gm, root, inp_path, cartesian):
        self.name = name
        rc = root + ":coordinates"
        self.source_centered, self.xy, self.ellipticity = _horizontal(gm, rc, name, cartesian)
        self.use_depth, self.depth_solid = _vertical(gm, rc, name)
        vars_, rank = _var_rank(gm, rc, name, 2)
        length, angle = _units(gm, rc, self.xy)
        rr = root + ":undulation_range"
        interface = gm.get(rr + ":interface", float)
        lo, hi = gm.get(rr + ":min_max:[0]", float), gm.get(rr + ":min_max:[1]", float)
        if interface >= hi or interface <= lo:
            raise Model3DError("Geometric3D::buildInparam || undulation_range:interface must lie within "
                               "undulation_range:min_max. || Model name: %s || Class name: StructuredGridG3D"
                               % name)
        self.interface, self.min, self.max = interface * length, lo * length, hi * length
        ru = root + ":undulation_data"
        self.grid = StructuredGrid(inp_path(gm.get(root + ":nc_data_file")), vars_,
                                   [(gm.get(ru + ":nc_var"), gm.get(ru + ":factor", float))], rank)
        _construct_units(self.grid.coords, self.source_centered, self.xy, False, length, angle, cartesian)
        self.lon360 = False if self.source_centered else _lon360(self.grid.coords, name)

    def at(self, spz, geo):
        """StructuredGridG3D::getUndulation on (s, phi, z) rows: (undulation, any in scope)."""
        crd = to_model(spz, geo, self.source_centered, self.xy, self.ellipticity, self.lon360, self.use_depth,
                       self.depth_solid, self.name)
        und = np.zeros(len(crd))
        rd = crd[:, 2]
        vals, ok, _ = self.grid.compute(crd[:, :2])
        inr = (rd >= self.min) & (rd <= self.max) & ok
        v = vals[:, 0]
        below = rd < self.interface
        ramp = np.where(below, v / (self.interface - self.min) * (rd - self.min),
                        v / (self.max - self.interface) * (self.max - rd))
        und[inr] = ramp[inr]
        return und, bool(inr.any())

    def undulation(self, nodal_sz, point_sz, point_nr, geo):
        """Per-point undulation of one quad, or None when it is out of the model."""
        g = self.grid.coords
        if not inplane_scope(nodal_sz, geo, self.source_centered and not self.xy, g[0][0], g[0][-1], True,
                             self.min, self.max, self.use_depth, self.depth_solid):
            return None
        und, any_in = self.at(element_spz(point_sz, point_nr), geo)
        return _split(und, point_nr) if any_in else None


class Ellipticity:
    """The Ellipticity geometric model (models3D/geometric/Ellipticity.cpp): every point
    moves from its radius r to the ellipsoid of flattening f(r) through it, a b / sqrt((a
    cos t)^2 + (b sin t)^2) - r with b = (1 - f)^(2/3) r and a = b / (1 - f), t the
    geographic colatitude; nothing on a Cartesian mesh or with zero flattening."""
    kind = "geometric"

    def __init__(self, name):
        self.name = name

    def at(self, spz, geo):
        if geo.cartesian or geo.outer_flattening < DEPS:
            return np.zeros(len(np.atleast_2d(spz))), False
        llr = to_model(spz, geo, False, False, False, False, False, False, self.name)
        tpr = geo.llr2tpr(llr, False)
        r, t = tpr[:, 2], tpr[:, 0]
        f = geo.flattening(r)
        b = (1. - f) ** (2. / 3.) * r
        a = b / (1. - f)
        tmp = (a * np.cos(t)) ** 2 + (b * np.sin(t)) ** 2
        return a * b / np.maximum(np.sqrt(tmp), DEPS) - r, True

    def undulation(self, nodal_sz, point_sz, point_nr, geo):
        und, any_in = self.at(element_spz(point_sz, point_nr), geo)
        return _split(und, point_nr) if any_in else None


class StructuredGridO3D:
    """An ocean-load 3-D model (models3D/ocean_load/StructuredGridO3D.cpp): sum(rho * depth)
    of the water column on a 2-D grid, taken where it is positive."""
    kind = "ocean"

    def __init__(self, name, gm, root, inp_path, cartesian):
        self.name = name
        rc = root + ":coordinates"
        self.source_centered, self.xy, self.ellipticity = _horizontal(gm, rc, name, cartesian)
        vars_, rank = _var_rank(gm, rc, name, 2)
        length, angle = _units(gm, rc, self.xy)
        rd = root + ":data_sum_rho_depth"
        self.grid = StructuredGrid(inp_path(gm.get(root + ":nc_data_file")), vars_,
                                   [(gm.get(rd + ":nc_var"), gm.get(rd + ":factor", float))], rank)
        _construct_units(self.grid.coords, self.source_centered, self.xy, False, length, angle, cartesian)
        self.lon360 = False if self.source_centered else _lon360(self.grid.coords, name)

    def sum_rho_depth(self, nodal_sz, edge_spz, edge_nr, geo):
        """StructuredGridO3D::getSumRhoDepth on the 5 surface-edge points of one quad (rows
        of (s, phi, z), 1 per slice): per-point arrays, or None when out of the model."""
        g = self.grid.coords
        if not inplane_scope(nodal_sz, geo, self.source_centered and not self.xy, g[0][0], g[0][-1], False,
                             0., 0., False, False):
            return None
        crd = to_model(edge_spz, geo, self.source_centered, self.xy, self.ellipticity, self.lon360, False, False,
                       self.name)
        vals, ok, _ = self.grid.compute(crd[:, :2])
        v = np.where(ok & (vals[:, 0] > 0.), vals[:, 0], 0.)
        if not np.any(ok & (vals[:, 0] > 0.)):
            return None
        return _split(v, edge_nr, 5)


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
        if cls == "StructuredGridV3D":
            models.append(StructuredGridV3D(name, gm, root, inp.path, cartesian))
        elif cls == "StructuredGridG3D":
            models.append(StructuredGridG3D(name, gm, root, inp.path, cartesian))
        elif cls == "Ellipticity":
            if any(isinstance(m, Ellipticity) for m in models):
                raise Model3DError("Geometric3D::buildInparam || Ellipticity model cannot be added more "
                                   "than once.")
            models.append(Ellipticity(name))
        elif cls == "StructuredGridO3D":
            models.append(StructuredGridO3D(name, gm, root, inp.path, cartesian))
        else:
            raise Model3DError("Model3D::buildInparam || 3-D model class %s is not supported by this "
                               "build. || Model name: %s" % (cls, name))
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
        if np.linalg.norm(a - a[0]) > np.linalg.norm(a) * DEPS:
            return False
    return True

