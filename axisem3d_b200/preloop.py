"""The preloop: an Exodus mesh and the reference's input files -> a `Model` for the engine.

This follows the reference's preloop (SOLVER/src/main.cpp:60-640) in its order and rules:
geodesy (preloop/exodus/geodesy.{hpp,cpp}), absorbing boundaries (exodus/ABC.cpp), the Nr
field (nr_field/NrField*.cpp, ExodusMesh::formNrAtNodes), quads (se_model/quad/Quad.cpp:
mapping, material, integral factor, normals, dt), materials (quad/physical/Material.cpp,
AttBuilder.cpp), GLL points and their boundaries (se_model/gll/GLLPoint.{hpp,cpp}), the time
step (SE_Model::computeDt), sources (preloop/source/Source.cpp, Mechanism.cpp, core STF.cpp)
and station groups (preloop/output/StationOutput.cpp).

Supported inputs: 1-D models from the Exodus radial profile (isotropic or transversely
isotropic, fluid layers, attenuation NONE / FULL / CG4), Cartesian and spherical meshes with
all three mappings, Clayton and sponge boundaries, constant Nr (bounded by the in-plane
resolution, rounded to FFT-friendly sizes), moment-tensor and force sources with Gaussian
source-time functions anywhere in the solid, and solid station groups recording displacement
(channels U, U1, U2, U3, U_NORM in the spz, RTZ, ENZ or xyz frame). Anything else named in the
inputs (3-D models, other Nr fields, fluid-pressure sources, file STFs, strain / stress /
curl channels, fluid stations, element output) raises `PreloopError` naming it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib as L
from .exodus import ExodusMesh
from .inparam import Inparam
from .meshgen import (cg4_correct, geometry_batch, iso_with_attenuation, lagrange, round_dt, tables,
                      tiso_with_attenuation, weights_cg4)
from .model import STF, Model
from .models3d import Model3DError, build_models, lin_interp_phi
from .solver import att_alpha_beta_gamma, quad_dt

EPS = np.finfo(np.float64).eps
DEPS = 1e-12                  # numerical::dEpsilon, the reference's tolerance for 1-D / zero tests
# vicinity::constants (mesh/topology/vicinity.hpp), nPol = 4
NODE_IPNT = (0, 20, 24, 4)
EDGE_IPNT = ((0, 5, 10, 15, 20), (20, 21, 22, 23, 24), (24, 19, 14, 9, 4), (4, 3, 2, 1, 0))
# exodus element_type -> this package's mapping codes
MAPPING = {0: L.AXG_MAP_SPHERICAL, 1: L.AXG_MAP_LINEAR, 2: L.AXG_MAP_SEMI_SPHERICAL}


class PreloopError(RuntimeError):
    """An input the preloop cannot use; messages follow "Class::method || text"."""


def cround(x):
    """C++ round(): halves away from zero."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


# ------------------------------------------------------------------ Nr field ---
def is_lucky(n: int) -> bool:
    """NrField::isLuckyNumber: largest prime factor <= 13, at most one factor 11 or 13."""
    num = n
    for p in (2, 3, 5, 7, 11, 13):
        while num % p == 0:
            num //= p
    if num != 1:
        return False
    e = 0
    num = n
    while num % 11 == 0:
        num //= 11
        e += 1
    while num % 13 == 0:
        num //= 13
        e += 1
    return e <= 1


def next_lucky(n: int) -> int:
    """NrField::nextLuckyNumber: the smallest lucky number >= n."""
    m = max(int(n), 1)
    while not is_lucky(m):
        m += 1
    return m


# ------------------------------------------------------------------- geodesy ---
class Geodesy:
    """geodesy::setup and the transforms of geodesy.hpp."""

    FLATTENING = {"SPHERE": 0., "WGS84": 1. / 298.257223563, "GRS80": 1. / 298.257222101,
                  "SPECFEM3D_GLOBE": 1. / 299.8}

    def __init__(self, mesh: ExodusMesh, inp: Inparam):
        self.cartesian = mesh.is_cartesian
        self.outer_radius = mesh.mesh_surface
        self.inner_radius = mesh.mesh_bottom
        self.outer_solid_radius = mesh.solid_surface
        key = "geodesy:flattening_on_surface"
        fl = inp.model.get(key)
        try:
            f = self.FLATTENING[fl] if fl in self.FLATTENING else float(fl)
        except ValueError:
            raise PreloopError("geodesy::setup || Invalid %s: %s" % (key, fl))
        if f < DEPS or self.cartesian:
            f = 0.
        self.outer_flattening = f
        self.ellip_r = mesh.ellipticity[0].copy()
        self.ellip_f = mesh.ellipticity[1] * f
        gz = inp.model.get("geodesy:lat_lon_north_pole_mesh")
        if gz == "SOURCE":
            name = inp.source.get("list_of_sources:{0}")
            root = "list_of_sources:[0]:%s:location" % name
            try:
                lat = inp.source.get_bounded(root + ":latitude_longitude:[0]", -90., 90.)
                lon = inp.source.get_bounded(root + ":latitude_longitude:[1]", -180., 180.)
            except Exception:
                raise PreloopError("geodesy::setup || Error determining the geographic location of the "
                                   "first || source in list_of_sources in inparam.source.yaml; || "
                                   "location:latitude_longitude must be presented.")
            if inp.source.contains(root + ":depth"):
                depth = inp.source.get_bounded(root + ":depth", 0., self.outer_radius)
                solid = inp.source.get(root + ":depth_below_solid_surface", bool)
                r = (self.outer_solid_radius if solid else self.outer_radius) - depth
            else:
                r = inp.source.get_bounded(root + ":radius", 0., self.outer_radius)
        else:
            lat = inp.model.get_bounded("geodesy:lat_lon_north_pole_mesh:[0]", -90., 90.)
            lon = inp.model.get_bounded("geodesy:lat_lon_north_pole_mesh:[1]", -180., 180.)
            r = self.outer_radius
        self.llr_axis = np.array([lat, lon, r])
        th, ph, _ = self.llr2tpr(self.llr_axis[None, :], True)[0]
        Q = np.array([[math.cos(th) * math.cos(ph), -math.sin(ph), math.sin(th) * math.cos(ph)],
                      [math.cos(th) * math.sin(ph), math.cos(ph), math.sin(th) * math.sin(ph)],
                      [-math.sin(th), 0., math.cos(th)]])
        self.src2geo = Q.T

    def flattening(self, r):
        """geodesy::computeFlattening: the ellipticity curve, clamped at its ends."""
        r = np.atleast_1d(np.asarray(r, dtype=np.float64))
        R, F = self.ellip_r, self.ellip_f
        tol = (R[-1] - R[0]) * EPS
        out = np.empty_like(r)
        for k, x in enumerate(r):
            if x < R[0] - tol or x > R[-1] + tol:
                out[k] = F[-1] if x > R[-1] else F[0]
                continue
            i1 = int(np.searchsorted(R, x, side="right"))
            i1 = 1 if i1 == 0 else (len(R) - 1 if i1 == len(R) else i1)
            i0 = i1 - 1
            f1 = (x - R[i0]) / (R[i1] - R[i0])
            out[k] = F[i0] * (1. - f1) + F[i1] * f1
        return out

    def llr2tpr(self, llr, ellipticity):
        llr = np.atleast_2d(llr)
        tpr = np.empty_like(llr, dtype=np.float64)
        t = np.radians(llr[:, 0])
        if ellipticity:
            t = np.arctan(np.tan(t) * (self.flattening(llr[:, 2]) - 1.) ** 2)
        tpr[:, 0] = np.pi / 2. - t
        tpr[:, 1] = np.radians(llr[:, 1])
        tpr[:, 2] = llr[:, 2]
        return tpr

    def tpr2llr(self, tpr, ellipticity):
        tpr = np.atleast_2d(tpr)
        llr = np.empty_like(tpr, dtype=np.float64)
        lat = np.pi / 2. - tpr[:, 0]
        if ellipticity:
            lat = np.arctan(np.tan(lat) / (self.flattening(tpr[:, 2]) - 1.) ** 2)
        llr[:, 0] = np.degrees(lat)
        llr[:, 1] = np.degrees(tpr[:, 1])
        llr[:, 2] = tpr[:, 2]
        return llr

    @staticmethod
    def _xy2sphi(x, y, undefined):
        s = np.hypot(x, y)
        with np.errstate(invalid="ignore"):
            p = np.where((np.abs(x) < DEPS) & (np.abs(y) < DEPS), undefined, np.arctan2(y, x))
        return s, p

    def llr2spz(self, llr, ellipticity):
        tpr = self.llr2tpr(llr, ellipticity)
        xyz = np.stack([tpr[:, 2] * np.sin(tpr[:, 0]) * np.cos(tpr[:, 1]),
                        tpr[:, 2] * np.sin(tpr[:, 0]) * np.sin(tpr[:, 1]),
                        tpr[:, 2] * np.cos(tpr[:, 0])], axis=1)
        src = xyz @ self.src2geo.T
        err = np.finfo(np.float64).min
        s, p = self._xy2sphi(src[:, 0], src[:, 1], err)
        p = np.where(p < err * .9, tpr[:, 1], p)
        return np.stack([s, p, src[:, 2]], axis=1)

    def spz2llr(self, spz, ellipticity, lon360):
        spz = np.atleast_2d(spz)
        xyz = np.stack([spz[:, 0] * np.cos(spz[:, 1]), spz[:, 0] * np.sin(spz[:, 1]), spz[:, 2]], axis=1)
        geo = xyz @ self.src2geo
        err = np.finfo(np.float64).min
        s, p = self._xy2sphi(geo[:, 0], geo[:, 1], err)
        p = np.where(p < err * .9, spz[:, 1], p)
        r = np.hypot(s, geo[:, 2])
        t = np.where(r < DEPS, 0., np.arccos(np.clip(geo[:, 2] / np.maximum(r, DEPS), -1., 1.)))
        llr = self.tpr2llr(np.stack([t, p, r], axis=1), ellipticity)
        llr[:, 2] = np.hypot(spz[:, 0], spz[:, 2])
        if lon360:
            llr[:, 1] = np.where(llr[:, 1] < 0., llr[:, 1] + 360., llr[:, 1])
        else:
            llr[:, 1] = np.where(llr[:, 1] > 180., llr[:, 1] - 360., llr[:, 1])
        return llr

    def back_azimuth(self, llr, ellipticity):
        """geodesy::backAzimuth."""
        src = self.llr2tpr(self.llr_axis[None, :], ellipticity)[0]
        d, e = math.sin(src[1]), -math.cos(src[1])
        f, c = -math.sin(src[0]), math.cos(src[0])
        a, b = f * e, -f * d
        tpr = self.llr2tpr(llr, ellipticity)
        dd, ee = np.sin(tpr[:, 1]), -np.cos(tpr[:, 1])
        ff, cc = -np.sin(tpr[:, 0]), np.cos(tpr[:, 0])
        gg, hh = -cc * ee, cc * dd
        x = (a - gg) ** 2 + (b - hh) ** 2 + (c - ff) ** 2 - 2.
        y = (a - dd) ** 2 + (b - ee) ** 2 + c * c - 2.
        return self._xy2sphi(x, y, 0.)[1]


def sz2rtheta(s, z):
    """geodesy::sz2rtheta: r and the polar angle acos(z / r) (0 at r = 0)."""
    r = np.hypot(s, z)
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(r < DEPS, 0., np.arccos(np.clip(z / np.maximum(r, DEPS), -1., 1.)))
    return r, t


# ----------------------------------------------------------------------- ABC ---
@dataclass
class ABC:
    """ABC::buildInparam: the boundaries the user asked for and the mesh has."""
    user_keys: List[str] = field(default_factory=list)
    keys: List[str] = field(default_factory=list)
    clayton: bool = False
    sponge: bool = False
    outer_span: dict = field(default_factory=dict)
    expr_solid: str = ""
    expr_fluid: str = ""
    t0: float = 0.0

    def u0(self, span, vp, vs, rho, fluid):
        """ABC::getU0Solid / getU0Fluid: the user's gamma expression."""
        expr = self.expr_fluid if fluid else self.expr_solid
        env = {"VP": vp, "RHO": rho, "SPAN": span, "T0": self.t0, "exp": np.exp, "sqrt": np.sqrt,
               "log": np.log, "abs": np.abs, "sin": np.sin, "cos": np.cos, "tan": np.tan, "pi": math.pi,
               "pow": np.power, "min": np.minimum, "max": np.maximum}
        if not fluid:
            env["VS"] = vs
        try:
            return np.asarray(eval(expr.replace("^", "**"), {"__builtins__": {}}, env), dtype=np.float64)
        except Exception as ex:
            raise PreloopError("ABC::buildInparam || Error evaluating Kosloff_Kosloff::gamma_expr_%s: %s"
                               % ("fluid" if fluid else "solid", ex))


def build_abc(mesh: ExodusMesh, inp: Inparam) -> ABC:
    gm = inp.model
    root = "absorbing_boundary"
    abc = ABC()
    abc.user_keys = gm.get_vector(root + ":boundaries")
    if not abc.user_keys:
        return abc
    if len(abc.user_keys) > 3:
        raise PreloopError("ABC::buildInparam || Parameter absorbing_boundary:boundaries || "
                           "cannot contain more than three entities.")
    if len(set(abc.user_keys)) != len(abc.user_keys):
        raise PreloopError("ABC::buildInparam || Parameter absorbing_boundary:boundaries || "
                           "cannot contain duplicated entities.")
    for k in abc.user_keys:
        if k not in ("RIGHT", "BOTTOM", "TOP"):
            raise PreloopError("ABC::buildInparam || Parameter absorbing_boundary:boundaries || "
                               "contains an invalid entity: " + k)
    abc.clayton = gm.get(root + ":enable_Clayton_Enquist", bool)
    root += ":Kosloff_Kosloff"
    abc.sponge = gm.get(root + ":enable", bool)
    if not abc.clayton and not abc.sponge:
        raise PreloopError("ABC::buildInparam || Both Clayton-Enquist and Kosloff-Kosloff are disabled.")
    rel = []
    if abc.sponge:
        rel = gm.get_vector(root + ":relative_spans", float)
        if len(rel) != len(abc.user_keys):
            raise PreloopError("ABC::buildInparam || The number of Kosloff_Kosloff::relative_spans || "
                               "does not match the number of boundaries.")
        if min(rel) < .01 or max(rel) > .25:
            raise PreloopError("ABC::buildInparam || Kosloff_Kosloff:relative_spans must range "
                               "between 0.01 and 0.25.")
        abc.expr_solid = gm.get(root + ":gamma_expr_solid")
        abc.expr_fluid = gm.get(root + ":gamma_expr_fluid")
    for i, k in enumerate(abc.user_keys):
        present, outer, span = mesh.boundary_info_abc(k)
        if present:
            abc.keys.append(k)
            if abc.sponge:
                abc.outer_span[k] = (outer, rel[i] * span)
    if abc.sponge:
        abc.t0 = mesh.global_variables["minimum_period"]
    return abc


# ------------------------------------------------------------------- Nr field ---
def _nr_field(mesh: ExodusMesh, inp: Inparam, geo) -> np.ndarray:
    """NrField::buildInparam and getNrAtPoints at the mesh nodes: CONSTANT, ANALYTICAL (the
    depth-dependent default of NrFieldAnalytical.cpp), STRUCTURED (NrFieldStructured.cpp) or
    POINTWISE (NrFieldPointwise.cpp, inverse-distance average of the 4 nearest control points)."""
    from .models3d import Model3DError, StructuredGrid, _read_nc
    gm = inp.nr
    kind = gm.get_options("type_Nr", {"CONSTANT": "CONSTANT", "ANALYTICAL": "ANALYTICAL",
                                      "POINTWISE": "POINTWISE", "STRUCTURED": "STRUCTURED"})
    xy = mesh.coords
    n = mesh.num_nodes
    if kind == "CONSTANT":
        return np.full(n, gm.get_bounded("constant", 1, None, int), np.int64)
    if kind == "ANALYTICAL":
        code = "depth-dependent (AxiSEM3D default)"
        if gm.get("analytical:code_ID") != code:
            raise PreloopError("NrFieldAnalytical::NrFieldAnalytical || Inconsistent code ID's: || in "
                               "inparam.nr.yaml:       %s ||in NrFieldAnalytical.cpp: %s"
                               % (gm.get("analytical:code_ID"), code))
        root = "analytical:depth_dependent_AxiSEM3D_default"
        dep = np.array(gm.get_vector(root + ":control_depths", float))
        nrs = np.array(gm.get_vector(root + ":Nr_at_control_depths", float))
        if len(dep) != len(nrs):
            raise PreloopError("NrFieldAnalytical::NrFieldAnalytical || Depths and Nr's do not pair up.")
        if len(dep) < 2:
            raise PreloopError("NrFieldAnalytical::NrFieldAnalytical || Insufficient control depths, at "
                               "least 2.")
        if np.any(np.diff(dep) <= 0):
            raise PreloopError("NrFieldAnalytical::NrFieldAnalytical || Depths must be ascendingly sorted.")
        depth = geo.outer_radius - (xy[:, 1] if geo.cartesian else np.hypot(xy[:, 0], xy[:, 1]))
        tol = (dep[-1] - dep[0]) * EPS
        if np.any(depth < dep[0] - tol) or np.any(depth > dep[-1] + tol):
            raise PreloopError("NrFieldAnalytical::getNrAtPoints || Target depth is out of range.")
        i1 = np.searchsorted(dep, depth, side="right")
        i1 = np.where(i1 == 0, 1, np.where(i1 == len(dep), len(dep) - 1, i1))
        f1 = (depth - dep[i1 - 1]) / (dep[i1] - dep[i1 - 1])
        return cround(nrs[i1 - 1] * (1. - f1) + nrs[i1] * f1).astype(np.int64)
    if kind == "STRUCTURED":
        fname = inp.path(gm.get("structured:nc_data_file"))
        out_val = gm.get("structured:value_out_of_range", int)
        names = ("structured_s", "structured_z") if geo.cartesian else ("structured_r", "structured_t")
        try:
            grid = StructuredGrid(fname, list(names), [("structured_Nr", 1.)], [0, 1])
        except Model3DError as ex:
            raise PreloopError(str(ex))
        grid.data = cround(grid.data)                     # StructuredGrid<2, int>
        if geo.cartesian:
            crd = xy
        else:
            r, t = sz2rtheta(xy[:, 0], xy[:, 1])
            crd = np.stack([r, t], axis=1)
        v, ok, _ = grid.compute(crd)
        return np.where(ok, cround(v[:, 0]), out_val).astype(np.int64)
    # POINTWISE
    fname = inp.path(gm.get("pointwise:nc_data_file"))
    factor = gm.get("pointwise:multip_factor", float)
    try:
        nc = _read_nc(fname)
        sz = np.asarray(nc["pointwise_sz"], np.float64).reshape(-1, 2)
        nrc = np.asarray(nc["pointwise_Nr"], np.float64).reshape(-1)
    except (KeyError, Model3DError) as ex:
        raise PreloopError("NrFieldPointwise::NrFieldPointwise || %s: %s" % (fname, ex))
    from scipy.spatial import cKDTree
    tree = cKDTree(sz)
    k = min(4, len(sz))
    dist, idx = tree.query(xy, k=k)
    dist, idx = dist.reshape(n, k), idx.reshape(n, k)
    tol = mesh.global_variables["dist_tolerance"]
    out = np.empty(n, np.int64)
    for i in range(n):
        exact = np.nonzero(dist[i] < tol)[0]
        if len(exact):
            v = nrc[idx[i, exact[0]]]
        else:
            w = 1. / dist[i]
            v = cround(np.sum(nrc[idx[i]] * w) / np.sum(w))
        out[i] = int(cround(v * factor))
    return out


def nodal_nr(mesh: ExodusMesh, inp: Inparam, lucky: bool, geo=None) -> np.ndarray:
    """Nr at the mesh nodes (NrField::buildInparam, ExodusMesh::formNrAtNodes)."""
    nr = _nr_field(mesh, inp, geo)
    if nr.min() < 1:
        raise PreloopError("ExodusMesh::formNrAtNodes || Nr must be positive.")
    if inp.nr.get("bound_Nr_by_inplane", bool):
        conn, xy = mesh.connectivity, mesh.coords
        edges = np.zeros(mesh.num_quads)
        for a in range(4):
            b = (a + 1) % 4
            edges += np.hypot(*(xy[conn[:, a]] - xy[conn[:, b]]).T)
        tot = np.zeros(mesh.num_nodes)
        cnt = np.zeros(mesh.num_nodes)
        for a in range(4):
            np.add.at(tot, conn[:, a], edges)
            np.add.at(cnt, conn[:, a], 1.)
        ave = tot / np.maximum(cnt * 4 * 4, 1.)
        circ = 2. * np.pi * xy[:, 0]
        upper = np.maximum(cround(circ / np.where(ave > 0, ave, 1.)), 1).astype(np.int64)
        upper = np.where(xy[:, 0] < mesh.global_variables["dist_tolerance"], 5, upper)
        nr = np.minimum(nr, upper)
    if lucky:
        nr = np.array([next_lucky(int(n)) for n in nr], np.int64)
    return nr


def gll_shape(axial: np.ndarray) -> np.ndarray:
    """spectrals::interpolateGLL: (nq, 4, 25) bilinear shape functions at the element points."""
    t = tables()
    out = np.zeros((len(axial), 4, 25))
    for ax in (0, 1):
        xi = np.repeat(t["pGLJ"] if ax else t["pGLL"], 5)
        eta = np.tile(t["pGLL"], 5)
        lsf = np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta),
                        (1 - xi) * (1 + eta)]) / 4.
        out[np.asarray(axial) == ax] = lsf
    return out


# ------------------------------------------------------------------ the build ---
@dataclass
class StationGroup:
    """One station group of inparam.output.yaml after location (StationOutput::release)."""
    name: str
    keys: List[str]
    channels: List[str]
    frame: str
    interval: int
    tmin: float
    tmax: float
    fmt: str
    buffer_size: int
    first: int                                  # index of the group's first station in the model
    theta: np.ndarray = None
    baz: np.ndarray = None
    phi: np.ndarray = None


@dataclass
class Simulation:
    """What the preloop hands to the time loop."""
    model: Model
    nsteps: int
    t0: float
    dt: float
    groups: List[StationGroup]
    mesh: ExodusMesh
    cartesian: bool
    info: dict
    element_groups: List["ElementGroup"] = field(default_factory=list)


def _read_stf(gm, root, name, dt, path=None):
    """STF::buildInparam (core/source/elem_src/stf/STF.cpp:19-70): GaussianSTF, or a table
    from StreamSTF (two ascii columns, '#' comments) or NetCDF_STF (two variables)."""
    cls = gm.get(root + ":class_name")
    if cls in ("StreamSTF", "NetCDF_STF"):
        pad = gm.get(root + ":padding")
        padding, left, right = 0, 0., 0.
        if pad == "FIRST_LAST":
            padding = 1
        elif pad != "NONE":
            padding = 1
            left, right = gm.get(root + ":padding:[0]", float), gm.get(root + ":padding:[1]", float)
        if cls == "StreamSTF":
            fname = path(gm.get(root + ":ascii_data_file"))
            t, v = [], []
            with open(fname) as f:
                for line in f:
                    w = line.split()
                    if not w or w[0].startswith("#"):
                        continue
                    if len(w) != 2:
                        raise PreloopError("StreamSTF::StreamSTF || Input file for STF must contain two "
                                           "columns. || Ascii file: " + fname)
                    t.append(float(w[0]))
                    v.append(float(w[1]))
            where = "StreamSTF::StreamSTF"
        else:
            from .models3d import _read_nc
            fname = path(gm.get(root + ":nc_data_file"))
            nc = _read_nc(fname)
            t = list(np.asarray(nc[gm.get(root + ":nc_var_times")], np.float64).ravel())
            v = list(np.asarray(nc[gm.get(root + ":nc_var_data")], np.float64).ravel())
            where = "NetCDF_STF::NetCDF_STF"
        # NetCDF_STF.cpp:43-70 checks the count, then the order, then the lengths
        if len(t) < 2:
            raise PreloopError(where + " || Insufficient time points, at least 2. || File: " + fname)
        if np.any(np.diff(t) <= 0):
            raise PreloopError(where + " || Time points are not ascendingly sorted. || File: " + fname)
        if len(t) != len(v):
            raise PreloopError(where + " || Times and values have different lengths. || NetCDF file: " + fname)
        if pad == "FIRST_LAST":
            left, right = v[0], v[-1]
        return STF(table=(np.array(t), np.array(v)), padding=padding, left=left, right=right,
                   pad_first=int(cls == "NetCDF_STF"))
    if cls != "GaussianSTF":
        raise PreloopError("STF::buildInparam || Unknown class of source-time function. || Source name: "
                           "%s || STF class name: %s" % (name, cls))
    hdur = gm.get_bounded(root + ":half_duration", 0.)
    hdur = max(hdur, dt * 5.)                     # dt * 5 as the minimum
    decay = gm.get_bounded(root + ":decay_factor", 0.)
    shift = gm.get(root + ":time_shift", float)
    order = gm.get_options(root + ":use_derivative_integral",
                           {"ERF": -1, "GAUSSIAN": 0, "FIRST_DERIVATIVE": 1, "RICKER": 2})
    return STF(half_duration=hdur, decay_factor=decay, time_shift=shift, derivative_order=order)


class _Quads:
    """Per-quad geometry, boundaries and material in arrays over all quads."""

    def __init__(self, mesh: ExodusMesh, inp: Inparam, geo: Geodesy, abc: ABC, lucky: bool):
        self.mesh = mesh
        nq = mesh.num_quads
        conn = mesh.connectivity
        self.nodal = mesh.coords[conn].reshape(nq, 8)
        self.nodal_xy = self.nodal.reshape(nq, 4, 2)
        self.axial = np.array([mesh.left_side(q) >= 0 for q in range(nq)], np.uint8)
        self.fluid = mesh.is_fluid.astype(bool)
        self.sides = {"LEFT": [mesh.left_side(q) for q in range(nq)],
                      "RIGHT": [mesh.right_side(q) for q in range(nq)],
                      "BOTTOM": [mesh.bottom_side(q) for q in range(nq)],
                      "TOP": [mesh.top_side(q) for q in range(nq)],
                      "SOLID_FLUID": [mesh.side("solid_fluid_boundary", q) for q in range(nq)]}
        # mapping: operands and point coordinates
        self.geom = np.zeros((nq, 6, 25))
        self.sz = np.zeros((nq, 2, 25))
        for gt, mp in MAPPING.items():
            sel = np.nonzero(mesh.geometry_type == gt)[0]
            if len(sel):
                try:
                    g, s = geometry_batch(self.nodal[sel], self.axial[sel], mp)
                except RuntimeError:
                    raise PreloopError("Quad::Quad || Error identifying curved outer edge "
                                       "(element_type %d)." % gt)
                self.geom[sel], self.sz[sel] = g, s
        unknown = set(np.unique(mesh.geometry_type).tolist()) - set(MAPPING)
        if unknown:
            raise PreloopError("Quad::Quad || Unknown element_type %s." % sorted(unknown))
        # Jacobian at the points, recovered from the operands (exact inverse of the stored form)
        a, b, c, d = self.geom[:, 0], self.geom[:, 1], self.geom[:, 2], self.geom[:, 3]
        det = 1. / (a * d - b * c)
        self.J = np.stack([a * det, -b * det, -c * det, d * det], axis=-1).reshape(nq, 25, 2, 2)
        # point Nr: nodal Nr interpolated to the points and rounded (Quad::Quad)
        nnr = nodal_nr(mesh, inp, lucky, geo)
        shp = gll_shape(self.axial)
        self.pnr = cround(np.einsum("qk,qkp->qp", nnr[conn].astype(np.float64), shp)).astype(np.int64)
        if lucky:
            self.pnr = np.vectorize(next_lucky)(self.pnr)
        self._material(mesh, geo, shp)

    def _material(self, mesh, geo, shp):
        """Material::Material: the radial profile at the nodes, then at the points."""
        rc = mesh.radial_coords
        tol = mesh.global_variables["dist_tolerance"]
        xy = self.nodal.reshape(-1, 4, 2)
        r = xy[:, :, 1] if geo.cartesian else np.hypot(xy[:, :, 0], xy[:, :, 1])
        center = r.mean(axis=1)
        i1 = np.searchsorted(rc, center, side="right")
        i1 = np.where(i1 == 0, 1, np.where(i1 == len(rc), len(rc) - 1, i1))
        i0 = i1 - 1
        r0 = rc[i0] - tol
        r1 = rc[i1] + tol
        nodal = {}
        for name, vals in mesh.radial_variables.items():
            v0, v1 = vals[i0], vals[i1]
            nodal[name] = ((v1 - v0) / (r1 - r0))[:, None] * (r - r0[:, None]) + v0[:, None]
        vs_key = "VS" if "VS" in nodal else "VSV"
        fluid_mat = np.max(nodal[vs_key], axis=1) < DEPS
        if "VSH" in nodal:
            fluid_mat |= np.max(nodal["VSH"], axis=1) < DEPS
        if np.any(fluid_mat != self.fluid):
            q = int(np.nonzero(fluid_mat != self.fluid)[0][0])
            raise PreloopError("Material::getMass || Incompatible solid/fluid flags. || Element %d" % q)
        tiso = "VPV" in nodal
        iso_e = np.ones(len(center), bool)
        if tiso:
            nrm = lambda v: np.sqrt(np.sum(v * v, axis=1))     # noqa: E731
            iso_e = ((nrm(nodal["VPV"] - nodal["VPH"]) < nrm(nodal["VPV"]) * DEPS) &
                     (nrm(nodal["VSV"] - nodal["VSH"]) < nrm(nodal["VSV"]) * DEPS) &
                     (nrm(nodal["ETA"] - 1.) < 2. * DEPS))
        self.iso = iso_e
        self.tiso = tiso
        self.node_vals = nodal                       # the 4 nodal values of every property
        self.shp = shp
        self.gll_keys = {}                           # per quad, the keys a 3-D model has set
        pt = {k: np.einsum("qk,qkp->qp", v, shp) for k, v in nodal.items()}
        if tiso:
            pt.setdefault("VP", pt["VPV"].copy())
            pt.setdefault("VS", pt["VSV"].copy())
        self.prop = pt
        # getPointwiseNodal: the 1-D values the REF1D / REF_PERTURB kinds refer to
        self.prop1d = {k: v.copy() for k, v in pt.items()}
        # per quad, the properties that vary in phi: {q: {key: [25 arrays of nr_p values]}}
        self.p3 = {}
        rho = pt["RHO"]
        if tiso:
            vp_iso, vs_iso = pt["VPV"], pt["VSV"]
            self.vmax = np.where(iso_e[:, None], vp_iso, np.maximum(pt["VPV"], pt["VPH"]))
            self.vp_c = np.where(iso_e[:, None], vp_iso, pt["VPV"])
            self.vs_c = np.where(iso_e[:, None], vs_iso, pt["VSV"])
        else:
            self.vmax = pt["VP"]
            self.vp_c, self.vs_c = pt["VP"], pt["VS"]
        self.rho = rho

    def refresh_derived(self):
        """rho, the velocities used by boundaries and dt, and vmax from the current 1-D values."""
        P = self.prop
        self.rho = P["RHO"]
        if self.tiso:
            iso = self.iso[:, None]
            self.vmax = np.where(iso, P["VP"], np.maximum(P["VPV"], P["VPH"]))
            self.vp_c = np.where(iso, P["VP"], P["VPV"])
            self.vs_c = np.where(iso, P["VS"], P["VSV"])
        else:
            self.vmax, self.vp_c, self.vs_c = P["VP"], P["VP"], P["VS"]

    def abc_rho_vp_vs(self, q):
        """Material::getPointwiseRhoVpVs (Material.cpp:249-305): rho, vp, vs per point (25
        arrays of 1 or nr_p values) for Clayton and sponge conditions. TI elements use the
        Voigt averages of kappa and mu; with nodal-only properties (NodalPhysicalProperty
        arithmetic on the 4 nodes) they are formed on the nodes and then interpolated."""
        rho = self.pointwise(q, "RHO")
        if self.fluid[q]:
            return rho, self.pointwise(q, "VP"), [np.zeros(1)] * 25
        if self.iso[q]:
            return rho, self.pointwise(q, "VP"), self.pointwise(q, "VS")

        def voigt(r, vph, vpv, vsv, vsh, eta):
            A, C, Lm, N = r * vph ** 2, r * vpv ** 2, r * vsv ** 2, r * vsh ** 2
            F = eta * (A - Lm * 2.)
            kp = (A * 4. + C + F * 4. - N * 4.) / 9.
            mu = (A + C - F * 2. + Lm * 6. + N * 5.) / 15.
            return np.sqrt((kp + mu * (4. / 3.)) / r), np.sqrt(mu / r)

        keys = ("RHO", "VPH", "VPV", "VSV", "VSH", "ETA")
        if not (self.gll_keys.get(q, set()) & set(keys)):
            vp_n, vs_n = voigt(*(self.node_vals[k][q] for k in keys))
            vp, vs = vp_n @ self.shp[q], vs_n @ self.shp[q]
            return rho, [vp[p:p + 1] for p in range(25)], [vs[p:p + 1] for p in range(25)]
        pw = [self.pointwise(q, k) for k in keys]
        out = [voigt(*np.broadcast_arrays(*(x[p] for x in pw))) for p in range(25)]
        return rho, [o[0] for o in out], [o[1] for o in out]

    def vmax_slices(self, q):
        """Material::getMaxVelocity: the largest velocity of each slice of a 3-D quad."""
        nr_e = int(self.pnr[q].max())
        if self.fluid[q] or self.iso[q]:
            return np.max(self.elemental(q, "VP", nr_e), axis=1)
        return np.maximum(np.max(self.elemental(q, "VPV", nr_e), axis=1),
                          np.max(self.elemental(q, "VPH", nr_e), axis=1))

    def vmax_3d(self, q):
        """Material::getMaxVelocity over all slices of a quad with 3-D properties."""
        nr_e = int(self.pnr[q].max())
        if self.fluid[q] or self.iso[q]:
            return float(np.max(self.elemental(q, "VP", nr_e)))
        return float(max(np.max(self.elemental(q, "VPV", nr_e)), np.max(self.elemental(q, "VPH", nr_e))))

    # ---------------- 3-D properties (Material::addProperty3D, PhysicalProperty) ----------------
    def pointwise(self, q, key):
        """PhysicalProperty::getPointwise: 25 arrays (1 value, or nr_p values on phi slices)."""
        d = self.p3.get(q, {})
        if key in d:
            return d[key]
        return [self.prop[key][q, p:p + 1] for p in range(25)]

    def set_pointwise(self, q, key, arrs):
        """PhysicalProperty::setGLL with tryReduceTo1D."""
        from .models3d import try_reduce_1d
        self.gll_keys.setdefault(q, set()).add(key)
        if try_reduce_1d(arrs):
            self.prop[key][q, :] = [a[0] for a in arrs]
            self.p3.get(q, {}).pop(key, None)
        else:
            self.p3.setdefault(q, {})[key] = [np.asarray(a, dtype=np.float64) for a in arrs]

    def elemental(self, q, key, nr_e):
        """PhysicalProperty::getElemental: (1, 25) or (nr_e, 25) by linInterpPhi per point."""
        from .models3d import lin_interp_phi
        d = self.p3.get(q, {})
        if key not in d:
            return self.prop[key][q][None, :]
        return np.stack([lin_interp_phi(a, nr_e) for a in d[key]], axis=1)

    def is3d(self, q):
        return bool(self.p3.get(q))

    def _ensure_tiso_keys(self):
        for k, src in (("VPV", "VP"), ("VPH", "VP"), ("VSV", "VS"), ("VSH", "VS")):
            if k not in self.prop:
                self.prop[k] = self.prop[src].copy()
                self.prop1d[k] = self.prop1d[src].copy()
        if "ETA" not in self.prop:
            self.prop["ETA"] = np.ones_like(self.prop["RHO"])
            self.prop1d["ETA"] = np.ones_like(self.prop["RHO"])
        self.tiso = True

    def _evolve_iso_tiso(self, q):
        """Material::evolveISO_TISO: VPV = VPH = VP, VSV = VSH = VS, ETA = 1."""
        self._ensure_tiso_keys()
        for k, src in (("VPV", "VP"), ("VPH", "VP"), ("VSV", "VS"), ("VSH", "VS")):
            self.prop1d[k][q] = self.prop1d[src][q]
            self.prop[k][q] = self.prop[src][q]
            if k not in self.node_vals:
                self.node_vals[k] = self.node_vals[src].copy()
            self.node_vals[k][q] = self.node_vals[src][q]
            d = self.p3.get(q, {})
            if src in d:
                d[k] = [a.copy() for a in d[src]]
            if src in self.gll_keys.get(q, set()):
                self.gll_keys[q].add(k)
        self.prop["ETA"][q] = 1.
        self.prop1d["ETA"][q] = 1.
        if "ETA" not in self.node_vals:
            self.node_vals["ETA"] = np.ones_like(self.node_vals["RHO"])
        self.node_vals["ETA"][q] = 1.
        self.iso[q] = False

    def apply_model(self, md, geo, und=None):
        """Volumetric3D::applyTo + Material::addProperty3D for every quad in the model's scope
        (on the undulated geometry when the model asks for it)."""
        for q in range(len(self.axial)):
            uq = und.pointwise(q) if und is not None and q in und.und else None
            res = md.properties(self.nodal_xy[q], self.sz[q], self.pnr[q], geo, uq)
            if res is None:
                continue
            ok, vals = res
            for j, (key, _, _, ref) in enumerate(md.props):
                keys = [key]
                if self.fluid[q]:
                    if key not in ("RHO", "VP"):
                        raise PreloopError("Material::getProperty || Unacceptable property key: %s||Rheology "
                                           "type: FLUID || Model name: %s" % (key, md.name))
                elif not self.iso[q] and key in ("VP", "VS"):
                    keys = [key + "V", key + "H"]
                elif self.iso[q] and key in ("VPV", "VPH", "VSV", "VSH", "ETA"):
                    self._evolve_iso_tiso(q)
                if key in ("QMU", "QKAPPA") and key not in self.prop:
                    raise PreloopError("Material::getProperty || Unacceptable property key: %s (the mesh "
                                       "has no attenuation) || Model name: %s" % (key, md.name))
                for k in keys:
                    cur = self.pointwise(q, k)
                    nod = self.prop1d[k][q]
                    new = []
                    for p in range(25):
                        v = vals[p][:, j]
                        if ref == "ABS":
                            x = v.copy()
                        elif ref == "REF1D":
                            x = (v + 1.) * nod[p]
                        elif ref == "REF3D":
                            x = (v + 1.) * cur[p]
                        else:
                            x = (v + 1.) * (cur[p] - nod[p]) + nod[p]
                        c = np.broadcast_to(cur[p], x.shape)
                        new.append(np.where(ok[p], x, c))
                    self.set_pointwise(q, k, new)

    def finished3d(self):
        """Material::finished3D: a TISO quad touched by 3-D models whose V and H velocities
        agree and ETA is 1 becomes ISO."""
        for q in list(self.p3):
            if self.fluid[q] or self.iso[q]:
                continue
            nr_e = int(self.pnr[q].max())
            g = {k: self.elemental(q, k, nr_e) for k in ("VPV", "VPH", "VSV", "VSH", "ETA")}
            n = lambda x: float(np.linalg.norm(x))          # noqa: E731
            b = lambda x, y: np.broadcast_arrays(x, y)        # noqa: E731
            vpv, vph = b(g["VPV"], g["VPH"])
            vsv, vsh = b(g["VSV"], g["VSH"])
            if (n(vpv - vph) < n(vpv) * DEPS and n(vsv - vsh) < n(vsv) * DEPS and
                    n(g["ETA"] - 1.) < n(g["ETA"]) * DEPS):
                self.iso[q] = True
                self.prop["VP"][q] = self.prop["VPV"][q]
                self.prop["VS"][q] = self.prop["VSV"][q]
                d = self.p3.get(q, {})
                if "VPV" in d:
                    d["VP"] = d["VPV"]
                if "VSV" in d:
                    d["VS"] = d["VSV"]

    def normals(self, q, edge):
        """Quad::computeNormal: (points, (5, 2) normals) of one edge."""
        t = tables()
        ax = bool(self.axial[q])
        out = np.zeros((5, 2))
        pts = EDGE_IPNT[edge]
        for ip, p in enumerate(pts):
            J = self.J[q, p]
            if edge == 0:
                n = np.array([J[1, 0], -J[0, 0]])
            elif edge == 1:
                n = np.array([J[1, 1], -J[0, 1]])
            elif edge == 2:
                n = np.array([-J[1, 0], J[0, 0]])
            else:
                n = np.array([-J[1, 1], J[0, 1]])
            ipol, jpol = p // 5, p % 5
            if ax:
                if edge % 2 != 0:
                    raise PreloopError("Quad::computeNormal || Impossible.")
                n = n * t["wGLJ"][ipol]
            else:
                n = n * t["wGLL"][ipol if edge % 2 == 0 else jpol]
            s = self.sz[q, 0, p]
            if ax:
                n = n * (J[0, 0] if ipol == 0 else s / (1. + t["pGLJ"][ipol]))
            else:
                n = n * s
            out[ip] = n
        return list(pts), out


# ------------------------------------------------------------- undulation ---
class _Undulation:
    """Undulation (preloop/se_model/quad/physical/Undulation.cpp) of the quads that geometric
    3-D models touch: the radial (spherical) or vertical (Cartesian) displacement dZ of each
    (point, slice), its gradient in (R, T, Z), and what follows from it: the particle
    relabelling transformation, the Jacobian on the mass, 3-D normals and the slice-wise
    coordinates for dt."""

    def __init__(self, quads, cartesian):
        self.q = quads
        self.cartesian = cartesian
        self.und = {}            # quad -> 25 arrays (1 value, or nr_p values on phi slices)
        self._rtz = {}

    def add(self, q, arrs):
        """PhysicalProperty::addGLL: add per point (1-D + per-slice broadcast), then
        tryReduceTo1D."""
        from .models3d import try_reduce_1d
        cur = self.und.get(q)
        out = []
        for p in range(25):
            a = np.asarray(arrs[p], dtype=np.float64)
            if cur is not None:
                c = cur[p]
                n = max(len(a), len(c))
                a = np.broadcast_to(c, (n,)) + np.broadcast_to(a, (n,))
            out.append(np.array(a, dtype=np.float64))
        if try_reduce_1d(out):
            out = [a[:1].copy() for a in out]
        self.und[q] = out
        self._rtz.pop(q, None)

    def pointwise(self, q):
        return self.und[q]

    def elemental(self, q):
        """PhysicalProperty::getElemental: [max nr of the arrays, 25] by linInterpPhi."""
        from .models3d import lin_interp_phi
        a = self.und[q]
        nr = max(len(x) for x in a)
        return np.stack([lin_interp_phi(x, nr) for x in a], axis=1)

    def is3d(self, q):
        return q in self.und and max(len(x) for x in self.und[q]) > 1

    def rtz(self, q):
        """Undulation::finished3D: [nr, 3, 25] = (dZ/dR, dZ/dT, dZ/dZ) on the element's
        slices: the gradient (computeGrad3) of dZ's Fourier series, back on the slices and,
        on a spherical mesh, from (s, z) to (R, Z) with each point's theta."""
        if q in self._rtz:
            return self._rtz[q]
        from .solver import spectral_tables
        t = spectral_tables()
        gll, glj = t["gGLL"].reshape(5, 5), t["gGLJ"].reshape(5, 5)      # [k, i] = l_k'(x_i)
        dz = self.elemental(q)                                           # [nr, 25]
        nr = len(dz)
        c = np.fft.rfft(dz, axis=0) / nr                                 # [nu, 25]
        nu = c.shape[0]
        P = c.reshape(nu, 5, 5)
        ax = bool(self.q.axial[q])
        gx = glj if ax else gll
        X = np.einsum("ki,akj->aij", gx, P)
        Y = np.einsum("kj,aik->aij", gll, P)
        sx, se, zx, ze = (self.q.geom[q, k].reshape(5, 5) for k in range(4))
        inv_s = self.q.geom[q, 4].reshape(5, 5)
        al = np.arange(nu)[:, None, None]
        A = 1j * al * P
        g = np.zeros((nu, 3, 5, 5), np.complex128)
        g[:, 0] = X * ze + Y * zx
        g[:, 2] = X * se + Y * sx
        g[:, 1] = A * inv_s
        if ax:
            axv = np.einsum("k,akj->aj", gx[:, 0], A)
            ayv = np.einsum("kj,ak->aj", gll, A[:, 0, :])
            g[:, 1, 0, :] = axv * ze[0] + ayv * zx[0]
        d = np.fft.irfft(g.reshape(nu, 3, 25) * nr, n=nr, axis=0) if nr > 1 else g.reshape(1, 3, 25).real.copy()
        if not self.cartesian:
            th = sz2rtheta(self.q.sz[q, 0], self.q.sz[q, 1])[1]
            ct, st = np.cos(th), np.sin(th)
            ds, dzz = d[:, 0].copy(), d[:, 2].copy()
            d[:, 0] = ds * ct - dzz * st
            d[:, 2] = dzz * ct + ds * st
        self._rtz[q] = d
        return d

    def _j0(self, q, p, dz, j3):
        if self.cartesian:
            return np.ones_like(j3)
        Z = math.hypot(self.q.sz[q, 0, p], self.q.sz[q, 1, p])
        return 1. + dz / Z if Z > DEPS else j3

    def mass_jacobian(self, q):
        """Undulation::getMassJacobian: J0^2 J3 per point (1 or nr_p values)."""
        from .models3d import lin_interp_phi
        d = self.rtz(q)
        out = []
        for p in range(25):
            dz = self.und[q][p]
            j3 = 1. + lin_interp_phi(d[:, 2, p], len(dz))
            j0 = self._j0(q, p, dz, j3)
            J = j0 ** 2 * j3
            if J.min() < DEPS:
                raise PreloopError("Undulation::getMassJacobian || Negative Jacobian or distorted element "
                                   "occurred.")
            out.append(J)
        return out

    def prt(self, q):
        """Undulation::createPRT: [5, nr, 25] = X0 = 1/J0, X1 = -J1/(J0 J3), X2 = -J2/(J0 J3),
        X3 = 1/J3 and |J| = J0^2 J3 on the element's slices."""
        d = self.rtz(q)
        dz = self.elemental(q)
        j1, j2, j3 = d[:, 0], d[:, 1], 1. + d[:, 2]
        if self.cartesian:
            j0 = np.ones_like(j3)
        else:
            Z = np.broadcast_to(np.hypot(self.q.sz[q, 0], self.q.sz[q, 1]), j3.shape)
            j0 = np.where(Z > DEPS, 1. + dz / np.where(Z > DEPS, Z, 1.), j3)
        xj = j0 ** 2 * j3
        if xj.min() < DEPS:
            raise PreloopError("Undulation::createPRT || Negative Jacobian or distorted element occurred.")
        return np.stack([1. / j0, -j1 / (j0 * j3), -j2 / (j0 * j3), 1. / j3, xj])

    def normal3d(self, q, n1d, p):
        """Undulation::computeNormal3D: the (s, phi, z) normal [nr_p, 3] of an edge point."""
        from .models3d import lin_interp_phi
        if q not in self.und:
            return np.array([[n1d[0], 0., n1d[1]]])
        d = self.rtz(q)
        dz = self.und[q][p]
        n = len(dz)
        j1, j2 = lin_interp_phi(d[:, 0, p], n), lin_interp_phi(d[:, 1, p], n)
        j3 = 1. + lin_interp_phi(d[:, 2, p], n)
        j0 = self._j0(q, p, dz, j3)
        k0, k1, k2, k3 = j3 * j0, -j1 * j0, -j2 * j0, j0 * j0
        nR, nZ = n1d[0], n1d[1]
        if not self.cartesian:
            th = float(sz2rtheta(self.q.sz[q, 0, p], self.q.sz[q, 1, p])[1])
            st, ct = math.sin(th), math.cos(th)
            nR, nZ = n1d[0] * ct - n1d[1] * st, n1d[1] * ct + n1d[0] * st
        out = np.stack([k1 * nZ + k0 * nR, k2 * nZ, k3 * nZ], axis=1)
        if not self.cartesian:
            r = out.copy()
            out[:, 0] = r[:, 0] * ct + r[:, 2] * st
            out[:, 2] = r[:, 2] * ct - r[:, 0] * st
        return out

    def slices_sz(self, q):
        """Quad::computeDt: the point coordinates on each slice of dZ."""
        dz = self.elemental(q)
        out = []
        for k in range(len(dz)):
            sz = self.q.sz[q].copy()
            if self.cartesian:
                sz[1] += dz[k]
            else:
                th = sz2rtheta(self.q.sz[q, 0], self.q.sz[q, 1])[1]
                sz[0] += dz[k] * np.sin(th)
                sz[1] += dz[k] * np.cos(th)
            out.append(sz)
        return out

    def total(self, models, spz, geo):
        """SE_Model::getTotalUndulation at one (s, phi, z)."""
        return float(sum(md.at(np.asarray(spz, np.float64)[None, :], geo)[0][0] for md in models))

    def to_reference(self, models, spz, geo, tol):
        """SE_Model::undulatedToReference: bisection on the reference radius (or z) whose
        undulated position is the given one."""
        if not models:
            return spz
        spz = np.array(spz, dtype=np.float64)
        if self.cartesian:
            st = ct = 0.
            und_r = spz[2]
        else:
            th = float(sz2rtheta(spz[0], spz[2])[1])
            st, ct = math.sin(th), math.cos(th)
            und_r = math.hypot(spz[0], spz[2])

        def put(R, x):
            if self.cartesian:
                x[2] = R
            else:
                x[0], x[2] = R * st, R * ct

        ref = spz.copy()
        if und_r < geo.inner_radius:
            put(geo.inner_radius, ref)
        if und_r > geo.outer_radius:
            put(geo.outer_radius, ref)
        current = ref[2] if self.cartesian else math.hypot(ref[0], ref[2])
        upper, lower = geo.outer_radius, geo.inner_radius
        for _ in range(101):
            diff = self.total(models, ref, geo) + current - und_r
            if abs(diff) < tol:
                return ref
            if diff > 0.:
                upper = current
            else:
                lower = current
            current = .5 * (lower + upper)
            put(current, ref)
        raise PreloopError("SE_Model::undulatedToReference || Failed to find reference radius.")


def _gll_numbering(conn: np.ndarray) -> np.ndarray:
    """Global GLL point of every (quad, point), from the mesh topology: vertices by node,
    edge points by (sorted node pair, position from the lower node), the rest per quad."""
    nq = len(conn)
    keys = {}
    out = np.zeros((nq, 25), np.int64)
    edge_nodes = ((0, 1), (1, 2), (2, 3), (3, 0))
    where = {}
    for e, pts in enumerate(EDGE_IPNT):
        for k, p in enumerate(pts[1:4]):
            where[p] = (e, k + 1)
    for q in range(nq):
        c = conn[q]
        for p in range(25):
            if p in NODE_IPNT:
                key = ("v", int(c[NODE_IPNT.index(p)]))
            elif p in where:
                e, k = where[p]
                na, nb = int(c[edge_nodes[e][0]]), int(c[edge_nodes[e][1]])
                key = ("e", na, nb, k) if na < nb else ("e", nb, na, 4 - k)
            else:
                key = ("i", q, p)
            g = keys.get(key)
            if g is None:
                g = len(keys)
                keys[key] = g
            out[q, p] = g
    return out


def build(input_dir: str, max_steps: Optional[int] = None, skip_unsupported_channels: bool = False
          ) -> Simulation:
    """Run the preloop on one input directory. skip_unsupported_channels: drop station channels
    this engine does not record (strain, curl, ...) instead of raising; a group left without
    channels is dropped, and info["skipped_channels"] names them."""
    inp = Inparam(input_dir)
    mesh = ExodusMesh(inp.path(inp.model.get("model1D:exodus_mesh")))
    geo = Geodesy(mesh, inp)
    abc = build_abc(mesh, inp)
    lucky = inp.advanced.get("develop:fftw_lucky_numbers", bool) \
        if inp.advanced.contains("develop:fftw_lucky_numbers") else True
    quads = _Quads(mesh, inp, geo, abc, lucky)
    nq = mesh.num_quads
    # ---- 3-D models (Model3D::buildInparam, SE_Model: applyTo, finishing3D / finished3D)
    # geometric models (Geometric3D::applyTo) add undulation on the reference geometry;
    # volumetric models may read the undulated one; ocean-load models act on the surface
    und = _Undulation(quads, geo.cartesian)
    geo_models, ocean_models = [], []
    try:
        models = build_models(inp, geo.cartesian)
        for md in models:
            if md.kind == "volumetric":
                quads.apply_model(md, geo, und)
            elif md.kind == "geometric":
                geo_models.append(md)
                for q in range(nq):
                    arrs = md.undulation(quads.nodal_xy[q], quads.sz[q], quads.pnr[q], geo)
                    if arrs is not None:
                        und.add(q, arrs)
            else:
                ocean_models.append(md)
    except Model3DError as ex:
        raise PreloopError(str(ex))
    quads.finished3d()
    quads.refresh_derived()
    q3d = np.array([quads.is3d(q) for q in range(nq)], bool)
    has_und = np.array([q in und.und for q in range(nq)], bool)
    und3d = np.array([und.is3d(q) for q in range(nq)], bool)
    tol = mesh.global_variables["dist_tolerance"]

    # ---- time step (SE_Model::computeDt, main.cpp:431-470)
    courant = inp.source.get_bounded("time_axis:Courant_number", 0.0)
    dts = np.empty(nq)
    for q in range(nq):
        f = 1.
        if quads.sides["SOLID_FLUID"][q] != -1:
            f = .9
        if abc.clayton and any(quads.sides[k][q] != -1 for k in abc.keys):
            f = .5
        if has_und[q]:
            # slice by slice on the undulated coordinates (Quad::computeDt)
            vs = quads.vmax_slices(q) if q3d[q] else np.array([float(np.max(quads.vmax[q]))])
            szs = und.slices_sz(q)
            n = max(len(vs), len(szs))
            dts[q] = min(quad_dt(szs[0 if len(szs) == 1 else k], vs[0 if len(vs) == 1 else k])
                         for k in range(n)) * f * courant
            continue
        vmax = quads.vmax_3d(q) if q3d[q] else float(np.max(quads.vmax[q]))
        dts[q] = quad_dt(quads.sz[q], vmax) * f * courant
    dt_mesh = round_dt(float(dts.min()))
    enforced = inp.source.get("time_axis:enforced_dt")
    dt = dt_mesh if enforced == "NONE" or float(enforced) < DEPS else float(enforced)

    # ---- attenuation (main.cpp:482-499, AttBuilder)
    att = inp.model.get_options("attenuation", {"NONE": -1, "FULL": 0, "CG4": 1})
    sls = None
    if att >= 0 and mesh.has_attenuation:
        gv = mesh.global_variables
        n = int(gv["nr_lin_solids"])
        sls = {"w": np.array([gv["attenuation_w_%d" % i] for i in range(n)]),
               "y": np.array([gv["attenuation_y_%d" % i] for i in range(n)]),
               "fmin": gv["attenuation_f_min"], "fmax": gv["attenuation_f_max"],
               "fref": gv["attenuation_f_ref"]}
        fmesh = 1. / gv["minimum_period"]
        if fmesh < sls["fmin"] or fmesh > sls["fmax"]:
            raise PreloopError("AttBuilder::AttBuilder || Mesh frequency lies out of attenuation band.")

    # ---- GLL points
    gll = _gll_numbering(mesh.connectivity)
    ngll = int(gll.max()) + 1
    coords = np.zeros((ngll, 2))
    coords[gll.ravel(), 0] = quads.sz[:, 0, :].ravel()
    coords[gll.ravel(), 1] = quads.sz[:, 1, :].ravel()
    dev = np.abs(coords[gll, 0] - quads.sz[:, 0, :]) + np.abs(coords[gll, 1] - quads.sz[:, 1, :])
    if dev.max() > tol:
        raise PreloopError("LocalMesh::buildElementGLL || Non-conforming mesh: GLL points of "
                           "neighbouring elements differ by %g." % dev.max())
    pnr = np.zeros(ngll, np.int64)
    np.maximum.at(pnr, gll.ravel(), quads.pnr.ravel())
    solid_q = np.nonzero(~quads.fluid)[0]
    fluid_q = np.nonzero(quads.fluid)[0]
    sp_used = np.unique(gll[solid_q].ravel()) if len(solid_q) else np.zeros(0, np.int64)
    fp_used = np.unique(gll[fluid_q].ravel()) if len(fluid_q) else np.zeros(0, np.int64)
    sid = -np.ones(ngll, np.int64)
    fid = -np.ones(ngll, np.int64)
    sid[sp_used] = np.arange(len(sp_used))
    fid[fp_used] = np.arange(len(fp_used))
    ifact = quads.geom[:, 5, :]
    qm3 = q3d | has_und                         # quads whose masses go point by point
    s1d, f1d = solid_q[~qm3[solid_q]], fluid_q[~qm3[fluid_q]]
    smass = np.zeros(len(sp_used))
    np.add.at(smass, sid[gll[s1d]].ravel(), (quads.rho[s1d] * ifact[s1d]).ravel())
    fmass = np.zeros(len(fp_used))
    if len(f1d):
        kappa = quads.rho[f1d] * quads.vp_c[f1d] ** 2
        np.add.at(fmass, fid[gll[f1d]].ravel(), (ifact[f1d] / kappa).ravel())
    # quads with 3-D properties add per-slice masses (Mass3D where a point's mass varies)
    smass3, fmass3 = {}, {}
    for q in np.nonzero(qm3)[0]:
        rho = quads.pointwise(q, "RHO")
        vp = quads.pointwise(q, "VP") if quads.fluid[q] else None
        jac = und.mass_jacobian(q) if has_und[q] else None
        for p in range(25):
            if quads.fluid[q]:
                mval = ifact[q, p] / (np.broadcast_arrays(rho[p], vp[p])[0] * vp[p] ** 2)
                tgt, idx = fmass3, int(fid[gll[q, p]])
            else:
                mval = rho[p] * ifact[q, p]
                tgt, idx = smass3, int(sid[gll[q, p]])
            if jac is not None:
                mval = mval * jac[p]
            prev = tgt.get(idx)
            tgt[idx] = mval.copy() if prev is None else prev + mval
    # per-point contributions constant in phi are 1-D masses after all
    for tgt, one in ((smass3, smass), (fmass3, fmass)):
        for idx in list(tgt):
            v = np.atleast_1d(tgt[idx])
            if len(v) == 1 or np.linalg.norm(v - v[0]) <= np.linalg.norm(v) * DEPS:
                one[idx] += v[0]
                del tgt[idx]

    # ---- boundaries of the points (Quad::setupGLL, GLLPoint::release)
    axial_pt = np.zeros(ngll, bool)
    surface_pt = np.zeros(ngll, bool)
    normal = np.zeros((ngll, 2))
    cl_s, cl_f, cl3_s, cl3_f = [], [], [], []
    ocean_pts = {}                                # point -> [summed top normal [n][3], sum rho depth]
    normal3 = {}                                  # solid-fluid points whose normal varies with phi
    gamma_sum = np.zeros(ngll)
    gamma_cnt = np.zeros(ngll, np.int64)
    gamma3 = {}                                   # points whose gamma varies in phi
    for q in range(nq):
        if quads.axial[q]:
            for p in EDGE_IPNT[quads.sides["LEFT"][q]]:
                axial_pt[gll[q, p]] = True
        if quads.sides["TOP"][q] != -1:
            for p in EDGE_IPNT[quads.sides["TOP"][q]]:
                surface_pt[gll[q, p]] = True
            if ocean_models and not quads.fluid[q]:
                _ocean_on_quad(q, quads, und, ocean_models, geo, gll, ocean_pts)
        if quads.sides["SOLID_FLUID"][q] != -1:
            pts, nsf = quads.normals(q, quads.sides["SOLID_FLUID"][q])
            sign = .5 if quads.fluid[q] else -.5
            for p, n in zip(pts, nsf):
                if has_und[q]:
                    n3 = und.normal3d(q, n, p)
                    if len(n3) > 1 and np.linalg.norm(n3 - n3[0]) > np.linalg.norm(n3) * DEPS:
                        # varies with phi: SolidFluidCoupling3D at this point
                        g = int(gll[q, p])
                        cur = normal3.get(g)
                        normal3[g] = sign * n3 if cur is None else cur + sign * n3
                        continue
                    n = np.array([n3[0, 0], n3[0, 2]])
                normal[gll[q, p]] += sign * n
        if abc.clayton or abc.sponge:
            a_rho, a_vp, a_vs = quads.abc_rho_vp_vs(q)
        if abc.clayton:
            for key in abc.keys:
                edge = quads.sides[key][q]
                if edge == -1:
                    continue
                pts, nab = quads.normals(q, edge)
                for p, n in zip(pts, nab):
                    g = gll[q, p]
                    n3 = None
                    if has_und[q]:
                        n3 = und.normal3d(q, n, p)
                        if len(n3) == 1 or np.linalg.norm(n3 - n3[0]) <= np.linalg.norm(n3) * DEPS:
                            n, n3 = np.array([n3[0, 0], n3[0, 2]]), None
                    area = float(np.hypot(n[0], n[1]))
                    if area <= 0. and n3 is None:
                        continue
                    rvp = a_rho[p] * a_vp[p]
                    rvs = np.broadcast_arrays(a_rho[p], a_vs[p])[0] * a_vs[p]
                    if n3 is not None:
                        # ClaytonSolid3D / ClaytonFluid3D with the undulated normal of each slice
                        nrp = int(pnr[g])
                        n3 = np.broadcast_to(n3, (nrp, 3)) if len(n3) == 1 else n3
                        ar = np.linalg.norm(n3, axis=1)
                        ent = (int(fid[g] if quads.fluid[q] else sid[g]), np.broadcast_to(rvp, (nrp,)).copy(),
                               np.broadcast_to(rvs, (nrp,)).copy(), ar.copy(), n3 / ar[:, None])
                        (cl3_f if quads.fluid[q] else cl3_s).append(ent)
                    elif len(rvp) == 1 and len(rvs) == 1:
                        # ClaytonSolid1D / ClaytonFluid1D
                        if quads.fluid[q]:
                            cl_f.append((fid[g], float(rvp[0]), area))
                        else:
                            _, th = sz2rtheta(n[0], n[1])
                            cl_s.append((sid[g], float(rvp[0]), float(rvs[0]), area, float(th)))
                    else:
                        # ClaytonSolid3D / ClaytonFluid3D: per slice of the point
                        nrp = int(pnr[g])
                        unit = np.array([n[0] / area, 0., n[1] / area])
                        ent = (int(fid[g] if quads.fluid[q] else sid[g]), np.broadcast_to(rvp, (nrp,)).copy(),
                               np.broadcast_to(rvs, (nrp,)).copy(), np.full(nrp, area), np.tile(unit, (nrp, 1)))
                        (cl3_f if quads.fluid[q] else cl3_s).append(ent)
        if abc.sponge:
            for p in range(25):
                gmax = np.zeros(1)
                dmin = 1.
                s_, z_ = quads.sz[q, 0, p], quads.sz[q, 1, p]
                for key in abc.keys:
                    outer, span = abc.outer_span[key]
                    if geo.cartesian:
                        coord = s_ if key == "RIGHT" else z_
                        r_ = z_
                    else:
                        r_, t_ = sz2rtheta(s_, z_)
                        coord = float(t_) if key == "RIGHT" else float(r_)
                    dist = (outer - coord) / span
                    if dist > dmin:
                        continue
                    dmin = dist
                    pattern = math.cos(math.pi / 2. * dist) ** 2
                    if not geo.cartesian and key == "RIGHT":
                        span = span * float(r_)
                    vp, vs, rho = np.broadcast_arrays(a_vp[p], a_vs[p], a_rho[p])
                    gmax = np.atleast_1d(abc.u0(abs(span), vp, vs, rho, bool(quads.fluid[q]))) * pattern
                if np.linalg.norm(gmax) > DEPS:
                    g = gll[q, p]
                    gamma_cnt[g] += 1
                    if len(gmax) == 1 and g not in gamma3:
                        gamma_sum[g] += gmax[0]
                    else:
                        prev = gamma3.get(g, np.zeros(1))
                        gamma3[g] = prev + gmax

    # ---- model
    m = Model(dt=dt)
    m.sp_nr = pnr[sp_used].astype(np.int32)
    m.sp_mass, m.sp_mass_nr, m.sp_mass_off = _mass_layout(smass, smass3)
    m.sp_axial = axial_pt[sp_used].astype(np.uint8)
    m.sp_coords = coords[sp_used]
    m.fp_nr = pnr[fp_used].astype(np.int32)
    m.fp_mass, m.fp_mass_nr, m.fp_mass_off = _mass_layout(fmass, fmass3)

    m.fp_axial = axial_pt[fp_used].astype(np.uint8)
    m.fp_coords = coords[fp_used]
    fsurf = surface_pt & ("TOP" not in abc.keys)
    m.fp_surface = fsurf[fp_used].astype(np.uint8)
    if ocean_pts:
        _release_ocean(m, ocean_pts, sid)
    # solid elements
    ns = len(solid_q)
    enr = np.array([int(pnr[gll[q]].max()) for q in range(nq)], np.int64)
    theta = sz2rtheta(quads.sz[:, 0, :], quads.sz[:, 1, :])[1]
    m.se_nr = enr[solid_q].astype(np.int32)
    m.se_pts = sid[gll[solid_q]].astype(np.int32)
    m.se_axial = quads.axial[solid_q]
    m.se_geom = quads.geom[solid_q]
    m.se_theta = theta[solid_q]
    rheo = np.where(quads.iso[solid_q], L.AXG_ISO, L.AXG_TISO).astype(np.int32)
    m.se_rheo = rheo
    m.se_rtz = ((rheo == L.AXG_TISO) & (not geo.cartesian)).astype(np.uint8)
    nmod = np.where(rheo == L.AXG_ISO, 2, 5)
    # elements whose moduli vary in phi (op1D_3D::regularize1D): per-slice operands
    rows = np.ones(ns, np.int64)
    for k in np.nonzero(q3d[solid_q] | und3d[solid_q])[0]:
        q = solid_q[k]
        keys = (("RHO", "VP", "VS") if rheo[k] == L.AXG_ISO else
                ("RHO", "VPV", "VPH", "VSV", "VSH", "ETA")) + (("QMU", "QKAPPA") if sls is not None else ())
        if any(kk in quads.p3.get(q, {}) for kk in keys) or und3d[q]:
            rows[k] = enr[q]
    is3 = rows > 1
    m.se_is3d = is3.astype(np.uint8)
    mat_off = np.zeros(ns, np.int64)
    if ns:
        mat_off[1:] = np.cumsum(nmod * rows * 25)[:-1]
    moduli = np.zeros(int(np.sum(nmod * rows * 25)))
    P = quads.prop
    rho_s = quads.rho[solid_q]
    if quads.tiso:
        A = rho_s * P["VPH"][solid_q] ** 2
        Cm = rho_s * P["VPV"][solid_q] ** 2
        Lm = rho_s * P["VSV"][solid_q] ** 2
        N = rho_s * P["VSH"][solid_q] ** 2
        F = P["ETA"][solid_q] * (A - 2. * Lm)
    mu = rho_s * quads.vs_c[solid_q] ** 2
    lam = rho_s * quads.vp_c[solid_q] ** 2 - 2. * mu
    npa = 4 if att == 1 else 25
    if sls is not None:
        qk, qm = P["QKAPPA"][solid_q], P["QMU"][solid_q]
        att_mod = np.zeros(ns * 2 * npa)
        wcg4 = weights_cg4(ifact[solid_q]) if att == 1 else None
    iso_sel = np.nonzero((rheo == L.AXG_ISO) & ~is3)[0]
    ti_sel = np.nonzero((rheo == L.AXG_TISO) & ~is3)[0]
    dl_all = np.zeros((ns, npa))
    dm_all = np.zeros((ns, npa))
    if len(iso_sel):
        l_, m_ = lam[iso_sel], mu[iso_sel]
        if sls is not None and att == 0:
            l_, m_, dl, dm = iso_with_attenuation(l_, m_, qk[iso_sel], qm[iso_sel], sls)
            dl_all[iso_sel], dm_all[iso_sel] = dl, dm
        elif sls is not None:
            kp = (l_ + (2. / 3.) * m_)[:, None, :]
            kp2, mu2, dl4, dm4 = cg4_correct(kp, m_[:, None, :], qk[iso_sel][:, None, :],
                                             qm[iso_sel][:, None, :], wcg4[iso_sel], sls)
            l_, m_ = (kp2 - (2. / 3.) * mu2)[:, 0], mu2[:, 0]
            dl_all[iso_sel], dm_all[iso_sel] = dl4[:, 0], dm4[:, 0]
        for k, e in enumerate(iso_sel):
            moduli[mat_off[e]:mat_off[e] + 25] = l_[k]
            moduli[mat_off[e] + 25:mat_off[e] + 50] = m_[k]
    if len(ti_sel):
        a_, c_, f_, l_, n_ = (x[ti_sel] for x in (A, Cm, F, Lm, N))
        if sls is not None and att == 0:
            a_, c_, f_, l_, n_, dl, dm = tiso_with_attenuation(a_, c_, f_, l_, n_, qk[ti_sel], qm[ti_sel], sls)
            dl_all[ti_sel], dm_all[ti_sel] = dl, dm
        elif sls is not None:
            kp = (a_ * 4. + c_ + f_ * 4. - n_ * 4.) / 9.
            mu0 = (a_ + c_ - f_ * 2. + l_ * 6. + n_ * 5.) / 15.
            kp2, mu2, dl4, dm4 = cg4_correct(kp[:, None, :], mu0[:, None, :], qk[ti_sel][:, None, :],
                                             qm[ti_sel][:, None, :], wcg4[ti_sel], sls)
            kp2, mu2 = kp2[:, 0], mu2[:, 0]
            a_ = a_ - (kp + 4. / 3. * mu0) + (kp2 + 4. / 3. * mu2)
            c_ = c_ - (kp + 4. / 3. * mu0) + (kp2 + 4. / 3. * mu2)
            f_ = f_ - (kp - 2. / 3. * mu0) + (kp2 - 2. / 3. * mu2)
            l_ = l_ - mu0 + mu2
            n_ = n_ - mu0 + mu2
            dl_all[ti_sel], dm_all[ti_sel] = dl4[:, 0], dm4[:, 0]
        for k, e in enumerate(ti_sel):
            for j, v in enumerate((a_, c_, f_, l_, n_)):
                moduli[mat_off[e] + 25 * j:mat_off[e] + 25 * (j + 1)] = v[k]
    # 3-D elements, one at a time (Material::createIsotropic / createTISO on (nr, 25) arrays)
    att3 = {}
    for k in np.nonzero(is3)[0]:
        q = solid_q[k]
        R = int(rows[k])
        E = lambda key: np.broadcast_to(quads.elemental(q, key, R), (R, 25)).astype(np.float64)  # noqa: E731
        rho = E("RHO")
        if sls is not None:
            qk3, qm3 = E("QKAPPA"), E("QMU")
        if rheo[k] == L.AXG_ISO:
            vp, vs = E("VP"), E("VS")
            mu3 = rho * vs ** 2
            lam3 = rho * vp ** 2 - 2. * mu3
            if sls is not None and att == 0:
                lam3, mu3, dl, dm = iso_with_attenuation(lam3, mu3, qk3, qm3, sls)
                att3[k] = (dl, dm)
            elif sls is not None:
                kp = lam3 + (2. / 3.) * mu3
                kp2, mu2, dl4, dm4 = cg4_correct(kp[None], mu3[None], qk3[None], qm3[None], wcg4[k:k + 1], sls)
                lam3, mu3 = (kp2 - (2. / 3.) * mu2)[0], mu2[0]
                att3[k] = (dl4[0], dm4[0])
            mods = (lam3, mu3)
        else:
            A3, C3 = rho * E("VPH") ** 2, rho * E("VPV") ** 2
            L3, N3 = rho * E("VSV") ** 2, rho * E("VSH") ** 2
            F3 = E("ETA") * (A3 - 2. * L3)
            if sls is not None and att == 0:
                A3, C3, F3, L3, N3, dl, dm = tiso_with_attenuation(A3, C3, F3, L3, N3, qk3, qm3, sls)
                att3[k] = (dl, dm)
            elif sls is not None:
                kp = (A3 * 4. + C3 + F3 * 4. - N3 * 4.) / 9.
                mu0 = (A3 + C3 - F3 * 2. + L3 * 6. + N3 * 5.) / 15.
                kp2, mu2, dl4, dm4 = cg4_correct(kp[None], mu0[None], qk3[None], qm3[None], wcg4[k:k + 1], sls)
                kp2, mu2 = kp2[0], mu2[0]
                A3 = A3 - (kp + 4. / 3. * mu0) + (kp2 + 4. / 3. * mu2)
                C3 = C3 - (kp + 4. / 3. * mu0) + (kp2 + 4. / 3. * mu2)
                F3 = F3 - (kp - 2. / 3. * mu0) + (kp2 - 2. / 3. * mu2)
                L3 = L3 - mu0 + mu2
                N3 = N3 - mu0 + mu2
                att3[k] = (dl4[0], dm4[0])
            mods = (A3, C3, F3, L3, N3)
        for j, v in enumerate(mods):
            moduli[mat_off[k] + j * R * 25:mat_off[k] + (j + 1) * R * 25] = v.ravel()
    m.se_mat_off = mat_off
    m.se_moduli = moduli
    if sls is not None and ns:
        m.se_att = np.full(ns, L.AXG_ATT_CG4 if att == 1 else L.AXG_ATT_FULL, np.int32)
        asz = 2 * rows * npa
        att_off = np.zeros(ns, np.int64)
        att_off[1:] = np.cumsum(asz)[:-1]
        att_mod = np.zeros(int(np.sum(asz)))
        for k in range(ns):
            R = int(rows[k])
            dl, dm = att3[k] if k in att3 else (dl_all[k], dm_all[k])
            att_mod[att_off[k]:att_off[k] + R * npa] = np.asarray(dl).ravel()
            att_mod[att_off[k] + R * npa:att_off[k] + 2 * R * npa] = np.asarray(dm).ravel()
        m.se_att_off = att_off
        m.se_att_moduli = att_mod
        a, b, g = att_alpha_beta_gamma(sls["w"], sls["y"], dt)
        m.nsls, m.att_alpha, m.att_beta, m.att_gamma = len(a), a, b, g
    # fluid elements: K = 1 / rho (Material::createAcoustic)
    nf = len(fluid_q)
    m.fe_nr = enr[fluid_q].astype(np.int32)
    m.fe_pts = fid[gll[fluid_q]].astype(np.int32) if nf else np.zeros((0, 25), np.int32)
    m.fe_axial = quads.axial[fluid_q]
    m.fe_geom = quads.geom[fluid_q]
    m.fe_theta = theta[fluid_q]
    frows = np.array([int(enr[q]) if "RHO" in quads.p3.get(q, {}) or und3d[q] else 1 for q in fluid_q], np.int64)
    m.fe_is3d = (frows > 1).astype(np.uint8)
    fe_off = np.zeros(nf, np.int64)
    if nf:
        fe_off[1:] = np.cumsum(frows * 25)[:-1]
    m.fe_mat_off = fe_off
    m.fe_moduli = (np.concatenate([(1. / np.broadcast_to(quads.elemental(q, "RHO", int(frows[k])),
                                                          (int(frows[k]), 25))).ravel()
                                   for k, q in enumerate(fluid_q)]) if nf else np.zeros(0))
    # solid-fluid coupling
    iface = np.intersect1d(sp_used, fp_used)
    # SolidFluidCoupling3D where the normal or the fluid mass varies with phi (GLLPoint::release)
    three = [g for g in iface if int(g) in normal3 or
             (int(fid[g]) in fmass3 and np.ptp(fmass3[int(fid[g])]) > 0)]
    if three:
        ents = []
        for g in three:
            nrp = int(pnr[g])
            n3 = np.tile([normal[g, 0], 0., normal[g, 1]], (nrp, 1))
            if int(g) in normal3:
                n3 = n3 + np.broadcast_to(normal3[int(g)], (nrp, 3))
            mf = np.broadcast_to(fmass[fid[g]] + fmass3.get(int(fid[g]), np.zeros(1)), (nrp,)).copy()
            ents.append((int(sid[g]), int(fid[g]), n3, mf))
        off = np.concatenate([[0], np.cumsum([len(e[3]) for e in ents])[:-1]]).astype(np.int64)
        nrm = np.concatenate([e[2] for e in ents])
        m.sf3 = {"solid": np.array([e[0] for e in ents], np.int32), "fluid": np.array([e[1] for e in ents], np.int32),
                 "offset": off, "normal_u": nrm, "normal_a": nrm.copy(),
                 "mass_fluid": np.concatenate([e[3] for e in ents])}
        iface = np.setdiff1d(iface, np.array(three))
    m.sf_solid = sid[iface].astype(np.int32)
    m.sf_fluid = fid[iface].astype(np.int32)
    m.sf_nsu = normal[iface, 0].copy()
    m.sf_nzu = normal[iface, 1].copy()
    m.sf_nsa = normal[iface, 0].copy()
    m.sf_nza = normal[iface, 1].copy()
    m.sf_mass_fluid = fmass[fid[iface]] if len(iface) else np.zeros(0)
    # particle relabelling (Undulation::createPRT) on every quad a geometric model touched
    for sel, attr, local in ((solid_q, "prt", None), (fluid_q, "prt_fluid", None)):
        els = [k for k, q in enumerate(sel) if has_und[q]]
        if not els:
            continue
        xs, offs, is3 = [], [], []
        o = 0
        for k in els:
            q = sel[k]
            x = und.prt(q)                                          # [5, nr, 25]
            if x.shape[1] > 1 and x.shape[1] != enr[q]:
                x = np.stack([np.stack([lin_interp_phi(x[c, :, p], int(enr[q])) for p in range(25)], axis=1)
                              for c in range(5)])
            offs.append(o)
            is3.append(1 if x.shape[1] > 1 else 0)
            xs.append(x.ravel())
            o += x.size
        d = {"element": np.array(els, np.int32), "offset": np.array(offs, np.int64),
             "is3d_prt": np.array(is3, np.uint8), "x": np.concatenate(xs)}
        if attr == "prt_fluid" and not geo.cartesian:
            d["theta"] = np.stack([m.fe_theta[k] for k in els])
        setattr(m, attr, d)
    # absorbing boundaries
    if cl_s:
        a_ = np.array(cl_s)
        m.cl_solid = {"point": a_[:, 0].astype(np.int32), "rho_vp": a_[:, 1], "rho_vs": a_[:, 2],
                      "area": a_[:, 3], "theta": a_[:, 4]}
    if cl_f:
        a_ = np.array(cl_f)
        m.cl_fluid = {"point": a_[:, 0].astype(np.int32), "rho_vp": a_[:, 1], "area": a_[:, 2]}
    for ents, attr in ((cl3_s, "cl3_solid"), (cl3_f, "cl3_fluid")):
        if ents:
            off = np.concatenate([[0], np.cumsum([len(e[1]) for e in ents])[:-1]]).astype(np.int64)
            d3 = {"point": np.array([e[0] for e in ents], np.int32), "offset": off,
                  "rho_vp": np.concatenate([e[1] for e in ents]), "area": np.concatenate([e[3] for e in ents])}
            if attr == "cl3_solid":
                d3["rho_vs"] = np.concatenate([e[2] for e in ents])
                d3["normal"] = np.concatenate([e[4] for e in ents])
            setattr(m, attr, d3)
    if abc.sponge:
        # Sponge: the average over the contributing elements (GLLPoint::release), 1-D or per slice
        for g in list(gamma3):
            gamma3[g] = np.broadcast_to(gamma3[g] + gamma_sum[g], (int(pnr[g]),)) / gamma_cnt[g]
        gam = np.where(gamma_cnt > 0, gamma_sum / np.maximum(gamma_cnt, 1), 0.)
        for used, idx, one, three in ((sp_used, sid, "sponge_solid", "sponge3d_solid"),
                                      (fp_used, fid, "sponge_fluid", "sponge3d_fluid")):
            sel = used[(gamma_cnt[used] > 0) & np.array([g not in gamma3 for g in used], bool)]
            sel3 = [g for g in used if g in gamma3]
            if len(sel):
                setattr(m, one, (idx[sel].astype(np.int32), gam[sel]))
            if sel3:
                off = np.concatenate([[0], np.cumsum([len(gamma3[g]) for g in sel3])[:-1]]).astype(np.int64)
                setattr(m, three, (idx[np.array(sel3)].astype(np.int32), off,
                                   np.concatenate([gamma3[g] for g in sel3])))

    # ---- wavefield scanning (WavefieldScanning::setup, SE_Model::initScanningOnPoints)
    scan_file = None
    rs = "wavefield_scanning"
    if inp.nr.contains(rs + ":enable_scanning") and inp.nr.get(rs + ":enable_scanning", bool):
        gm = inp.nr
        nspp = gm.get_bounded(rs + ":advanced:num_steps_per_mesh_period", 4, None, int)
        interval = max(int(cround(mesh.global_variables["minimum_period"] / nspp / dt)), 1)
        iface_g = set(np.intersect1d(sp_used, fp_used).tolist())
        if gm.get(rs + ":advanced:vertex_only", bool):
            vs_ = sorted({int(sid[gll[q, p]]) for q in solid_q for p in NODE_IPNT})
            vf_ = sorted({int(fid[gll[q, p]]) for q in fluid_q for p in NODE_IPNT
                          if int(gll[q, p]) not in iface_g})
        else:
            vs_ = list(range(len(sp_used)))
            vf_ = [int(fid[g]) for g in fp_used if int(g) not in iface_g]
        m.scanning = {"tol_fourier_h1": gm.get_bounded(rs + ":threshold_Fourier_convergence", 1e-4, 1e-1),
                      "rel_tol_h1": gm.get_bounded(rs + ":relative_amplitude_skipped", 0., 1.),
                      "abs_tol_h1": gm.get_bounded(rs + ":advanced:absolute_amplitude_skipped", 1e-14, 1e-10),
                      "max_num_peaks": gm.get_bounded(rs + ":advanced:max_num_peaks", 1, None, int),
                      "interval": interval, "solid_points": np.array(vs_, np.int32),
                      "fluid_points": np.array(vf_, np.int32)}
        scan_file = gm.get(rs + ":output_file")

    # ---- sources (Source::release) and the time axis (main.cpp:580-620)
    ctx = _Locator(mesh, quads, geo, gll, solid_q, fluid_q)
    und_ctx = (und, geo_models, tol)
    t_min0 = _release_sources(inp, m, ctx, geo, enr, solid_q, dt, und_ctx)
    t1 = inp.source.get_bounded("time_axis:record_length", 0.)
    nmax = inp.advanced.get("develop:max_num_time_steps", int) \
        if inp.advanced.contains("develop:max_num_time_steps") else 0
    if nmax <= 0:
        nmax = np.iinfo(np.int64).max
    if max_steps is not None:
        nmax = min(nmax, max_steps)
    step0 = math.floor(t_min0 / dt)
    step1 = math.ceil(t1 / dt)
    nstep = int(min(step1 - step0 + 1, nmax))
    m.t0 = step0 * dt
    skipped = [] if skip_unsupported_channels else None
    groups = _release_stations(inp, m, ctx, geo, dt, m.t0, m.t0 + (nstep - 1) * dt, nstep, enr, solid_q,
                               skipped, und_ctx)
    egroups = _release_elements(inp, quads, coords, gll, ctx, geo, dt, m.t0, m.t0 + (nstep - 1) * dt, nstep,
                                enr, mesh.global_variables["dist_tolerance"])
    m.meta = {"workload": "exodus %s (%d solid + %d fluid quads, %s)" %
              (mesh.summary()["file"], ns, nf, mesh.records.get("model", "")),
              "dt_mesh": dt_mesh}
    info = {"dt_mesh": dt_mesh, "dt": dt, "nsteps": nstep, "t0": m.t0, "t1": step1 * dt,
            "abc_keys": abc.keys, "attenuation": ["NONE", "FULL", "CG4"][att + 1] if sls is not None else "NONE",
            "nr_range": (int(pnr.min()), int(pnr.max())), "skipped_channels": skipped or [],
            "scanning_file": scan_file,
            "stability_interval": inp.advanced.get("verbose:stability_interval", int)
            if inp.advanced.contains("verbose:stability_interval") else 0}
    return Simulation(model=m, nsteps=nstep, t0=m.t0, dt=dt, groups=groups, mesh=mesh,
                      cartesian=geo.cartesian, info=info, element_groups=egroups)


def _ocean_on_quad(q, quads, und, models, geo, gll, ocean_pts):
    """OceanLoad3D::applyTo and Quad::setupGLL's ocean part for one quad with a surface
    edge: sum(rho * depth) of the models at the edge points' slices (reference geometry),
    and each point's top normal (undulated), summed over the quads that share it."""
    from .models3d import try_reduce_1d
    edge = quads.sides["TOP"][q]
    ipnts = EDGE_IPNT[edge]
    nr = [int(quads.pnr[q][p]) for p in ipnts]
    rows = []
    for p, n in zip(ipnts, nr):
        phi = np.linspace(0., 2. * np.pi / n * (n - 1), n) if n > 1 else np.zeros(1)
        rows.append(np.stack([np.full(n, quads.sz[q, 0, p]), phi, np.full(n, quads.sz[q, 1, p])], axis=1))
    spz = np.concatenate(rows, axis=0)
    tot = None
    for md in models:
        v = md.sum_rho_depth(quads.nodal_xy[q], spz, nr, geo)
        if v is None:
            continue
        tot = v if tot is None else [a + b for a, b in zip(tot, v)]
    if tot is None:
        return
    if try_reduce_1d(tot):
        tot = [a[:1] for a in tot]
    pts, n2 = quads.normals(q, edge)
    for ip, p in enumerate(pts):
        n3 = und.normal3d(q, n2[ip], p)
        g = int(gll[q, p])
        cur = ocean_pts.get(g)
        if cur is None:
            ocean_pts[g] = [n3.copy(), tot[ip]]
        else:
            k = max(len(cur[0]), len(n3))
            cur[0] = np.broadcast_to(cur[0], (k, 3)) + np.broadcast_to(n3, (k, 3))
            cur[1] = tot[ip]


def _release_ocean(m, ocean_pts, sid):
    """GLLPoint::release for solid points under an ocean (GLLPoint.cpp:55-90):
    MassOceanLoad1D where the mass, sum(rho * depth) and the top normal are all 1-D, else
    MassOceanLoad3D with the ocean mass sum(rho * depth) |n| and the unit normal per slice."""
    one, three = [], []
    for g in sorted(ocean_pts):
        i = int(sid[g])
        if i < 0:
            continue
        ntop, srd = ocean_pts[g]
        if len(ntop) > 1 and np.linalg.norm(ntop - ntop[0]) <= np.linalg.norm(ntop) * DEPS:
            ntop = ntop[:1]
        mass1d = m.sp_mass_nr is None or int(m.sp_mass_nr[i]) == 1
        nrp = int(m.sp_nr[i])
        if mass1d and len(srd) == 1 and len(ntop) == 1:
            r, t = sz2rtheta(ntop[0, 0], ntop[0, 2])
            one.append((i, float(srd[0]) * float(r), float(t)))
        else:
            area = np.linalg.norm(ntop, axis=1)
            mo = np.broadcast_to(srd, (nrp,)) * np.broadcast_to(area, (nrp,))
            unit = np.broadcast_to(ntop / area[:, None], (nrp, 3)).copy()
            three.append((i, mo, unit))
    if one:
        m.ocean_load = (np.array([x[0] for x in one], np.int32), np.array([x[1] for x in one]),
                        np.array([x[2] for x in one]))
    if three:
        off = np.concatenate([[0], np.cumsum([len(x[1]) for x in three])[:-1]]).astype(np.int64)
        m.ocean_load3d = (np.array([x[0] for x in three], np.int32), off, np.concatenate([x[1] for x in three]),
                          np.concatenate([x[2] for x in three]))


def _mass_layout(mass1d, mass3d):
    """Point masses: 1-D values plus the per-slice contributions of elements with 3-D density
    (GLLPoint::addMass); (values, per-point count, offsets), the last two None when every
    point's mass is 1-D (Mass1D) and per-point nr values where it varies (Mass3D)."""
    out, nr, off = [], np.ones(len(mass1d), np.int32), np.zeros(len(mass1d), np.int64)
    any3 = False
    o = 0
    for p in range(len(mass1d)):
        v = mass3d.get(p)
        tot = np.array([mass1d[p]]) if v is None else v + mass1d[p]
        if len(tot) > 1 and np.linalg.norm(tot - tot[0]) > np.linalg.norm(tot) * DEPS:
            any3 = True
        else:
            tot = tot[:1]
        off[p] = o
        nr[p] = len(tot)
        out.append(tot)
        o += len(tot)
    if not any3:
        return np.array([x[0] for x in out]), None, None
    return np.concatenate(out), nr, off


# --------------------------------------------------------- location in the mesh ---
class _Locator:
    """SE_Model::locateInplane and computeInplaneFactor."""

    def __init__(self, mesh, quads, geo, gll, solid_q, fluid_q):
        self.quads = quads
        self.geo = geo
        self.centers = quads.nodal.reshape(-1, 4, 2).mean(axis=1)
        self.solid_q, self.fluid_q = solid_q, fluid_q
        self.solid_index = -np.ones(mesh.num_quads, np.int64)
        self.solid_index[solid_q] = np.arange(len(solid_q))
        self.fluid_index = -np.ones(mesh.num_quads, np.int64)
        self.fluid_index[fluid_q] = np.arange(len(fluid_q))
        xy = mesh.coords
        tol = mesh.global_variables["dist_tolerance"]
        self.tol = tol
        self.range_s = (xy[:, 0].min() - tol, xy[:, 0].max() + tol)
        self.range_z = (xy[:, 1].min() - tol, xy[:, 1].max() + tol)
        r, t = sz2rtheta(xy[:, 0], xy[:, 1])
        self.range_r = (r.min() - tol, r.max() + tol)
        self.range_t = (t.min(), t.max())
        nodes = quads.nodal.reshape(-1, 4, 2)
        e = np.stack([np.hypot(*(nodes[:, a] - nodes[:, (a + 1) % 4]).T) for a in range(4)], axis=1)
        self.min_edge = e.min(axis=1)

    def _map(self, q, xi, eta):
        """Mapping::mapping and jacobian at one (xi, eta) of quad q."""
        mp = MAPPING[int(self.quads.mesh.geometry_type[q])]
        return _map_point(mp, self.quads.nodal[q], xi, eta)

    def inverse(self, q, s, z, max_iter=10, tolerance=1e-9):
        """Mapping::inverseMapping: Newton from (0, 0)."""
        xe = np.zeros(2)
        target = np.array([s, z])
        it = 0
        for it in range(max_iter):
            p, J = self._map(q, xe[0], xe[1])
            d = target - p
            if np.hypot(d[0], d[1]) < tolerance * self.min_edge[q]:
                break
            xe = xe + np.linalg.solve(J, d)
        else:
            return None
        b = 1. + tolerance * 20.
        if xe.min() > -b and xe.max() < b:
            return xe
        return None

    def locate(self, s, z, fluid):
        if not (self.range_s[0] <= s <= self.range_s[1] and self.range_z[0] <= z <= self.range_z[1]):
            return -1, None
        r, t = sz2rtheta(s, z)
        if (r < self.range_r[0] or r > self.range_r[1] or t * r < self.range_t[0] * r - self.tol or
                t * r > self.range_t[1] * r + self.tol):
            return -1, None
        cand = self.fluid_q if fluid else self.solid_q
        d = np.hypot(self.centers[cand, 0] - s, self.centers[cand, 1] - z)
        for k in np.argsort(d, kind="stable")[:30]:
            q = int(cand[k])
            xe = self.inverse(q, s, z)
            if xe is not None:
                return q, xe
        return -1, None

    def weights(self, q, xe):
        t = tables()
        wx = lagrange(t["pGLJ"] if self.quads.axial[q] else t["pGLL"], xe[0])
        we = lagrange(t["pGLL"], xe[1])
        return np.outer(wx, we).ravel()


def _map_point(mp, nodal, xi, eta):
    """One point of a mapping and its Jacobian (axg_quad_map)."""
    lib = L.lib()
    nod = np.ascontiguousarray(nodal, dtype=np.float64)
    out = np.zeros(6)
    rc = lib.axg_quad_map(int(mp), nod.ctypes.data_as(L.P_f64), float(xi), float(eta),
                          out.ctypes.data_as(L.P_f64))
    if rc != L.AXG_OK:
        raise PreloopError("Mapping::mapping || Error identifying curved outer edge.")
    return out[:2], out[2:].reshape(2, 2)


def _compute_spz(geo, crd, source_centered, xy, ellipticity, use_depth, depth_solid, enforce_axis, und_ctx=None):
    """Source::computeSPZ (preloop/source/Source.cpp:97-191). und_ctx = (undulation, geometric
    models, distance tolerance) when the location is given in the undulated geometry: a depth
    is then taken below the undulated surface, and the point is mapped back to the
    reference geometry (SE_Model::undulatedToReference)."""
    crd_in = np.array(crd, dtype=np.float64)
    spz = _compute_spz_ref(geo, crd, source_centered, xy, ellipticity, use_depth, depth_solid, enforce_axis)
    if und_ctx is None or not und_ctx[1]:
        return spz
    und, models, tol = und_ctx
    if use_depth:
        R = geo.outer_solid_radius if depth_solid else geo.outer_radius
        if geo.cartesian:
            spz[2] = R
            spz[2] = R + und.total(models, spz, geo) - crd_in[2]
        else:
            th = float(sz2rtheta(spz[0], spz[2])[1])
            spz[0], spz[2] = R * math.sin(th), R * math.cos(th)
            r = R + und.total(models, spz, geo) - crd_in[2]
            spz[0], spz[2] = r * math.sin(th), r * math.cos(th)
    return und.to_reference(models, spz, geo, tol)


def _compute_spz_ref(geo, crd, source_centered, xy, ellipticity, use_depth, depth_solid, enforce_axis):
    crd = np.array(crd, dtype=np.float64)
    if use_depth:
        R = geo.outer_solid_radius if depth_solid else geo.outer_radius
        crd[2] = R - crd[2]
    if enforce_axis:
        crd[0] = crd[1] = 0.
    elif source_centered:
        if xy:
            x, y = crd[0], crd[1]
            crd[0] = math.hypot(x, y)
            crd[1] = 0. if crd[0] < DEPS else math.atan2(y, x)
        elif not geo.cartesian:
            r, th = crd[2], crd[0]
            crd[0], crd[2] = r * math.sin(th), r * math.cos(th)
    else:
        crd = geo.llr2spz(crd[None, :], ellipticity)[0]
        if geo.cartesian:
            r, t = sz2rtheta(crd[0], crd[2])
            un = np.array([float(t) * float(r), crd[1], float(r)])
            if un[2] < un[0] * 10.:
                raise PreloopError("Source::computeSPZ || Invalid geographic location in Cartesian mesh.")
            crd = un
    return crd


def _qzsp(geo, spz, axial, source_centered, crd_in, use_depth, depth_solid, ellipticity):
    """Source::computeQzsp: rotation from the input frame to (z, s, phi)."""
    Q = np.eye(3)
    if axial:
        return Q
    if not source_centered:
        llr = np.array(crd_in, dtype=np.float64)
        if use_depth:
            R = geo.outer_solid_radius if depth_solid else geo.outer_radius
            llr[2] = R - llr[2]
        baz = float(geo.back_azimuth(llr[None, :], ellipticity)[0])
        Q[1, 1] = Q[2, 2] = math.cos(baz)
        Q[1, 2] = -math.sin(baz)
        Q[2, 1] = math.sin(baz)
    if not geo.cartesian:
        th = float(sz2rtheta(spz[0], spz[2])[1])
        Qt = np.eye(3)
        Qt[0, 0] = Qt[1, 1] = math.cos(th)
        Qt[0, 1] = -math.sin(th)
        Qt[1, 0] = math.sin(th)
        Q = Q @ Qt
    return Q


def _release_sources(inp, m, ctx, geo, enr, solid_q, dt, und_ctx=None):
    gm = inp.source
    n = gm.get("list_of_sources:[?]", int) if gm.contains("list_of_sources") and \
        gm._walk("list_of_sources") else 0
    ms, fs, ps = [], [], []
    t0 = np.inf
    north_source = inp.model.get("geodesy:lat_lon_north_pole_mesh") == "SOURCE"
    for k in range(n):
        name = gm.get("list_of_sources:{%d}" % k)
        root = "list_of_sources:[%d]:%s" % (k, name)
        rl = root + ":location"
        axial, centered, ellip = False, False, True
        crd = np.zeros(3)
        if gm.contains(rl + ":latitude_longitude"):
            if gm.get(rl + ":latitude_longitude") == "ON_AXIS":
                axial = True
            else:
                crd[0] = gm.get_bounded(rl + ":latitude_longitude:[0]", -90., 90.)
                crd[1] = gm.get_bounded(rl + ":latitude_longitude:[1]", -180., 180.)
                ellip = gm.get(rl + ":ellipticity", bool)
        elif gm.contains(rl + ":distance_azimuth"):
            if gm.get(rl + ":distance_azimuth") == "ON_AXIS":
                axial = True
            else:
                centered = True
                crd[0] = gm.get_bounded(rl + ":distance_azimuth:[0]", 0., None if geo.cartesian else math.pi)
                crd[1] = gm.get_bounded(rl + ":distance_azimuth:[1]", 0., 2. * math.pi)
        else:
            raise PreloopError("Source::buildInparam || Either location:latitude_longitude or || "
                               "location:distance_azimuth must exist. || Source name: " + name)
        if k == 0 and north_source:
            axial = True
        use_depth, depth_solid = False, False
        if gm.contains(rl + ":depth"):
            use_depth = True
            crd[2] = gm.get(rl + ":depth", float)
            depth_solid = gm.get(rl + ":depth_below_solid_surface", bool)
        elif gm.contains(rl + ":radius"):
            crd[2] = gm.get(rl + ":radius", float)
        else:
            raise PreloopError("Source::buildInparam || Either location:radius or location:depth must "
                               "exist. || Source name: " + name)
        rm = root + ":mechanism"
        mtype = gm.get_options(rm + ":type", {"MOMENT_TENSOR": "M", "FORCE_VECTOR": "F",
                                              "FLUID_PRESSURE": "P"})
        data = np.array(gm.get_vector(rm + ":data", float)) * gm.get(rm + ":unit", float)
        undulated = gm.get(rl + ":undulated_geometry", bool) if gm.contains(rl + ":undulated_geometry") else False
        spz = _compute_spz(geo, crd, centered, False, ellip, use_depth, depth_solid, axial,
                           und_ctx if undulated else None)
        q, xe = ctx.locate(spz[0], spz[2], mtype == "P")
        if q < 0:
            raise PreloopError("Source::release || Error locating source in mesh. || "
                               "Source index = %d || Source name  = %s" % (k, name))
        w = ctx.weights(q, xe)
        stf = _read_stf(gm, root + ":source_time_function", name, dt, inp.path)
        t0 = min(t0, stf.start_time())
        Q = _qzsp(geo, spz, axial, centered, crd, use_depth, depth_solid, ellip)
        nu_1 = int(enr[q]) // 2 + 1
        e = int(ctx.fluid_index[q] if mtype == "P" else ctx.solid_index[q])
        pat = _pattern(mtype, data, Q, axial, w, float(spz[1]), nu_1, bool(ctx.quads.axial[q]))
        {"M": ms, "F": fs, "P": ps}[mtype].append((e, pat, stf))
    if n == 0:
        t0 = 0.
    for lst, pre in ((ms, "ms"), (fs, "fs"), (ps, "ps")):
        if not lst:
            continue
        setattr(m, pre + "_elem", np.array([x[0] for x in lst], np.int32))
        setattr(m, pre + "_nu", np.array([x[1].shape[0] for x in lst], np.int32))
        off = np.zeros(len(lst), np.int64)
        sizes = [x[1].size for x in lst]
        off[1:] = np.cumsum(sizes)[:-1]
        setattr(m, pre + "_pat_off", off)
        setattr(m, pre + "_pattern", np.concatenate([x[1].ravel() for x in lst]))
        setattr(m, pre + "_stf", [x[2] for x in lst])
    return t0


def _pattern(mtype, data, Q, on_axis, w, phi, nu_1, axial_quad):
    """Mechanism::release (Mechanism.cpp:42-222) for fluid pressures, force vectors and moment
    tensors."""
    ephi = lambda a: np.exp(1. * a * (-1j * phi))         # noqa: E731
    if mtype == "P":
        p = data[0] * w
        nu = min(nu_1, 1) if on_axis else nu_1
        pat = np.zeros((nu, 25), np.complex128)
        if not on_axis:
            for a in range(nu):
                pat[a] = ephi(a) * p
        if axial_quad:
            pat[:, 0:5] = 0.
            pat[0, 0:5] = p[0:5]
            pat /= 2. * np.pi
        return pat
    if mtype == "F":
        f = Q @ data[:3]
        fs_, fp_, fz_ = f[1] * w, f[2] * w, f[0] * w
        nu = min(nu_1, 2) if on_axis else nu_1
        pat = np.zeros((nu, 3, 25), np.complex128)
        if not on_axis:
            for a in range(nu):
                pat[a, 0], pat[a, 1], pat[a, 2] = ephi(a) * fs_, ephi(a) * fp_, ephi(a) * fz_
        if axial_quad:
            pat[:, :, 0:5] = 0.
            pat[0, 2, 0:5] = fz_[0:5]
            if nu >= 2:
                pat[1, 0, 0:5] = (fs_[0:5] - 1j * fp_[0:5]) / 2.
                pat[1, 1, 0:5] = 1j * pat[1, 0, 0:5]
            pat /= 2. * np.pi
        return pat
    mt = np.zeros((3, 3))
    mt[0, 0], mt[1, 1], mt[2, 2] = data[0], data[1], data[2]
    mt[0, 1] = mt[1, 0] = data[3]
    mt[0, 2] = mt[2, 0] = data[4]
    mt[1, 2] = mt[2, 1] = data[5]
    mt = Q @ mt @ Q.T
    mss, mpp, mzz = mt[1, 1] * w, mt[2, 2] * w, mt[0, 0] * w
    mpz, msz, msp = mt[0, 2] * w, mt[0, 1] * w, mt[1, 2] * w
    nu = min(nu_1, 3) if on_axis else nu_1
    pat = np.zeros((nu, 6, 25), np.complex128)
    if not on_axis:
        for a in range(nu):
            for d, v in enumerate((mss, mpp, mzz, mpz, msz, msp)):
                pat[a, d] = ephi(a) * v
    if axial_quad:
        pat[:, :, 0:5] = 0.
        pat[0, 0, 0:5] = pat[0, 1, 0:5] = (mss[0:5] + mpp[0:5]) / 2.
        pat[0, 2, 0:5] = mzz[0:5]
        if nu >= 2:
            pat[1, 4, 0:5] = (msz[0:5] - 1j * mpz[0:5]) / 2.
            pat[1, 3, 0:5] = 1j * pat[1, 4, 0:5]
        if nu >= 3:
            pat[2, 0, 0:5] = (mss[0:5] - mpp[0:5] - 2. * 1j * msp[0:5]) / 4.
            pat[2, 1, 0:5] = -pat[2, 0, 0:5]
            pat[2, 5, 0:5] = 1j * pat[2, 0, 0:5]
        pat /= 2. * np.pi
    return pat


# ----------------------------------------------------------------- stations ---
# channel::solid::gChannelMap (core/output/channel.hpp:37-73): standard name, the names a user
# may give, field; kept in the map's order. Stress channels (S*) need the stress of the
# element at the station and are not recorded by this engine.
SOLID_CHANNELS = (
    ("U1", ("U1", "U"), "U"), ("U2", ("U2", "U"), "U"), ("U3", ("U3", "U"), "U"),
    ("U_NORM", ("U_NORM", "|U|"), "U"),
    ("G11", ("G11", "G"), "G"), ("G12", ("G12", "G"), "G"), ("G13", ("G13", "G"), "G"),
    ("G21", ("G21", "G"), "G"), ("G22", ("G22", "G"), "G"), ("G23", ("G23", "G"), "G"),
    ("G31", ("G31", "G"), "G"), ("G32", ("G32", "G"), "G"), ("G33", ("G33", "G"), "G"),
    ("G_I1", ("G_I1", "Gii"), "G"),
    ("E11", ("E11", "E"), "E"), ("E22", ("E22", "E"), "E"), ("E33", ("E33", "E"), "E"),
    ("E23", ("E23", "E", "E32"), "E"), ("E31", ("E31", "E", "E13"), "E"), ("E12", ("E12", "E", "E21"), "E"),
    ("E_I1", ("E_I1", "Eii"), "E"), ("E_J2", ("E_J2",), "E"),
    ("R1", ("R1", "R"), "R"), ("R2", ("R2", "R"), "R"), ("R3", ("R3", "R"), "R"),
    ("R_NORM", ("R_NORM", "|R|"), "R"),
)
UNSUPPORTED_CHANNELS = ("S11", "S22", "S33", "S23", "S32", "S31", "S13", "S12", "S21", "S", "S_I1", "Sii",
                        "S_J2")


def standard_channels(user, skipped=None):
    """channel::solid::ChannelOptions: the user's channels as standard names in the map's
    order; stress channels raise, or are listed in `skipped` when a list is given."""
    out = set()
    for uch in user:
        found = False
        for std, names, _ in SOLID_CHANNELS:
            if uch in names:
                out.add(std)
                found = True
        if not found:
            if skipped is None or uch not in UNSUPPORTED_CHANNELS:
                raise PreloopError("channel::solid::ChannelOptions::ChannelOptions || %s: %s" %
                                   ("Stress channels are not supported by this engine"
                                    if uch in UNSUPPORTED_CHANNELS else "Unknown channel for solid", uch))
            skipped.append(uch)
    return [std for std, _, _ in SOLID_CHANNELS if std in out]


def _release_stations(inp, m, ctx, geo, dt, tmin_simu, tmax_simu, nsteps, enr, solid_q, skipped=None,
                      und_ctx=None):
    gm = inp.output
    groups = []
    if not gm.contains("list_of_station_groups") or not gm._walk("list_of_station_groups"):
        _set_stations(m, [], [], [], 1)
        return groups
    n = gm.get("list_of_station_groups:[?]", int)
    st_e, st_w, st_phi = [], [], []
    names = set()
    intervals = []
    for g in range(n):
        name = gm.get("list_of_station_groups:{%d}" % g)
        if name in names:
            raise PreloopError("StationOutput::release || Station group name must be unique. || "
                               "Duplicated station group name: " + name)
        names.add(name)
        root = "list_of_station_groups:[%d]:%s" % (g, name)
        rl = root + ":locations"
        fname = gm.get(rl + ":station_file")
        h = gm.get(rl + ":horizontal_x1_x2")
        centered = {"LATITUDE_LONGITUDE": False, "DISTANCE_AZIMUTH": True, "XY_CARTESIAN": True}[h]
        xy = h == "XY_CARTESIAN"
        use_depth = gm.get_options(rl + ":vertical_x3", {"RADIUS": False, "DEPTH": True})
        ellip = gm.get(rl + ":ellipticity", bool) if not centered else False
        depth_solid = gm.get(rl + ":depth_below_solid_surface", bool) if use_depth else False
        undulated = gm.get(rl + ":undulated_geometry", bool) if gm.contains(rl + ":undulated_geometry") else False
        rw = root + ":wavefields"
        frame = gm.get_options(rw + ":coordinate_frame", {"spz": "spz", "RTZ": "RTZ", "ENZ": "ENZ",
                                                          "xyz": "xyz"})
        if gm.get_options(rw + ":medium", {"SOLID": False, "FLUID": True}):
            raise PreloopError("StationOutput::release || Fluid station groups are not supported by "
                               "this engine. || Station group name: " + name)
        chans = standard_channels(gm.get_vector(rw + ":channels"), skipped)
        if not chans:
            continue
        rt = root + ":temporal"
        sp = gm.get(rt + ":sampling_period")
        if sp == "DT":
            period = dt
        elif sp.startswith("DTx"):
            period = dt * int(sp[3:])
        else:
            period = float(sp)
        tmin, tmax = tmin_simu, tmax_simu
        if gm.get(rt + ":time_window") != "FULL":
            tmin = max(tmin_simu, gm.get(rt + ":time_window:[0]", float))
            tmax = min(tmax_simu, gm.get(rt + ":time_window:[1]", float))
        rf = root + ":file_options"
        fmt = gm.get_options(rf + ":format", {"ASCII_STATION": "ASCII_STATION",
                                              "ASCII_CHANNEL": "ASCII_CHANNEL", "NETCDF": "NETCDF"})
        bsize = gm.get_bounded(rf + ":buffer_size", 1, None, int)
        keys, crds = [], []
        with open(inp.path(fname)) as f:
            for line in f:
                words = line.split()
                if not words or words[0].startswith("#"):
                    continue
                if len(words) not in (5, 6):
                    raise PreloopError("StationOutput::release || Input file for stations must contain "
                                       "five or six columns. || Ascii file: %s || Station group name: %s"
                                       % (fname, name))
                key = words[1] + "." + words[0]
                if key in keys:
                    raise PreloopError("StationOutput::release || Station key must be unique. || "
                                       "Duplicated station key: %s || Station group name: %s" % (key, name))
                keys.append(key)
                crds.append([float(words[2]), float(words[3]), float(words[-1])])
        intv = int(period / dt)
        intv = 1 if intv == 0 else intv
        if intv < 0:
            intv = np.iinfo(np.int32).max
        nrec = sum(1 for t in range(0, nsteps, intv)
                   if tmin - dt / 2. <= tmin_simu + t * dt <= tmax + dt / 2.)
        if nrec == 0:
            raise PreloopError("StationOutput::release || No time step to record in the given time "
                               "window. ||Station group name: " + name)
        grp = StationGroup(name=name, keys=keys, channels=chans, frame=frame, interval=intv,
                           tmin=tmin - dt / 2., tmax=tmax + dt / 2., fmt=fmt, buffer_size=bsize,
                           first=len(st_e))
        th, baz, phi = [], [], []
        for key, c in zip(keys, crds):
            spz = _compute_spz(geo, c, centered, xy, ellip, use_depth, depth_solid, False,
                               und_ctx if undulated else None)
            q, xe = ctx.locate(spz[0], spz[2], False)
            if q < 0:
                raise PreloopError("StationOutput::release || Error locating station in mesh. || "
                                   "Station key: %s || Station group name: %s" % (key, name))
            st_e.append(int(ctx.solid_index[q]))
            st_w.append(ctx.weights(q, xe))
            st_phi.append(float(spz[1]))
            th.append(float(sz2rtheta(spz[0], spz[2])[1]))
            llr = geo.spz2llr(spz[None, :], True, False)
            baz.append(float(geo.back_azimuth(llr, True)[0]))
            phi.append(float(spz[1]))
        grp.theta, grp.baz, grp.phi = np.array(th), np.array(baz), np.array(phi)
        if any(c[0] in "GER" for c in chans):
            m.st_gradient = True
        intervals.append(intv)
        groups.append(grp)
    interval = int(np.gcd.reduce(intervals)) if intervals else 1
    interval = max(1, min(interval, nsteps))
    _set_stations(m, st_e, st_w, st_phi, interval)
    return groups


# ---------------------------------------------------------- element groups ---
# vicinity::constants::gEdgeIPnt (preloop/spectral/vicinity.hpp): GLL points along each edge
EDGE_IPNT = ((0, 5, 10, 15, 20), (20, 21, 22, 23, 24), (24, 19, 14, 9, 4), (4, 3, 2, 1, 0))


@dataclass
class ElementGroup:
    """One element group (ElementOutput::buildInparam, preloop/output/ElementOutput.cpp:27-143,
    and ElementOutput::release :276-400, ElementOpGroup::initialize, core/output/element-wise/
    element/ElementOpGroup.hpp:66-150)."""
    name: str
    channels: List[str]
    frame: str                      # spz or RTZ
    interval: int
    tmin: float                     # the window already widened by dt / 2
    tmax: float
    buffer_size: int
    flush: bool
    npnts: int                      # GLL points per element
    phis: np.ndarray                # azimuths (phi_list, then lat_lon_list); empty = Fourier
    tags: np.ndarray                # mesh quad index of each element
    elems: np.ndarray               # solid-element index in the model
    ipnts: np.ndarray               # [element, npnts] GLL point (ipol * 5 + jpol)
    coords: np.ndarray              # [element, npnts, 2] (s, z) of the points
    theta: np.ndarray               # [element, npnts] polar angle of the points (RTZ)
    nr: np.ndarray                  # nr of each element
    na: np.ndarray                  # element nr (Fourier) or the number of azimuths
    na_grid: np.ndarray
    elem_na: np.ndarray             # [element, 5]: tag, na, na-grid value, index in it, global index
    nrec: int = 0


def _na_grid(na, na_space):
    """ElementOpGroup::initialize (ElementOpGroup.hpp:96-118): from the largest na down, keep
    an na only when it is at least na_space below the last kept one."""
    srt = sorted(set(int(x) for x in na))
    grid = []
    if srt:
        grid.append(srt[-1])
        for v in srt[-2::-1]:
            if v <= grid[-1] - na_space:
                grid.append(v)
    return np.array(sorted(set(grid)), np.int64)


def _release_elements(inp, quads, coords, gll, ctx, geo, dt, tmin_simu, tmax_simu, nsteps, enr, dist_tol):
    """ElementOutput::release (ElementOutput.cpp:276-480) for solid groups; fluid groups and
    stress channels raise."""
    gm = inp.output
    key = "list_of_element_groups"
    if not gm.contains(key) or not gm._walk(key):
        return []
    groups, names = [], set()
    nq = len(quads.fluid)
    centers = quads.nodal_xy.mean(axis=1)                          # [quad, (s, z)]
    if geo.cartesian:
        cR, cZ = centers[:, 0], centers[:, 1]
    else:
        r, t = sz2rtheta(centers[:, 0], centers[:, 1])
        cR, cZ = t, r
    for gi in range(gm.get(key + ":[?]", int)):
        name = gm.get(key + ":{%d}" % gi)
        root = key + ":[%d]:%s" % (gi, name)
        re_ = root + ":elements"
        minR, maxR = gm.get(re_ + ":horizontal_range:[0]", float), gm.get(re_ + ":horizontal_range:[1]", float)
        minZ, maxZ = gm.get(re_ + ":vertical_range:[0]", float), gm.get(re_ + ":vertical_range:[1]", float)
        ri = root + ":inplane"
        edge_dim = gm.get_options(ri + ":edge_dimension", {"HORIZONTAL": 0, "VERTICAL": 1, "BOTH": -1})
        edge_pos = gm.get(ri + ":edge_position", float) if edge_dim >= 0 else 0.
        if gm.get(ri + ":GLL_points_one_edge") == "FULL":
            ipols = list(range(5))
        else:
            ipols = sorted(set(int(x) for x in gm.get_vector(ri + ":GLL_points_one_edge")))
        if not ipols:
            raise PreloopError("ElementOutput::buildInparam || elements:GLL_points_one_edge cannot be empty.")
        if ipols[0] < 0 or ipols[-1] > 4:
            raise PreloopError("ElementOutput::buildInparam || elements:GLL_points_one_edge must be "
                               "ranged between 0 and 4.")
        ra = root + ":azimuthal"
        phis = [gm.get_bounded(ra + ":phi_list:[%d]" % k, 0., 2. * math.pi)
                for k in range(gm.get(ra + ":phi_list:[?]", int))]
        lats, lons = [], []
        for k in range(gm.get(ra + ":lat_lon_list:[?]", int)):
            lats.append(gm.get_bounded(ra + ":lat_lon_list:[%d]:[0]" % k, -90., 90.))
            lons.append(gm.get_bounded(ra + ":lat_lon_list:[%d]:[1]" % k, -180., 180.))
        na_space = gm.get_bounded(ra + ":na_space", 1, None, int)
        rw = root + ":wavefields"
        frame = gm.get_options(rw + ":coordinate_frame", {"spz": "spz", "RTZ": "RTZ"})
        fluid = gm.get_options(rw + ":medium", {"SOLID": False, "FLUID": True})
        if fluid:
            raise PreloopError("ElementOutput::release || Fluid element groups are not supported by "
                               "this engine. || Element group name: " + name)
        chans = standard_channels(gm.get_vector(rw + ":channels"))
        rt = root + ":temporal"
        sp = gm.get(rt + ":sampling_period")
        period = dt if sp == "DT" else dt * int(sp[3:]) if sp.startswith("DTx") else float(sp)
        tmin, tmax = tmin_simu, tmax_simu
        if gm.get(rt + ":time_window") != "FULL":
            tmin = max(tmin_simu, gm.get(rt + ":time_window:[0]", float))
            tmax = min(tmax_simu, gm.get(rt + ":time_window:[1]", float))
        rf = root + ":file_options"
        bsize = gm.get_bounded(rf + ":buffer_size", 1, None, int)
        flush = gm.get(rf + ":flush", bool)
        if name in names:
            raise PreloopError("ElementOutput::release || Element group name must be unique. || "
                               "Duplicated element group name: " + name)
        names.add(name)
        # elements by the (R, Z) of their centers (theta and r in a spherical mesh)
        sel = [q for q in range(nq) if minR < cR[q] < maxR and minZ < cZ[q] < maxZ and
               bool(quads.fluid[q]) == fluid]
        use, ipnts = [], []
        if edge_dim < 0:
            uni = [i * 5 + j for i in ipols for j in ipols]
            use = sel
            ipnts = [uni] * len(sel)
        else:
            for q in sel:
                sz = quads.nodal_xy[q].T                                  # [2, 4]
                if geo.cartesian:
                    RZ = sz
                else:
                    r4, t4 = sz2rtheta(sz[0], sz[1])
                    RZ = np.stack([t4, r4])
                if edge_dim == 0 and not geo.cartesian:
                    rmean = RZ[1].mean()
                    x = RZ[0] * rmean
                    xmin, xmax = edge_pos * rmean - dist_tol, edge_pos * rmean + dist_tol
                else:
                    x = RZ[edge_dim]
                    xmin, xmax = edge_pos - dist_tol, edge_pos + dist_tol
                for ie in range(4):
                    je = 0 if ie == 3 else ie + 1
                    if xmin < x[ie] < xmax and xmin < x[je] < xmax:
                        use.append(q)
                        ipnts.append([EDGE_IPNT[ie][i] for i in ipols])
                        break
        # azimuths: phi_list, then the lat_lon_list at the surface
        if lats:
            llr = np.stack([lats, lons, np.full(len(lats), geo.outer_radius)], axis=1)
            phis = phis + list(geo.llr2spz(llr, True)[:, 1])
        intv = int(period / dt)
        intv = 1 if intv == 0 else intv
        if intv < 0:
            intv = np.iinfo(np.int32).max
        nrec = sum(1 for t in range(0, nsteps, intv)
                   if tmin - dt / 2. <= tmin_simu + t * dt <= tmax + dt / 2.)
        if nrec == 0:
            raise PreloopError("ElementOutput::release || No time step to record in the given time "
                               "window. ||Element group name: " + name)
        npnts = len(ipols) ** 2 if edge_dim < 0 else len(ipols)
        use = np.array(use, np.int64)
        ip = np.array(ipnts, np.int64).reshape(len(use), npnts)
        tags = use.astype(np.int64)
        elems = ctx.solid_index[use].astype(np.int64) if len(use) else np.zeros(0, np.int64)
        pts = gll[use[:, None], ip] if len(use) else np.zeros((0, npnts), np.int64)
        crd = coords[pts] if len(use) else np.zeros((0, npnts, 2))
        theta = sz2rtheta(crd[..., 0], crd[..., 1])[1] if len(use) else np.zeros((0, npnts))
        nr = enr[use].astype(np.int64) if len(use) else np.zeros(0, np.int64)
        na = nr.copy() if not phis else np.full(len(use), len(phis), np.int64)
        grid = _na_grid(na, na_space)
        info = np.zeros((len(use), 5), np.int64)
        count = np.zeros(len(grid), np.int64)
        for k in range(len(use)):
            gidx = int(np.searchsorted(grid, na[k]))
            info[k] = (tags[k], na[k], grid[gidx], count[gidx], count[gidx])
            count[gidx] += 1
        groups.append(ElementGroup(name=name, channels=chans, frame=frame, interval=intv, tmin=tmin - dt / 2.,
                                   tmax=tmax + dt / 2., buffer_size=bsize, flush=flush, npnts=npnts,
                                   phis=np.array(phis, np.float64), tags=tags, elems=elems, ipnts=ip,
                                   coords=crd, theta=theta, nr=nr, na=na, na_grid=grid, elem_na=info,
                                   nrec=nrec))
    return groups


def _set_stations(m, st_e, st_w, st_phi, interval):
    m.st_elem = np.array(st_e, np.int32)
    m.st_w = np.array(st_w).reshape(-1, 25)
    m.st_phi = np.array(st_phi, np.float64)
    m.st_interval = int(interval)
