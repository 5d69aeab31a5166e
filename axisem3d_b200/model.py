"""Host-side description of one sub-mesh, in the struct-of-arrays form of the C ABI.

A ``Model`` holds numpy arrays for points, elements, boundary couplings,
sources and stations, plus the time-step constants. ``Model.c_structs()``
builds the ctypes structs of include/axg.h that point into those arrays (the
arrays stay owned by the Model), so the same Model feeds the engine and the
CPU oracle.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import ctypes as C
import numpy as np

from . import _lib as L


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _i64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int64)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class STF:
    """GaussianSTF parameters (GaussianSTF.hpp:35-58), or a StreamSTF / NetCDF_STF table:
    `table` = (times, values), padding 0 (none) or 1 (left / right values), and pad_first
    for NetCDF_STF's order of tests."""
    half_duration: float = 0.0
    decay_factor: float = 0.0
    time_shift: float = 0.0
    derivative_order: int = 2
    table: Optional[tuple] = None
    padding: int = 0
    left: float = 0.0
    right: float = 0.0
    pad_first: int = 0

    def start_time(self):
        """STF::getStartTime: -2.5 half durations + shift (Gaussian) or the first time."""
        if self.table is not None:
            return float(self.table[0][0])
        return -self.half_duration * 2.5 + self.time_shift


@dataclass
class Model:
    dt: float
    t0: float = 0.0
    nsls: int = 0
    att_alpha: np.ndarray = field(default_factory=lambda: np.zeros(0))
    att_beta: np.ndarray = field(default_factory=lambda: np.zeros(0))
    att_gamma: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # solid points
    sp_nr: np.ndarray = None
    sp_mass: np.ndarray = None
    sp_mass_nr: Optional[np.ndarray] = None
    sp_mass_off: Optional[np.ndarray] = None
    sp_axial: Optional[np.ndarray] = None
    sp_coords: Optional[np.ndarray] = None        # (n, 2) s, z (not used by the engine)
    # fluid points
    fp_nr: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fp_mass: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fp_mass_nr: Optional[np.ndarray] = None
    fp_mass_off: Optional[np.ndarray] = None
    fp_axial: Optional[np.ndarray] = None
    fp_surface: Optional[np.ndarray] = None
    fp_coords: Optional[np.ndarray] = None        # (n, 2) s, z (not used by the engine)
    # solid elements
    se_nr: np.ndarray = None
    se_pts: np.ndarray = None                     # (ne, 25)
    se_axial: np.ndarray = None
    se_geom: np.ndarray = None                    # (ne, 6, 25)
    se_rheo: np.ndarray = None
    se_is3d: Optional[np.ndarray] = None
    se_mat_off: np.ndarray = None
    se_moduli: np.ndarray = None
    se_att: Optional[np.ndarray] = None
    se_att_off: Optional[np.ndarray] = None
    se_att_moduli: Optional[np.ndarray] = None
    se_part: Optional[np.ndarray] = None          # (ne,) 0 / 1 element parts (overlapped exchange)
    fe_part: Optional[np.ndarray] = None
    se_rtz: Optional[np.ndarray] = None
    se_theta: Optional[np.ndarray] = None         # (ne, 25)
    # fluid elements
    fe_nr: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fe_pts: np.ndarray = field(default_factory=lambda: np.zeros((0, 25), np.int32))
    fe_theta: Optional[np.ndarray] = None         # (n, 25) polar angle (not used by the engine)
    fe_axial: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))
    fe_geom: np.ndarray = field(default_factory=lambda: np.zeros((0, 6, 25)))
    fe_is3d: Optional[np.ndarray] = None
    fe_mat_off: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    fe_moduli: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # solid-fluid coupling
    sf_solid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    sf_fluid: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    sf_nsu: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sf_nzu: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sf_nsa: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sf_nza: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sf_mass_fluid: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # moment sources
    ms_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ms_nu: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ms_pat_off: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    ms_pattern: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex128))
    ms_stf: List[STF] = field(default_factory=list)
    ms_wave: Optional[np.ndarray] = None          # wavefield of each source (batched sources)
    # force sources
    fs_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fs_nu: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    fs_pat_off: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    fs_pattern: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex128))
    fs_stf: List[STF] = field(default_factory=list)
    fs_wave: Optional[np.ndarray] = None
    # FluidPressure sources on fluid elements: pattern [nu][25] complex per source
    ps_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ps_nu: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ps_pat_off: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    ps_pattern: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex128))
    ps_stf: List[STF] = field(default_factory=list)
    ps_wave: Optional[np.ndarray] = None
    nwave: int = 1                                # independent wavefields on this mesh
    # stations
    st_elem: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    st_w: np.ndarray = field(default_factory=lambda: np.zeros((0, 25)))
    st_phi: np.ndarray = field(default_factory=lambda: np.zeros(0))
    st_interval: int = 1
    st_gradient: bool = False                     # also record d_j u_i at the stations
    # absorbing boundaries (Clayton 1-D coefficients; sponge gamma per point)
    cl_solid: Optional[dict] = None               # point, rho_vp, rho_vs, area, theta
    cl_fluid: Optional[dict] = None               # point, rho_vp, area
    sponge_solid: Optional[tuple] = None          # (points, gamma)
    sponge_fluid: Optional[tuple] = None
    # MassOceanLoad1D on solid surface points: (points, ocean mass, normal polar angle)
    ocean_load: Optional[tuple] = None
    # MassOceanLoad3D: (points, offsets, per-slice ocean mass, per-slice unit normal [n][3])
    ocean_load3d: Optional[tuple] = None
    # 3-D absorbing boundaries: Clayton dicts with point, offset and per-slice rho_vp,
    # rho_vs, area, normal [n][3] (solid); sponges as (points, offsets, per-slice gamma)
    # wavefield scanning: dict(tol_fourier_h1, rel_tol_h1, abs_tol_h1, max_num_peaks, interval,
    # solid_points=None (all), fluid_points=None (all))
    scanning: Optional[dict] = None
    # PRT (undulated geometry): dict(element, offset, is3d_prt, x) with x per element
    # [5][nslice][25] (X0..X3, |J|) from offset
    prt: Optional[dict] = None
    # the same for fluid elements, plus theta [n][25] for the RTZ frame (None: cartesian)
    prt_fluid: Optional[dict] = None
    # SolidFluidCoupling3D: dict(solid, fluid, offset, normal_u [n][3], normal_a [n][3], mass_fluid [n])
    sf3: Optional[dict] = None
    cl3_solid: Optional[dict] = None
    cl3_fluid: Optional[dict] = None
    sponge3d_solid: Optional[tuple] = None
    sponge3d_fluid: Optional[tuple] = None
    meta: dict = field(default_factory=dict)
    meta_rho: Optional[np.ndarray] = None          # (ne, 25) density at element points (generators)

    # ------------------------------------------------------------ sizes ---
    @property
    def n_solid_elements(self):
        return 0 if self.se_nr is None else len(self.se_nr)

    @property
    def n_fluid_elements(self):
        return len(self.fe_nr)

    def solid_field_size(self):
        return int(np.sum(np.asarray(self.sp_nr) // 2 + 1)) * 3 * max(1, self.nwave)

    def fluid_field_size(self):
        return int(np.sum(np.asarray(self.fp_nr) // 2 + 1)) if len(self.fp_nr) else 0

    def updates_per_step(self):
        """GLL-point x mode updates of one stiffness evaluation: sum_e 25 nu_e."""
        u = 25 * int(np.sum(np.asarray(self.se_nr) // 2 + 1))
        if len(self.fe_nr):
            u += 25 * int(np.sum(np.asarray(self.fe_nr) // 2 + 1))
        return u

    # ---------------------------------------------------------- C structs ---
    def config(self, precision, device=0, stability_interval=0, compensated=1, plain=0, autotune=0,
               deterministic=0):
        cfg = L.axg_config()
        cfg.precision = L.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        cfg.device = device
        cfg.dt = float(self.dt)
        cfg.t0 = float(self.t0)
        cfg.nsls = int(self.nsls)
        for i in range(self.nsls):
            cfg.att_alpha[i] = float(self.att_alpha[i])
            cfg.att_beta[i] = float(self.att_beta[i])
            cfg.att_gamma[i] = float(self.att_gamma[i])
        cfg.stability_interval = stability_interval
        cfg.deterministic = int(bool(deterministic))
        cfg.compensated = compensated
        cfg.plain = int(bool(plain))
        cfg.autotune = int(bool(autotune))
        cfg.nwave = int(self.nwave)
        return cfg

    def c_structs(self):
        """ctypes structs of the model; the returned dict keeps every array alive."""
        keep = {}

        def k(name, a, conv, ctype):
            a = conv(a)
            keep[name] = a
            return L.ptr(a, ctype)

        sp = L.axg_solid_points()
        sp.count = len(self.sp_nr)
        sp.nr = k("sp_nr", self.sp_nr, _i32, C.c_int32)
        sp.mass_nr = k("sp_mass_nr", self.sp_mass_nr, _i32, C.c_int32)
        sp.mass_offset = k("sp_mass_off", self.sp_mass_off, _i64, C.c_int64)
        sp.mass = k("sp_mass", self.sp_mass, _f64, C.c_double)
        sp.axial = k("sp_axial", self.sp_axial, _u8, C.c_uint8)

        fp = L.axg_fluid_points()
        fp.count = len(self.fp_nr)
        fp.nr = k("fp_nr", self.fp_nr, _i32, C.c_int32)
        fp.mass_nr = k("fp_mass_nr", self.fp_mass_nr, _i32, C.c_int32)
        fp.mass_offset = k("fp_mass_off", self.fp_mass_off, _i64, C.c_int64)
        fp.mass = k("fp_mass", self.fp_mass, _f64, C.c_double)
        fp.axial = k("fp_axial", self.fp_axial, _u8, C.c_uint8)
        fp.surface = k("fp_surface", self.fp_surface, _u8, C.c_uint8)

        se = L.axg_solid_elements()
        se.count = self.n_solid_elements
        se.nr = k("se_nr", self.se_nr, _i32, C.c_int32)
        se.points = k("se_pts", self.se_pts, _i32, C.c_int32)
        se.axial = k("se_axial", self.se_axial, _u8, C.c_uint8)
        se.geometry = k("se_geom", self.se_geom, _f64, C.c_double)
        se.rtz = k("se_rtz", self.se_rtz, _u8, C.c_uint8)
        se.theta = k("se_theta", self.se_theta, _f64, C.c_double)
        se.rheology = k("se_rheo", self.se_rheo, _i32, C.c_int32)
        se.is3d = k("se_is3d", self.se_is3d, _u8, C.c_uint8)
        se.mat_offset = k("se_mat_off", self.se_mat_off, _i64, C.c_int64)
        se.moduli = k("se_moduli", self.se_moduli, _f64, C.c_double)
        se.attenuation = k("se_att", self.se_att, _i32, C.c_int32)
        se.att_offset = k("se_att_off", self.se_att_off, _i64, C.c_int64)
        se.att_moduli = k("se_att_moduli", self.se_att_moduli, _f64, C.c_double)

        fe = L.axg_fluid_elements()
        fe.count = self.n_fluid_elements
        fe.nr = k("fe_nr", self.fe_nr, _i32, C.c_int32)
        fe.points = k("fe_pts", self.fe_pts, _i32, C.c_int32)
        fe.axial = k("fe_axial", self.fe_axial, _u8, C.c_uint8)
        fe.geometry = k("fe_geom", self.fe_geom, _f64, C.c_double)
        fe.is3d = k("fe_is3d", self.fe_is3d, _u8, C.c_uint8)
        fe.mat_offset = k("fe_mat_off", self.fe_mat_off, _i64, C.c_int64)
        fe.moduli = k("fe_moduli", self.fe_moduli, _f64, C.c_double)

        sf = L.axg_solid_fluid()
        sf.count = len(self.sf_solid)
        sf.solid_point = k("sf_solid", self.sf_solid, _i32, C.c_int32)
        sf.fluid_point = k("sf_fluid", self.sf_fluid, _i32, C.c_int32)
        sf.ns_unassembled = k("sf_nsu", self.sf_nsu, _f64, C.c_double)
        sf.nz_unassembled = k("sf_nzu", self.sf_nzu, _f64, C.c_double)
        sf.ns_assembled = k("sf_nsa", self.sf_nsa, _f64, C.c_double)
        sf.nz_assembled = k("sf_nza", self.sf_nza, _f64, C.c_double)
        sf.mass_fluid = k("sf_mf", self.sf_mass_fluid, _f64, C.c_double)

        def sources(kind, cls, ndim):
            s = cls()
            n = len(getattr(self, kind + "_elem"))
            s.count = n
            s.element = k(kind + "_elem", getattr(self, kind + "_elem"), _i32, C.c_int32)
            s.nu = k(kind + "_nu", getattr(self, kind + "_nu"), _i32, C.c_int32)
            s.pattern_offset = k(kind + "_po", getattr(self, kind + "_pat_off"), _i64, C.c_int64)
            pat = np.ascontiguousarray(getattr(self, kind + "_pattern"), dtype=np.complex128)
            keep[kind + "_pat"] = pat
            s.pattern = pat.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))
            stfs = (L.axg_stf * max(n, 1))()
            for i, st in enumerate(getattr(self, kind + "_stf")):
                stfs[i].half_duration = st.half_duration
                stfs[i].decay_factor = st.decay_factor
                stfs[i].time_shift = st.time_shift
                stfs[i].derivative_order = st.derivative_order
            keep[kind + "_stf"] = stfs
            s.stf = C.cast(stfs, C.POINTER(L.axg_stf))
            s.wavefield = k(kind + "_wave", getattr(self, kind + "_wave"), _i32, C.c_int32)
            return s

        ms = sources("ms", L.axg_moment_sources, 6)
        fs = sources("fs", L.axg_force_sources, 3)
        ps = sources("ps", L.axg_pressure_sources, 1)

        st = L.axg_stations()
        st.count = len(self.st_elem)
        st.element = k("st_elem", self.st_elem, _i32, C.c_int32)
        st.weights = k("st_w", self.st_w, _f64, C.c_double)
        st.phi = k("st_phi", self.st_phi, _f64, C.c_double)

        def clay(name, d, solid):
            c = L.axg_clayton()
            if not d:
                c.count = 0
                return c
            c.count = len(d["point"])
            c.point = k(name + "_pt", d["point"], _i32, C.c_int32)
            c.rho_vp = k(name + "_rvp", d["rho_vp"], _f64, C.c_double)
            c.area = k(name + "_area", d["area"], _f64, C.c_double)
            if solid:
                c.rho_vs = k(name + "_rvs", d["rho_vs"], _f64, C.c_double)
                c.theta = k(name + "_th", d["theta"], _f64, C.c_double)
            return c

        def clay3(name, d, solid):
            c = L.axg_clayton3d()
            if not d:
                c.count = 0
                return c
            c.count = len(d["point"])
            c.point = k(name + "_pt", d["point"], _i32, C.c_int32)
            c.offset = k(name + "_off", d["offset"], _i64, C.c_int64)
            c.nvalues = len(d["rho_vp"])
            c.rho_vp = k(name + "_rvp", d["rho_vp"], _f64, C.c_double)
            c.area = k(name + "_area", d["area"], _f64, C.c_double)
            if solid:
                c.rho_vs = k(name + "_rvs", d["rho_vs"], _f64, C.c_double)
                c.normal = k(name + "_nrm", np.asarray(d["normal"]).ravel(), _f64, C.c_double)
            return c

        def sponge3(name, t):
            if not t:
                return (None, None, None)
            pt, off, g = _i32(t[0]), _i64(t[1]), _f64(t[2])
            keep[name + "_pt"], keep[name + "_off"], keep[name + "_g"] = pt, off, g
            return (pt, off, g)

        def scan():
            d = self.scanning
            if not d:
                return None
            c = L.axg_scanning()
            c.tol_fourier_h1, c.rel_tol_h1, c.abs_tol_h1 = d["tol_fourier_h1"], d["rel_tol_h1"], d["abs_tol_h1"]
            c.max_num_peaks, c.interval = int(d["max_num_peaks"]), int(d["interval"])
            for key, nk, pk in (("solid_points", "n_solid", "scs"), ("fluid_points", "n_fluid", "scf")):
                pts = d.get(key)
                if pts is None:
                    setattr(c, nk, -1)
                else:
                    setattr(c, nk, len(pts))
                    setattr(c, key, k(pk, pts, _i32, C.c_int32))
            return c

        def prt(d, name):
            if not d:
                return None
            e, off = _i32(d["element"]), _i64(d["offset"])
            x3 = np.ascontiguousarray(d["is3d_prt"], dtype=np.uint8)
            x = _f64(np.asarray(d["x"]).ravel())
            th = _f64(np.asarray(d["theta"]).ravel()) if d.get("theta") is not None else None
            keep[name + "_e"], keep[name + "_off"], keep[name + "_x3"], keep[name + "_x"] = e, off, x3, x
            keep[name + "_th"] = th
            return (e, off, x3, x, th)

        def ocean3():
            if not self.ocean_load3d:
                return None
            t = self.ocean_load3d
            pt, off, mo, nrm = _i32(t[0]), _i64(t[1]), _f64(t[2]), _f64(np.asarray(t[3]).ravel())
            keep["o3_pt"], keep["o3_off"], keep["o3_mo"], keep["o3_n"] = pt, off, mo, nrm
            return (pt, off, mo, nrm)

        def ocean():
            if not self.ocean_load:
                return (None, None, None)
            pt, mo, th = _i32(self.ocean_load[0]), _f64(self.ocean_load[1]), _f64(self.ocean_load[2])
            keep["oc_pt"], keep["oc_mo"], keep["oc_th"] = pt, mo, th
            return (pt, mo, th)

        def sponge(name, t):
            if not t:
                return (None, None)
            pt, g = _i32(t[0]), _f64(t[1])
            keep[name + "_pt"], keep[name + "_g"] = pt, g
            return (pt, g)

        return {"sp": sp, "fp": fp, "se": se, "fe": fe, "sf": sf, "ms": ms, "fs": fs, "ps": ps, "st": st,
                "cl_s": clay("cls", self.cl_solid, True), "cl_f": clay("clf", self.cl_fluid, False),
                "sg_s": sponge("sgs", self.sponge_solid), "sg_f": sponge("sgf", self.sponge_fluid),
                "ocean": ocean(), "scan": scan(), "ocean3": ocean3(), "prt": prt(self.prt, "prt"), "prt_f": prt(self.prt_fluid, "prtf"),
                "cl3_s": clay3("c3s", self.cl3_solid, True), "cl3_f": clay3("c3f", self.cl3_fluid, False),
                "sg3_s": sponge3("g3s", self.sponge3d_solid), "sg3_f": sponge3("g3f", self.sponge3d_fluid),
                "keep": keep}
