"""ctypes wrapper of the CPU oracle (liboracle.so) -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker of the CUDA engine; the product path never imports it.
The oracle consumes the same ``axisem3d_b200.model.Model`` as the engine.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, HERE)
import spectral  # noqa: E402


def build():
    srcs = [os.path.join(HERE, "axg_oracle.cpp"), os.path.join(HERE, "axg_operands_oracle.cpp"),
            os.path.join(HERE, "..", "include", "axg.h")]
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        from axisem3d_b200 import _lib as L
        O = C.CDLL(LIB_PATH)
        V = C.c_void_p
        sig = {
            "axo_set_spectral": (C.c_int, [L.P_f64, L.P_f64]),
            "axo_create": (V, [C.POINTER(L.axg_config)]),
            "axo_destroy": (None, [V]),
            "axo_last_error": (C.c_char_p, [V]),
            "axo_set_solid_points": (C.c_int, [V, C.POINTER(L.axg_solid_points)]),
            "axo_set_fluid_points": (C.c_int, [V, C.POINTER(L.axg_fluid_points)]),
            "axo_set_solid_elements": (C.c_int, [V, C.POINTER(L.axg_solid_elements)]),
            "axo_set_fluid_elements": (C.c_int, [V, C.POINTER(L.axg_fluid_elements)]),
            "axo_set_solid_fluid": (C.c_int, [V, C.POINTER(L.axg_solid_fluid)]),
            "axo_set_moment_sources": (C.c_int, [V, C.POINTER(L.axg_moment_sources)]),
            "axo_set_force_sources": (C.c_int, [V, C.POINTER(L.axg_force_sources)]),
            "axo_set_pressure_sources": (C.c_int, [V, C.POINTER(L.axg_pressure_sources)]),
            "axo_set_solid_fluid3d": (C.c_int, [V, C.c_int, L.P_i32, L.P_i32, L.P_i64, L.P_f64, L.P_f64, L.P_f64]),
            "axo_set_stf_table": (C.c_int, [V, C.c_int, C.c_int, C.c_int, L.P_f64, L.P_f64, C.c_int, C.c_double,
                                            C.c_double, C.c_int]),
            "axo_set_stations": (C.c_int, [V, C.POINTER(L.axg_stations), C.c_int]),
            "axo_apply_sources": (C.c_int, [V, C.c_int]),
            "axo_set_clayton": (C.c_int, [V, C.c_int, C.POINTER(L.axg_clayton)]),
            "axo_set_sponge": (C.c_int, [V, C.c_int, C.c_int, L.P_i32, L.P_f64]),
            "axo_set_ocean_load": (C.c_int, [V, C.c_int, L.P_i32, L.P_f64, L.P_f64]),
            "axo_set_clayton3d": (C.c_int, [V, C.c_int, C.POINTER(L.axg_clayton3d)]),
            "axo_set_scanning": (C.c_int, [V, C.POINTER(L.axg_scanning)]),
            "axo_set_prt": (C.c_int, [V, C.c_int, L.P_i32, L.P_i64, L.P_u8, L.P_f64]),
            "axo_set_prt_fluid": (C.c_int, [V, C.c_int, L.P_i32, L.P_i64, L.P_u8, L.P_f64, L.P_f64]),
            "axo_set_ocean_load3d": (C.c_int, [V, C.c_int, L.P_i32, L.P_i64, L.P_f64, L.P_f64]),
            "axo_scanning_nr": (C.c_int, [V, L.P_i32, L.P_i32]),
            "axo_set_sponge3d": (C.c_int, [V, C.c_int, C.c_int, L.P_i32, L.P_i64, L.P_f64]),
            "axo_compute_stiffness": (C.c_int, [V, C.c_int]),
            "axo_compute_stiffness_part": (C.c_int, [V, C.c_int, C.c_int]),
            "axo_set_element_parts": (C.c_int, [V, C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
            "axo_bc_before": (C.c_int, [V]),
            "axo_bc_after": (C.c_int, [V]),
            "axo_stiff_to_accel": (C.c_int, [V]),
            "axo_newmark": (C.c_int, [V]),
            "axo_record": (C.c_int, [V, C.c_int]),
            "axo_run": (C.c_int, [V, C.c_int, C.c_int]),
            "axo_get_field": (C.c_int, [V, C.c_int, C.c_int, L.P_f64]),
            "axo_set_field": (C.c_int, [V, C.c_int, C.c_int, L.P_f64]),
            "axo_field_size": (C.c_int64, [V, C.c_int]),
            "axo_get_seismograms": (C.c_int, [V, L.P_f64]),
            "axo_reset_attenuation": (C.c_int, [V]),
            "axo_current_step": (C.c_int, [V]),
            "axo_quad_geometry_batch": (C.c_int, [C.c_int, C.c_int, L.P_f64, L.P_u8, L.P_f64, L.P_f64, L.P_f64]),
            "axo_quad_dt": (C.c_int, [L.P_f64, C.c_double, L.P_f64]),
            "axo_att_alpha_beta_gamma": (C.c_int, [C.c_int, L.P_f64, L.P_f64, C.c_double, L.P_f64, L.P_f64,
                                                   L.P_f64]),
            "axo_att_moduli": (C.c_int, [C.c_int, L.P_f64, L.P_f64, C.c_double, C.c_double, C.c_double, C.c_int,
                                         L.P_f64, L.P_f64, L.P_f64, L.P_f64, L.P_f64, L.P_f64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(O, name)
            f.restype = res
            f.argtypes = args
        t = spectral.tables()
        gll = np.ascontiguousarray(t["gGLL"])
        glj = np.ascontiguousarray(t["gGLJ"])
        O.axo_set_spectral(gll.ctypes.data_as(L.P_f64), glj.ctypes.data_as(L.P_f64))
        _lib = O
    return _lib


class OracleOperands:
    """The oracle's own restatement of the preloop numbers (axg_operands_oracle.cpp: the
    mappings, Quad::computeIntegralFactor / createGradient, Quad::computeDt and AttBuilder),
    with the GLL / GLJ tables of spectral.py. It has the methods of
    ``axisem3d_b200.meshgen.EngineOperands``, so ``meshgen.operands(OracleOperands())`` builds
    a workload without the engine's library: the CPU baselines use it, and the tests compare
    the two builders."""

    MAP_LINEAR, MAP_SPHERICAL = 0, 1

    def tables(self):
        return spectral.tables()

    def geometry_batch(self, nodal, axial, mapping=0):
        from axisem3d_b200 import _lib as L
        ne = len(axial)
        nodal = np.ascontiguousarray(nodal, dtype=np.float64).reshape(ne, 8)
        ax = np.ascontiguousarray(axial, dtype=np.uint8)
        t = spectral.tables()
        tab = np.ascontiguousarray(np.concatenate([t["pGLL"], t["pGLJ"], t["wGLL"], t["wGLJ"]]))
        g = np.zeros((ne, 6, 25))
        sz = np.zeros((ne, 2, 25))
        rc = lib().axo_quad_geometry_batch(ne, int(mapping), nodal.ctypes.data_as(L.P_f64),
                                           ax.ctypes.data_as(L.P_u8), tab.ctypes.data_as(L.P_f64),
                                           g.ctypes.data_as(L.P_f64), sz.ctypes.data_as(L.P_f64))
        if rc != 0:
            raise RuntimeError("oracle: MappingSpherical::MappingSpherical || Error identifying curved outer edge.")
        return g, sz

    def quad_dt(self, sz, vmax):
        from axisem3d_b200 import _lib as L
        s = np.ascontiguousarray(sz, dtype=np.float64).reshape(50)
        dt = C.c_double()
        lib().axo_quad_dt(s.ctypes.data_as(L.P_f64), float(vmax), C.byref(dt))
        return dt.value

    def att_alpha_beta_gamma(self, w, y, dt):
        from axisem3d_b200 import _lib as L
        w = np.ascontiguousarray(w, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        a, b, g = np.zeros(len(w)), np.zeros(len(w)), np.zeros(len(w))
        lib().axo_att_alpha_beta_gamma(len(w), w.ctypes.data_as(L.P_f64), y.ctypes.data_as(L.P_f64), float(dt),
                                       a.ctypes.data_as(L.P_f64), b.ctypes.data_as(L.P_f64),
                                       g.ctypes.data_as(L.P_f64))
        return a, b, g

    def att_moduli(self, w, y, fmin, fmax, fref, qkappa, qmu, kp, mu):
        from axisem3d_b200 import _lib as L
        w = np.ascontiguousarray(w, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        qk = np.ascontiguousarray(np.broadcast_to(qkappa, np.shape(kp)), dtype=np.float64).ravel()
        qm = np.ascontiguousarray(np.broadcast_to(qmu, np.shape(kp)), dtype=np.float64).ravel()
        kp2 = np.array(kp, dtype=np.float64).ravel().copy()
        mu2 = np.array(mu, dtype=np.float64).ravel().copy()
        dk, dm = np.zeros_like(kp2), np.zeros_like(kp2)
        P = L.P_f64
        lib().axo_att_moduli(len(w), w.ctypes.data_as(P), y.ctypes.data_as(P), float(fmin), float(fmax),
                             float(fref), len(kp2), qk.ctypes.data_as(P), qm.ctypes.data_as(P),
                             kp2.ctypes.data_as(P), mu2.ctypes.data_as(P), dk.ctypes.data_as(P),
                             dm.ctypes.data_as(P))
        shp = np.shape(kp)
        return kp2.reshape(shp), mu2.reshape(shp), dk.reshape(shp), dm.reshape(shp)


class Oracle:
    """CPU restatement of the time loop; precision 'fp64' (default) or 'fp32'."""

    def __init__(self, model, precision="fp64", threads=1):
        from axisem3d_b200 import _lib as L
        self.O = lib()
        self.L = L
        self.model = model
        self.threads = threads
        cfg = model.config("fp32" if precision == "fp32" else "fp64")
        self.h = self.O.axo_create(C.byref(cfg))
        if not self.h:
            raise RuntimeError("oracle: spectral tables not set")
        s = model.c_structs()
        self._keep = s
        self._chk(self.O.axo_set_solid_points(self.h, C.byref(s["sp"])))
        self._chk(self.O.axo_set_fluid_points(self.h, C.byref(s["fp"])))
        self._chk(self.O.axo_set_solid_elements(self.h, C.byref(s["se"])))
        self._chk(self.O.axo_set_fluid_elements(self.h, C.byref(s["fe"])))
        self._chk(self.O.axo_set_solid_fluid(self.h, C.byref(s["sf"])))
        self._chk(self.O.axo_set_moment_sources(self.h, C.byref(s["ms"])))
        self._chk(self.O.axo_set_force_sources(self.h, C.byref(s["fs"])))
        if s["ps"].count:
            self._chk(self.O.axo_set_pressure_sources(self.h, C.byref(s["ps"])))
        if getattr(model, "sf3", None):
            d3 = model.sf3
            self._sf3 = [np.ascontiguousarray(d3[k], dt) for k, dt in (
                ("solid", np.int32), ("fluid", np.int32), ("offset", np.int64), ("normal_u", np.float64),
                ("normal_a", np.float64), ("mass_fluid", np.float64))]
            a = self._sf3
            self._chk(self.O.axo_set_solid_fluid3d(self.h, len(a[0]), a[0].ctypes.data_as(L.P_i32), a[1].ctypes.data_as(L.P_i32),
                 a[2].ctypes.data_as(L.P_i64),  a[3].ctypes.data_as(L.P_f64),
                 a[4].ctypes.data_as(L.P_f64), a[5].ctypes.data_as(L.P_f64)))
        for kind, lst in enumerate((model.ms_stf, model.fs_stf, model.ps_stf)):
            for i, st in enumerate(lst):
                if getattr(st, "table", None) is not None:
                    tt = np.ascontiguousarray(st.table[0], np.float64)
                    vv = np.ascontiguousarray(st.table[1], np.float64)
                    self._chk(self.O.axo_set_stf_table(self.h, kind, i, len(tt), tt.ctypes.data_as(L.P_f64), vv.ctypes.data_as(L.P_f64),
                        int(st.padding), float(st.left), float(st.right), int(st.pad_first)))
        self._chk(self.O.axo_set_stations(self.h, C.byref(s["st"]), int(model.st_interval)))
        for solid, key in ((1, "cl_s"), (0, "cl_f")):
            if s[key].count:
                self._chk(self.O.axo_set_clayton(self.h, solid, C.byref(s[key])))
        for solid, (pt, g) in ((1, s["sg_s"]), (0, s["sg_f"])):
            if pt is not None and len(pt):
                self._chk(self.O.axo_set_sponge(self.h, solid, len(pt), pt.ctypes.data_as(L.P_i32),
                                                g.ctypes.data_as(L.P_f64)))
        for solid, key in ((1, "cl3_s"), (0, "cl3_f")):
            if s[key].count:
                self._chk(self.O.axo_set_clayton3d(self.h, solid, C.byref(s[key])))
        for solid, (pt, off, g) in ((1, s["sg3_s"]), (0, s["sg3_f"])):
            if pt is not None and len(pt):
                self._chk(self.O.axo_set_sponge3d(self.h, solid, len(pt), pt.ctypes.data_as(L.P_i32),
                                                  off.ctypes.data_as(L.P_i64), g.ctypes.data_as(L.P_f64)))
        if s["scan"] is not None:
            self._chk(self.O.axo_set_scanning(self.h, C.byref(s["scan"])))
        if s["prt"] is not None:
            e, off, x3, x, _ = s["prt"]
            self._chk(self.O.axo_set_prt(self.h, len(e), e.ctypes.data_as(L.P_i32), off.ctypes.data_as(L.P_i64),
                                         x3.ctypes.data_as(L.P_u8), x.ctypes.data_as(L.P_f64)))
        if s["prt_f"] is not None:
            e, off, x3, x, th = s["prt_f"]
            self._chk(self.O.axo_set_prt_fluid(self.h, len(e), e.ctypes.data_as(L.P_i32),
                                               off.ctypes.data_as(L.P_i64), x3.ctypes.data_as(L.P_u8),
                                               x.ctypes.data_as(L.P_f64),
                                               th.ctypes.data_as(L.P_f64) if th is not None else None))
        if s["ocean3"] is not None:
            pt, off, mo, nrm = s["ocean3"]
            self._chk(self.O.axo_set_ocean_load3d(self.h, len(pt), pt.ctypes.data_as(L.P_i32),
                                                  off.ctypes.data_as(L.P_i64), mo.ctypes.data_as(L.P_f64),
                                                  nrm.ctypes.data_as(L.P_f64)))
        pt, mo, th = s["ocean"]
        if pt is not None and len(pt):
            self._chk(self.O.axo_set_ocean_load(self.h, len(pt), pt.ctypes.data_as(L.P_i32),
                                                mo.ctypes.data_as(L.P_f64), th.ctypes.data_as(L.P_f64)))
        sp_, fp_ = getattr(model, "se_part", None), getattr(model, "fe_part", None)
        if sp_ is not None or fp_ is not None:
            self._parts = [np.ascontiguousarray(x, np.uint8) if x is not None else None for x in (sp_, fp_)]
            a, b = self._parts
            self._chk(self.O.axo_set_element_parts(self.h, a.ctypes.data if a is not None else None,
                                                   0 if a is None else len(a),
                                                   b.ctypes.data if b is not None else None,
                                                   0 if b is None else len(b)))

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(self.O.axo_last_error(self.h).decode())

    def close(self):
        if self.h:
            self.O.axo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def apply_sources(self, tstep):
        self._chk(self.O.axo_apply_sources(self.h, int(tstep)))

    def compute_stiffness(self):
        self._chk(self.O.axo_compute_stiffness(self.h, int(self.threads)))

    def compute_stiffness_part(self, part):
        self._chk(self.O.axo_compute_stiffness_part(self.h, int(self.threads), int(part)))

    def apply_bc_before_assembly(self):
        self._chk(self.O.axo_bc_before(self.h))

    def apply_bc_after_assembly(self):
        self._chk(self.O.axo_bc_after(self.h))

    def stiff_to_accel(self):
        self._chk(self.O.axo_stiff_to_accel(self.h))

    def newmark_update(self):
        self._chk(self.O.axo_newmark(self.h))

    def record_stations(self, tstep):
        self._chk(self.O.axo_record(self.h, int(tstep)))

    def run(self, nsteps):
        self._chk(self.O.axo_run(self.h, int(nsteps), int(self.threads)))

    def scanning_nr(self):
        ns, nf = len(self.model.sp_nr), len(self.model.fp_nr)
        a = np.zeros(max(ns, 1), np.int32)
        b = np.zeros(max(nf, 1), np.int32)
        self._chk(self.O.axo_scanning_nr(self.h, a.ctypes.data_as(self.L.P_i32), b.ctypes.data_as(self.L.P_i32)))
        return a[:ns], b[:nf]

    def reset_attenuation(self):
        self._chk(self.O.axo_reset_attenuation(self.h))

    def field_size(self, solid=True):
        return int(self.O.axo_field_size(self.h, int(bool(solid))))

    def get_field(self, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        out = np.zeros(self.field_size(solid), dtype=np.complex128)
        if out.size:
            self._chk(self.O.axo_get_field(self.h, int(bool(solid)), w,
                                           out.view(np.float64).ctypes.data_as(self.L.P_f64)))
        return out

    def set_field(self, values, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        v = np.ascontiguousarray(values, dtype=np.complex128)
        assert v.size == self.field_size(solid)
        self._chk(self.O.axo_set_field(self.h, int(bool(solid)), w,
                                       v.view(np.float64).ctypes.data_as(self.L.P_f64)))

    def seismograms(self):
        n = self.O.axo_get_seismograms(self.h, None)
        ns = len(self.model.st_elem)
        out = np.zeros((n, ns, 3))
        if n and ns:
            self.O.axo_get_seismograms(self.h, out.ctypes.data_as(self.L.P_f64))
        return out
