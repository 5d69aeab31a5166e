"""Python mirror of the engine's C ABI, shaped like the reference's time loop.

``Solver`` wraps one ``axg_solver`` handle. Its methods are the per-step hooks
of AxiSEM3D's Domain / NewmarkTimeScheme, in the order of
NewmarkTimeScheme::solve (SOLVER/src/core/time/NewmarkTimeScheme.cpp:41-108):

    apply_sources(tstep)       Domain::applySources
    compute_stiffness()        Domain::computeStiffness
    apply_bc_before_assembly() Domain::applyBC_BeforeAssemblingStiff
    record_stations(tstep)     Domain::recordOutput (station displacement)
    apply_bc_after_assembly()  Domain::applyBC_AfterAssemblingStiff
    stiff_to_accel()           Domain::computeStiffToAccel
    newmark_update()           NewmarkTimeScheme::update on all points
    run(nsteps)                the whole loop body, one CUDA graph per step

Errors raise ``RuntimeError`` with the engine's "Class::method || message"
text, as the reference throws std::runtime_error.
"""
import ctypes as C

import numpy as np

from . import _lib as L


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Solver:
    def __init__(self, model, precision="fp32", device=0, stability_interval=0, compensated=True,
                 team_sizes=None, plain=False, autotune=False, deterministic=False):
        self.lib = L.lib()
        self.model = model
        self.precision = precision
        cfg = model.config(precision, device=device, stability_interval=stability_interval,
                           compensated=int(bool(compensated)), plain=plain, autotune=autotune,
                           deterministic=deterministic)
        h = C.c_void_p()
        rc = self.lib.axg_create(C.byref(cfg), C.byref(h))
        if rc != L.AXG_OK:
            raise EngineError(rc, "axg_create failed (%d): %s" % (rc, self.lib.axg_last_error(None).decode()))
        self.h = h
        s = model.c_structs()
        self._keep = s
        self._check(self.lib.axg_set_solid_points(h, C.byref(s["sp"])))
        if s["fp"].count:
            self._check(self.lib.axg_set_fluid_points(h, C.byref(s["fp"])))
        self._check(self.lib.axg_set_solid_elements(h, C.byref(s["se"])))
        if s["fe"].count:
            self._check(self.lib.axg_set_fluid_elements(h, C.byref(s["fe"])))
        if s["sf"].count:
            self._check(self.lib.axg_set_solid_fluid(h, C.byref(s["sf"])))
        if s["ms"].count:
            self._check(self.lib.axg_set_moment_sources(h, C.byref(s["ms"])))
        if s["fs"].count:
            self._check(self.lib.axg_set_force_sources(h, C.byref(s["fs"])))
        if s["ps"].count:
            self._check(self.lib.axg_set_pressure_sources(h, C.byref(s["ps"])))
        if getattr(model, "sf3", None):
            d3 = model.sf3
            self._sf3 = [np.ascontiguousarray(d3[k], dt) for k, dt in (
                ("solid", np.int32), ("fluid", np.int32), ("offset", np.int64), ("normal_u", np.float64),
                ("normal_a", np.float64), ("mass_fluid", np.float64))]
            a = self._sf3
            self._check(self.lib.axg_set_solid_fluid3d(h, len(a[0]), a[0].ctypes.data_as(L.P_i32), a[1].ctypes.data_as(L.P_i32),
                 a[2].ctypes.data_as(L.P_i64),  len(a[5]), a[3].ctypes.data_as(L.P_f64),
                 a[4].ctypes.data_as(L.P_f64), a[5].ctypes.data_as(L.P_f64)))
        for kind, lst in enumerate((model.ms_stf, model.fs_stf, model.ps_stf)):
            for i, st in enumerate(lst):
                if getattr(st, "table", None) is not None:
                    tt = np.ascontiguousarray(st.table[0], np.float64)
                    vv = np.ascontiguousarray(st.table[1], np.float64)
                    self._check(self.lib.axg_set_stf_table(h, kind, i, len(tt), tt.ctypes.data_as(L.P_f64), vv.ctypes.data_as(L.P_f64),
                        int(st.padding), float(st.left), float(st.right), int(st.pad_first)))
        if s["st"].count:
            self._check(self.lib.axg_set_stations(h, C.byref(s["st"]), int(model.st_interval)))
            if getattr(model, "st_gradient", False):
                self._check(self.lib.axg_set_station_gradient(h, 1))
        for solid, key in ((1, "cl_s"), (0, "cl_f")):
            if s[key].count:
                self._check(self.lib.axg_set_clayton(h, solid, C.byref(s[key])))
        for solid, (pt, g) in ((1, s["sg_s"]), (0, s["sg_f"])):
            if pt is not None and len(pt):
                self._check(self.lib.axg_set_sponge(h, solid, len(pt), pt.ctypes.data_as(L.P_i32),
                                                    g.ctypes.data_as(L.P_f64)))
        for solid, key in ((1, "cl3_s"), (0, "cl3_f")):
            if s[key].count:
                self._check(self.lib.axg_set_clayton3d(h, solid, C.byref(s[key])))
        for solid, (pt, off, g) in ((1, s["sg3_s"]), (0, s["sg3_f"])):
            if pt is not None and len(pt):
                self._check(self.lib.axg_set_sponge3d(h, solid, len(pt), pt.ctypes.data_as(L.P_i32),
                                                      off.ctypes.data_as(L.P_i64), len(g),
                                                      g.ctypes.data_as(L.P_f64)))
        if s["scan"] is not None:
            self._check(self.lib.axg_set_scanning(h, C.byref(s["scan"])))
        if s["prt"] is not None:
            e, off, x3, x, _ = s["prt"]
            self._check(self.lib.axg_set_prt(h, len(e), e.ctypes.data_as(L.P_i32), off.ctypes.data_as(L.P_i64),
                                             x3.ctypes.data_as(L.P_u8), len(x), x.ctypes.data_as(L.P_f64)))
        if s["prt_f"] is not None:
            e, off, x3, x, th = s["prt_f"]
            self._check(self.lib.axg_set_prt_fluid(h, len(e), e.ctypes.data_as(L.P_i32),
                                                   off.ctypes.data_as(L.P_i64), x3.ctypes.data_as(L.P_u8), len(x),
                                                   x.ctypes.data_as(L.P_f64),
                                                   th.ctypes.data_as(L.P_f64) if th is not None else None))
        if s["ocean3"] is not None:
            pt, off, mo, nrm = s["ocean3"]
            self._check(self.lib.axg_set_ocean_load3d(h, len(pt), pt.ctypes.data_as(L.P_i32),
                                                      off.ctypes.data_as(L.P_i64), len(mo),
                                                      mo.ctypes.data_as(L.P_f64), nrm.ctypes.data_as(L.P_f64)))
        pt, mo, th = s["ocean"]
        if pt is not None and len(pt):
            self._check(self.lib.axg_set_ocean_load(h, len(pt), pt.ctypes.data_as(L.P_i32),
                                                    mo.ctypes.data_as(L.P_f64), th.ctypes.data_as(L.P_f64)))
        for cls, team in (team_sizes or {}).items():
            self._check(self.lib.axg_set_team_size(h, int(cls), int(team)))
        sp_, fp_ = getattr(model, "se_part", None), getattr(model, "fe_part", None)
        if sp_ is not None or fp_ is not None:
            a = np.ascontiguousarray(sp_, np.uint8) if sp_ is not None else None
            b = np.ascontiguousarray(fp_, np.uint8) if fp_ is not None else None
            self._check(self.lib.axg_set_element_parts(h, a.ctypes.data if a is not None else None,
                                                       b.ctypes.data if b is not None else None))
        self._check(self.lib.axg_finalize(h))

    # ------------------------------------------------------------------ util ---
    def _check(self, rc):
        if rc != L.AXG_OK:
            msg = self.lib.axg_last_error(self.h).decode()
            raise EngineError(rc, msg or ("axg error %d" % rc))

    def close(self):
        if getattr(self, "h", None):
            self.lib.axg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------------ hooks ---
    def apply_sources(self, tstep):
        self._check(self.lib.axg_apply_sources(self.h, int(tstep)))

    def compute_stiffness(self):
        self._check(self.lib.axg_compute_stiffness(self.h))

    def scanning_nr(self):
        """Point::reportScanningNr of every solid and fluid point (-1: not scanned)."""
        ns, nf = len(self.model.sp_nr), len(self.model.fp_nr)
        a = np.zeros(max(ns, 1), np.int32)
        b = np.zeros(max(nf, 1), np.int32)
        self._check(self.lib.axg_scanning_nr(self.h, a.ctypes.data_as(L.P_i32), b.ctypes.data_as(L.P_i32)))
        return a[:ns], b[:nf]

    def compute_stiffness_noalloc(self, solid_x, solid_f, fluid_x=None, fluid_f=None):
        """f -= K x for caller-owned device buffers (integer device addresses, complex in the
        handle's stiffness precision), with no device allocation by the library: the
        evaluation's SLS memory lives in the library's fixed device array (see
        axg_compute_stiffness_noalloc in include/axg.h for its limit and sharing rules)."""
        self._check(self.lib.axg_compute_stiffness_noalloc(self.h, solid_x, solid_f, fluid_x, fluid_f))

    def gather_stiffness(self, slots_ptr, n, buf_ptr, solid=True):
        """buf[i] = stiff[slots[i]] for n DEVICE slots (int64) into a DEVICE buffer of complex
        values in the stiffness precision (MessageRank::gatherFromPoints)."""
        self._check(self.lib.axg_gather_stiffness(self.h, int(bool(solid)), int(n), slots_ptr, buf_ptr))

    def scatter_add_stiffness(self, slots_ptr, n, buf_ptr, solid=True):
        """stiff[slots[i]] += buf[i] (MessageRank::scatterToPoints / SolidPoint::extractComm)."""
        self._check(self.lib.axg_scatter_add_stiffness(self.h, int(bool(solid)), int(n), slots_ptr, buf_ptr))

    @property
    def complex_dtype(self):
        """numpy dtype of the stiffness field on the device."""
        return np.complex128 if self.precision == "fp64" else np.complex64

    def compute_stiffness_part(self, part):
        """Domain::computeStiffness for the elements of one part (model.se_part / fe_part)."""
        self._check(self.lib.axg_compute_stiffness_part(self.h, int(part)))

    def apply_bc_before_assembly(self):
        self._check(self.lib.axg_apply_bc_before_assembly(self.h))

    def apply_bc_after_assembly(self):
        self._check(self.lib.axg_apply_bc_after_assembly(self.h))

    def stiff_to_accel(self):
        self._check(self.lib.axg_stiff_to_accel(self.h))

    def newmark_update(self):
        self._check(self.lib.axg_newmark_update(self.h))

    def record_stations(self, tstep):
        self._check(self.lib.axg_record_stations(self.h, int(tstep)))

    def run(self, nsteps, graph=True):
        self._check(self.lib.axg_run(self.h, int(nsteps), int(bool(graph))))

    def synchronize(self):
        self._check(self.lib.axg_synchronize(self.h))

    @property
    def step(self):
        t = C.c_int32()
        self._check(self.lib.axg_current_step(self.h, C.byref(t)))
        return t.value

    # ----------------------------------------------------------------- fields ---
    def field_size(self, solid=True):
        n = C.c_int64()
        self._check(self.lib.axg_field_size(self.h, int(bool(solid)), C.byref(n)))
        return n.value

    def get_field(self, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        n = self.field_size(solid)
        out = np.zeros(n, dtype=np.complex128)
        if n:
            self._check(self.lib.axg_get_field(self.h, int(bool(solid)), w,
                                               out.view(np.float64).ctypes.data_as(L.P_f64)))
        return out

    def set_field(self, values, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        v = np.ascontiguousarray(values, dtype=np.complex128)
        if v.size != self.field_size(solid):
            raise EngineError(L.AXG_E_ARG, "axg_set_field || size mismatch")
        self._check(self.lib.axg_set_field(self.h, int(bool(solid)), w,
                                           v.view(np.float64).ctypes.data_as(L.P_f64)))

    def field_raw_bytes(self, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        n = C.c_int64()
        self._check(self.lib.axg_field_raw_bytes(self.h, int(bool(solid)), w, C.byref(n)))
        return n.value

    def set_field_raw(self, host_ptr, nbytes, which="displ", solid=True):
        """Asynchronous native-precision copy from a (pinned) host address."""
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        self._check(self.lib.axg_set_field_raw(self.h, int(bool(solid)), w, C.c_void_p(host_ptr), int(nbytes)))

    def get_field_raw(self, host_ptr, nbytes, which="displ", solid=True):
        w = {"stiff": 0, "displ": 1, "veloc": 2, "accel": 3}[which]
        self._check(self.lib.axg_get_field_raw(self.h, int(bool(solid)), w, C.c_void_p(host_ptr), int(nbytes)))

    def seismograms(self):
        """(nrecords, nstations, 3) displacement in s, phi, z; with batched
        wavefields (nrecords, nwave, nstations, 3)."""
        n = C.c_int32()
        self._check(self.lib.axg_get_seismograms(self.h, None, C.byref(n)))
        ns = len(self.model.st_elem)
        nw = max(1, int(self.model.nwave))
        out = np.zeros((n.value, nw, ns, 3))
        if n.value and ns:
            self._check(self.lib.axg_get_seismograms(self.h, out.ctypes.data_as(L.P_f64), C.byref(n)))
        return out[:, 0] if nw == 1 else out

    def station_gradients(self):
        """(nrecords, nstations, 9) displacement gradient d_j u_i (index 3 i + j, s / phi / z)
        at the stations; with batched wavefields (nrecords, nwave, nstations, 9)."""
        n = C.c_int32()
        self._check(self.lib.axg_get_station_gradients(self.h, None, C.byref(n)))
        ns = len(self.model.st_elem)
        nw = max(1, int(self.model.nwave))
        out = np.zeros((n.value, nw, ns, 9))
        if n.value and ns:
            self._check(self.lib.axg_get_station_gradients(self.h, out.ctypes.data_as(L.P_f64), C.byref(n)))
        return out[:, 0] if nw == 1 else out

    def set_element_record(self, elem, gll, kind, interval, ring):
        """Record, every `interval` steps into a device ring of `ring` records, the Fourier
        coefficients (orders < nr/2 + 1 of the element) of the displacement (kind 0) or its
        gradient (kind 1) at GLL point gll[i] of solid element elem[i]."""
        e = np.ascontiguousarray(elem, np.int32)
        g = np.ascontiguousarray(gll, np.int32)
        k = np.ascontiguousarray(kind, np.int32)
        if not (len(e) == len(g) == len(k)):
            raise ValueError("elem, gll and kind differ in length")
        self._check(self.lib.axg_set_element_record(self.h, len(e), e.ctypes.data_as(L.P_i32),
                                                    g.ctypes.data_as(L.P_i32), k.ctypes.data_as(L.P_i32),
                                                    int(interval), int(ring)))
        w = C.c_int64()
        self._check(self.lib.axg_element_record_words(self.h, C.byref(w)))
        self._er_words = int(w.value)
        return self._er_words

    def element_records(self, rec_first, nrec):
        """Records rec_first .. rec_first + nrec - 1 as complex [nrec, nwave, words]
        (without the wavefield axis for one wavefield)."""
        nw = max(1, int(self.model.nwave))
        out = np.zeros((int(nrec), nw, self._er_words, 2))
        self._check(self.lib.axg_get_element_records(self.h, int(rec_first), int(nrec),
                                                     out.ctypes.data_as(L.P_f64)))
        c = out[..., 0] + 1j * out[..., 1]
        return c[:, 0] if nw == 1 else c

    # -------------------------------------------------------- differentiation ---
    def forward_checkpointed(self, nsteps, interval=100):
        """nsteps forward steps keeping a device checkpoint every `interval` steps."""
        self._check(self.lib.axg_forward_checkpointed(self.h, int(nsteps), int(interval)))

    def adjoint(self, seis_adjoint, slices=False):
        """Discrete adjoint of the last checkpointed run for dJ/d(seismograms).

        Returns dJ/d(moduli) per element point, dJ/d(point mass), and dJ/d(initial
        displacement / velocity) in the field layout. The moduli gradient follows each
        element's moduli (lambda, mu; A, C, F, L, N; the 21 Cij), then, for an attenuating
        element, its dlambda, dmu (with CG4 at the four CG4 points): an (ne, nmod, 25) array when
        every element has the same rheology, (ne, 2, 25) for an isotropic model, else a list of
        (nmod_e, 25) arrays. With slices=True also
        the per-slice sensitivities of the 3-D parameterisation: "moduli_slices", a list of
        (2, nr_e, 25) arrays (lambda, mu at phi_k = 2 pi k / nr_e), and "mass_slices", a list of
        (nr_p,) arrays per solid point."""
        ne = self.model.n_solid_elements
        self._check(self.lib.axg_set_adjoint_slices(self.h, int(bool(slices))))
        r = np.ascontiguousarray(seis_adjoint, dtype=np.float64)
        nmod = np.array([{L.AXG_ISO: 2, L.AXG_TISO: 5, L.AXG_ANISO: 21}[int(r)]
                         for r in np.asarray(self.model.se_rheo).ravel()], np.int64)
        if self.model.se_att is not None:       # attenuating elements: + dlambda, dmu
            nmod = nmod + 2 * (np.asarray(self.model.se_att).ravel() != L.AXG_ATT_NONE)
        gflat = np.zeros(int(np.sum(nmod)) * 25)
        gmass = np.zeros(len(self.model.sp_nr))
        nf = self.field_size(True)
        gu = np.zeros(nf, dtype=np.complex128)
        gv = np.zeros(nf, dtype=np.complex128)
        self._check(self.lib.axg_adjoint_run(self.h, r.ctypes.data_as(L.P_f64), gflat.ctypes.data_as(L.P_f64),
                                             gmass.ctypes.data_as(L.P_f64),
                                             gu.view(np.float64).ctypes.data_as(L.P_f64),
                                             gv.view(np.float64).ctypes.data_as(L.P_f64)))
        if ne == 0 or np.all(nmod == nmod[0]):
            gm = gflat.reshape(ne, int(nmod[0]) if ne else 2, 25)
        else:
            go = np.concatenate([[0], np.cumsum(nmod * 25)])
            gm = [gflat[go[e]:go[e + 1]].reshape(nmod[e], 25) for e in range(ne)]
        out = {"moduli": gm, "mass": gmass, "displ0": gu, "veloc0": gv}
        if slices:
            enr = np.asarray(self.model.se_nr, np.int64)
            pnr = np.asarray(self.model.sp_nr, np.int64)
            g3 = np.zeros(int(np.sum(2 * enr * 25)))
            m3 = np.zeros(int(np.sum(pnr)))
            self._check(self.lib.axg_get_adjoint_slices(self.h, g3.ctypes.data_as(L.P_f64),
                                                        m3.ctypes.data_as(L.P_f64)))
            eo = np.concatenate([[0], np.cumsum(2 * enr * 25)])
            po = np.concatenate([[0], np.cumsum(pnr)])
            out["moduli_slices"] = [g3[eo[e]:eo[e + 1]].reshape(2, enr[e], 25) for e in range(ne)]
            out["mass_slices"] = [m3[po[p]:po[p + 1]] for p in range(len(pnr))]
        return out

    # ------------------------------------------------------------ diagnostics ---
    def launch_count(self):
        n = C.c_int64()
        self._check(self.lib.axg_launch_count(self.h, C.byref(n)))
        return n.value

    def set_timing(self, on=True):
        self._check(self.lib.axg_set_timing(self.h, int(bool(on))))

    def stiffness_time(self):
        ms, n = C.c_double(), C.c_int64()
        self._check(self.lib.axg_stiffness_time_ms(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def stiffness_cost(self):
        b, f = C.c_double(), C.c_double()
        self._check(self.lib.axg_stiffness_cost(self.h, C.byref(b), C.byref(f)))
        return b.value, f.value

    def point_cost(self):
        b = C.c_double()
        self._check(self.lib.axg_point_cost(self.h, C.byref(b)))
        return b.value

    def set_stream(self, stream_ptr):
        self._check(self.lib.axg_set_stream(self.h, C.c_void_p(stream_ptr)))


# --------------------------------------------------------- operand builders ---
def spectral_tables():
    lib = L.lib()
    bufs = [np.zeros(5) for _ in range(4)] + [np.zeros(25), np.zeros(25)]
    lib.axg_spectral_tables(*[b.ctypes.data_as(L.P_f64) for b in bufs])
    return dict(zip(["pGLL", "pGLJ", "wGLL", "wGLJ", "gGLL", "gGLJ"], bufs))


def quad_geometry(nodal_sz, axial, mapping=L.AXG_MAP_LINEAR):
    """Quad::createGradient operands: (6, 25) geometry and (2, 25) point coordinates."""
    lib = L.lib()
    n = np.ascontiguousarray(nodal_sz, dtype=np.float64).reshape(8)
    g = np.zeros(150)
    sz = np.zeros(50)
    rc = lib.axg_quad_geometry(int(mapping), n.ctypes.data_as(L.P_f64), int(bool(axial)),
                               g.ctypes.data_as(L.P_f64), sz.ctypes.data_as(L.P_f64))
    if rc != L.AXG_OK:
        raise EngineError(rc, "axg_quad_geometry failed (%d)" % rc)
    return g.reshape(6, 25), sz.reshape(2, 25)


def quad_dt(sz, vmax):
    lib = L.lib()
    s = np.ascontiguousarray(sz, dtype=np.float64).reshape(50)
    dt = C.c_double()
    rc = lib.axg_quad_dt(s.ctypes.data_as(L.P_f64), float(vmax), C.byref(dt))
    if rc != L.AXG_OK:
        raise EngineError(rc, "axg_quad_dt failed")
    return dt.value


def att_alpha_beta_gamma(w, y, dt):
    lib = L.lib()
    w = np.ascontiguousarray(w, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    a, b, g = np.zeros(len(w)), np.zeros(len(w)), np.zeros(len(w))
    rc = lib.axg_att_alpha_beta_gamma(len(w), w.ctypes.data_as(L.P_f64), y.ctypes.data_as(L.P_f64),
                                      float(dt), a.ctypes.data_as(L.P_f64), b.ctypes.data_as(L.P_f64),
                                      g.ctypes.data_as(L.P_f64))
    if rc != L.AXG_OK:
        raise EngineError(rc, "axg_att_alpha_beta_gamma failed")
    return a, b, g


def att_moduli(w, y, fmin, fmax, fref, qkappa, qmu, kp, mu):
    """AttBuilder::createAttenuation (FULL): returns (kp_unrelaxed, mu_unrelaxed, dkp, dmu)."""
    lib = L.lib()
    w = np.ascontiguousarray(w, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    qk = np.ascontiguousarray(np.broadcast_to(qkappa, np.shape(kp)), dtype=np.float64).ravel()
    qm = np.ascontiguousarray(np.broadcast_to(qmu, np.shape(kp)), dtype=np.float64).ravel()
    kp2 = np.array(kp, dtype=np.float64).ravel().copy()
    mu2 = np.array(mu, dtype=np.float64).ravel().copy()
    dk, dm = np.zeros_like(kp2), np.zeros_like(kp2)
    rc = lib.axg_att_moduli(len(w), w.ctypes.data_as(L.P_f64), y.ctypes.data_as(L.P_f64),
                            float(fmin), float(fmax), float(fref), len(kp2),
                            qk.ctypes.data_as(L.P_f64), qm.ctypes.data_as(L.P_f64),
                            kp2.ctypes.data_as(L.P_f64), mu2.ctypes.data_as(L.P_f64),
                            dk.ctypes.data_as(L.P_f64), dm.ctypes.data_as(L.P_f64))
    if rc != L.AXG_OK:
        raise EngineError(rc, "axg_att_moduli failed")
    shp = np.shape(kp)
    return kp2.reshape(shp), mu2.reshape(shp), dk.reshape(shp), dm.reshape(shp)
