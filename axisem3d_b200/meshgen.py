"""Seeded synthetic meshes and models for the benchmark and parity workloads.

The reference reads Exodus meshes written by its Python mesher and builds
operands in its preloop; this module plays that role for synthetic inputs. It
lays out structured quad meshes, calls the engine's host operand builders
(``axg_quad_geometry_batch``, ``axg_quad_dt``, ``axg_att_*`` -- the
restatements of Quad::createGradient, Quad::computeDt and AttBuilder) and
applies the material formulas of Material::createIsotropic / createTISO /
createAnisotropic (SOLVER/src/preloop/se_model/quad/physical/Material.cpp:385-609).
All randomness comes from numpy PCG64 generators with the seeds given.

Workloads (sizes in SI units):
  cartesian_model   plain forward case: 40 x 40 quads on 100 km x 100 km with the
                    axis at s = 0, nr = 5, homogeneous isotropic medium, moment
                    tensor on the axis at 10 km depth, Ricker 1 Hz, 20 surface
                    receivers, dt from Courant 0.6.
  microbench_model  stiffness microbenchmark: ~200k non-axial solid quads, nr per
                    element log-uniform on [1, 64], transversely isotropic moduli at
                    +-10 % around vp = 8, vs = 4.5 km/s, rho = 3.3 g/cc per
                    (element, slice, point), 3 SLS with Q_mu uniform in [80, 600].
  spherical_model   spherical-shell analogue: annulus 3480-6371 km with a fluid
                    layer 3480-3600 km, 1-D layered background, 2 % Gaussian
                    random-field dlnVs setting per-element nr, Q = 300.
"""
import contextlib
import math

import numpy as np

from . import _lib as L
from .model import Model, STF


# ------------------------------------------------------- operand builders ---
class EngineOperands:
    """The engine's host operand builders (libaxg.so: axg_spectral_tables,
    axg_quad_geometry_batch, axg_quad_dt, axg_att_alpha_beta_gamma, axg_att_moduli), the
    restatements of the reference's preloop numbers that every workload here is built with."""

    def tables(self):
        from .solver import spectral_tables
        return spectral_tables()

    def geometry_batch(self, nodal, axial, mapping=L.AXG_MAP_LINEAR):
        lib = L.lib()
        ne = len(axial)
        nodal = np.ascontiguousarray(nodal, dtype=np.float64).reshape(ne, 8)
        ax = np.ascontiguousarray(axial, dtype=np.uint8)
        g = np.zeros((ne, 6, 25))
        sz = np.zeros((ne, 2, 25))
        rc = lib.axg_quad_geometry_batch(ne, int(mapping), nodal.ctypes.data_as(L.P_f64),
                                         ax.ctypes.data_as(L.P_u8), g.ctypes.data_as(L.P_f64),
                                         sz.ctypes.data_as(L.P_f64))
        if rc != L.AXG_OK:
            raise RuntimeError("axg_quad_geometry_batch failed (%d)" % rc)
        return g, sz

    def quad_dt(self, sz, vmax):
        from .solver import quad_dt
        return quad_dt(sz, vmax)

    def att_alpha_beta_gamma(self, w, y, dt):
        from .solver import att_alpha_beta_gamma
        return att_alpha_beta_gamma(w, y, dt)

    def att_moduli(self, w, y, fmin, fmax, fref, qkappa, qmu, kp, mu):
        from .solver import att_moduli
        return att_moduli(w, y, fmin, fmax, fref, qkappa, qmu, kp, mu)


# the builder in use: the engine's, unless a caller installs another with `operands`
_OPS = [EngineOperands()]
_TAB = {}


@contextlib.contextmanager
def operands(builder):
    """Build workloads with another operand builder inside the block: an object with the
    methods of EngineOperands (tables, geometry_batch, quad_dt, att_alpha_beta_gamma,
    att_moduli). The models come out the same up to the builders' rounding; a model built
    this way needs no engine library."""
    _OPS.append(builder)
    try:
        yield builder
    finally:
        _OPS.pop()


def tables():
    """GLL / GLJ tables (nPol = 4) of the builder in use."""
    b = _OPS[-1]
    if id(b) not in _TAB:
        _TAB[id(b)] = (b, b.tables())
    return _TAB[id(b)][1]


def quad_dt(sz, vmax):
    return _OPS[-1].quad_dt(sz, vmax)


def att_alpha_beta_gamma(w, y, dt):
    return _OPS[-1].att_alpha_beta_gamma(w, y, dt)


def att_moduli(w, y, fmin, fmax, fref, qkappa, qmu, kp, mu):
    return _OPS[-1].att_moduli(w, y, fmin, fmax, fref, qkappa, qmu, kp, mu)


def lagrange(nodes, x):
    """Lagrange basis values l_j(x) on the given nodes (SE_Model::computeInplaneFactor)."""
    n = len(nodes)
    w = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                w[j] *= (x - nodes[k]) / (nodes[j] - nodes[k])
    return w


def inplane_weights(xi, eta, axial):
    t = tables()
    wx = lagrange(t["pGLJ"] if axial else t["pGLL"], xi)
    we = lagrange(t["pGLL"], eta)
    return np.outer(wx, we).ravel()


def round_dt(dt):
    """SE_Model::computeDt: round to 4 significant figures ("%.3e")."""
    return float("%.3e" % dt)


# ------------------------------------------------------------------ geometry ---
def geometry_batch(nodal, axial, mapping=L.AXG_MAP_LINEAR):
    """Quad::createGradient for all quads: (ne, 6, 25) operands and (ne, 2, 25) s, z."""
    return _OPS[-1].geometry_batch(nodal, axial, mapping)


def structured_points(nx, nz):
    """Element -> GLL point map of an nx x nz structured quad grid (I = 4i + ipol, J = 4j + jpol)."""
    nJ = 4 * nz + 1
    i = np.arange(nx)[:, None, None, None]
    j = np.arange(nz)[None, :, None, None]
    ip = np.arange(5)[None, None, :, None]
    jp = np.arange(5)[None, None, None, :]
    pts = (4 * i + ip) * nJ + (4 * j + jp)
    return pts.reshape(nx * nz, 25).astype(np.int32), (4 * nx + 1) * nJ


def assemble_mass(pts, ifact, density, npoints):
    """Material::getMass: mass[ipnt] = density * integral factor, summed over elements."""
    m = np.zeros(npoints)
    np.add.at(m, pts.ravel(), (density * ifact).ravel())
    return m


# ------------------------------------------------------------------ materials ---
def isotropic_moduli(rho, vp, vs):
    """Material::createIsotropic without attenuation: lambda = rho vp^2 - 2 mu, mu = rho vs^2."""
    mu = rho * vs ** 2
    lam = rho * vp ** 2 - 2.0 * mu
    return lam, mu


def tiso_with_attenuation(A, C, F, Lm, N, qkappa, qmu, sls):
    """Material::createTISO with attenuation (Material.cpp:497-560) -> unrelaxed A, C, F, L, N,
    dlambda, dmu (AttBuilder::createAttenuation, FULL)."""
    kp = (A * 4. + C + F * 4. - N * 4.) / 9.
    mu = (A + C - F * 2. + Lm * 6. + N * 5.) / 15.
    A = A - (kp + 4. / 3. * mu)
    C = C - (kp + 4. / 3. * mu)
    F = F - (kp - 2. / 3. * mu)
    Lm = Lm - mu
    N = N - mu
    kp2, mu2, dkp, dmu = att_moduli(sls["w"], sls["y"], sls["fmin"], sls["fmax"], sls["fref"],
                                    qkappa, qmu, kp, mu)
    A = A + (kp2 + 4. / 3. * mu2)
    C = C + (kp2 + 4. / 3. * mu2)
    F = F + (kp2 - 2. / 3. * mu2)
    Lm = Lm + mu2
    N = N + mu2
    dlam = dkp - (2. / 3.) * dmu
    return A, C, F, Lm, N, dlam, dmu


def iso_with_attenuation(lam, mu, qkappa, qmu, sls):
    """Material::createIsotropic with attenuation (Material.cpp:563-609)."""
    kp = lam + (2. / 3.) * mu
    kp2, mu2, dkp, dmu = att_moduli(sls["w"], sls["y"], sls["fmin"], sls["fmax"], sls["fref"],
                                    qkappa, qmu, kp, mu)
    lam2 = kp2 - (2. / 3.) * mu2
    return lam2, mu2, dkp - (2. / 3.) * dmu, dmu


def att_factors(q, sls):
    """AttBuilder::createAttenuation factors for one quality factor array
    (AttBuilder.cpp:106-124): (NA, d, AT) with modulus_unrelaxed = modulus * AT
    (FULL) and dmodulus = d * modulus."""
    w, y = np.asarray(sls["w"]), np.asarray(sls["y"])
    ysum = y.sum()
    w0 = sls["fref"] * (2 * np.pi)
    w1 = math.sqrt(sls["fmin"] * sls["fmax"]) * (2. * np.pi)
    w10f = 2. * math.log(w1 / w0) / np.pi
    fact = float(np.sum(y * w ** 2 / (w ** 2 + w1 * w1)) / ysum)
    q = np.asarray(q, dtype=np.float64)
    na = 1. + w10f / q
    d = na / (q / ysum + (1. - fact))
    return na, d, na + d * fact


CG4_POINTS = np.array([6, 8, 16, 18])


def weights_cg4(ifact):
    """Quad::computeWeightsCG4 (Quad.cpp:487-511) from the (.., 25) integral factor."""
    f = np.asarray(ifact).reshape(-1, 5, 5)
    w = np.zeros((f.shape[0], 4))
    w[:, 0] = (f[:, 0, 0] + f[:, 0, 1] + f[:, 1, 0] + f[:, 1, 1] +
               0.50 * (f[:, 0, 2] + f[:, 1, 2] + f[:, 2, 0] + f[:, 2, 1]) + 0.25 * f[:, 2, 2]) / f[:, 1, 1]
    w[:, 1] = (f[:, 0, 3] + f[:, 0, 4] + f[:, 1, 3] + f[:, 1, 4] +
               0.50 * (f[:, 0, 2] + f[:, 1, 2] + f[:, 2, 3] + f[:, 2, 4]) + 0.25 * f[:, 2, 2]) / f[:, 1, 3]
    w[:, 2] = (f[:, 3, 0] + f[:, 3, 1] + f[:, 4, 0] + f[:, 4, 1] +
               0.50 * (f[:, 2, 0] + f[:, 2, 1] + f[:, 3, 2] + f[:, 4, 2]) + 0.25 * f[:, 2, 2]) / f[:, 3, 1]
    w[:, 3] = (f[:, 3, 3] + f[:, 3, 4] + f[:, 4, 3] + f[:, 4, 4] +
               0.50 * (f[:, 2, 3] + f[:, 2, 4] + f[:, 3, 2] + f[:, 4, 2]) + 0.25 * f[:, 2, 2]) / f[:, 3, 3]
    return w


def cg4_correct(kp, mu, qkappa, qmu, wcg4, sls):
    """AttBuilder::createAttenuation, CG4 branch (AttBuilder.cpp:140-166), on arrays of
    shape (ne, nslice, 25): returns unrelaxed kp, mu and (ne, nslice, 4) dkappa4, dmu4
    already weighted by the CG4 weights."""
    kna, kd, kat = att_factors(np.broadcast_to(qkappa, kp.shape), sls)
    mna, md, mat = att_factors(np.broadcast_to(qmu, mu.shape), sls)
    dkp, dmu = kd * kp, md * mu
    dlm = dkp - (2. / 3.) * dmu
    w = wcg4[:, None, :]
    dlm4 = w * dlm[:, :, CG4_POINTS]
    dmu4 = w * dmu[:, :, CG4_POINTS]
    kp2, mu2 = kp * kna, mu * mna
    kp2[:, :, CG4_POINTS] *= 1. + w * (kat[:, :, CG4_POINTS] / kna[:, :, CG4_POINTS] - 1.)
    mu2[:, :, CG4_POINTS] *= 1. + w * (mat[:, :, CG4_POINTS] / mna[:, :, CG4_POINTS] - 1.)
    return kp2, mu2, dlm4, dmu4


def default_sls(nsls=3, fmin=0.05, fmax=1.0):
    """SLS relaxation frequencies and weights as the mesher's attenuation_w_i / y_i."""
    w = 2 * np.pi * np.logspace(np.log10(fmin), np.log10(fmax), nsls)
    y = np.array([1.69, 1.12, 1.43, 1.2, 1.3, 1.1, 1.0, 1.0][:nsls])
    return {"w": w, "y": y, "fmin": fmin, "fmax": fmax, "fref": fmax}


# ------------------------------------------------------------------- sources ---
def moment_pattern_axial(mt, weights, nu_elem, axial_quad=True):
    """Mechanism::release, moment tensor on the axis (Mechanism.cpp:131-222).

    mt = (Mrr, Mtt, Mpp, Mrt, Mrp, Mtp) in the source frame; for an axial source
    Qzsp is the identity (Source::computeQzsp). Returns (nu, 6, 25) complex."""
    m = np.zeros((3, 3))
    m[0, 0], m[1, 1], m[2, 2] = mt[0], mt[1], mt[2]
    m[0, 1] = m[1, 0] = mt[3]
    m[0, 2] = m[2, 0] = mt[4]
    m[1, 2] = m[2, 1] = mt[5]
    mss, mpp, mzz = m[1, 1] * weights, m[2, 2] * weights, m[0, 0] * weights
    mpz, msz, msp = m[0, 2] * weights, m[0, 1] * weights, m[1, 2] * weights
    nu = min(nu_elem, 3)
    pat = np.zeros((nu, 6, 25), dtype=np.complex128)
    if axial_quad:
        ax = slice(0, 5)
        pat[0, 0, ax] = pat[0, 1, ax] = (mss[ax] + mpp[ax]) / 2.
        pat[0, 2, ax] = mzz[ax]
        if nu >= 2:
            pat[1, 4, ax] = (msz[ax] - 1j * mpz[ax]) / 2.
            pat[1, 3, ax] = 1j * pat[1, 4, ax]
        if nu >= 3:
            pat[2, 0, ax] = (mss[ax] - mpp[ax] - 2. * 1j * msp[ax]) / 4.
            pat[2, 1, ax] = -pat[2, 0, ax]
            pat[2, 5, ax] = 1j * pat[2, 0, ax]
        pat /= (2. * np.pi)
    return pat


def moment_pattern_offaxis(mt, weights, nu_elem, phi=0.0):
    """Mechanism::release, moment tensor off the axis in a non-axial quad (Qzsp = I)."""
    m = np.zeros((3, 3))
    m[0, 0], m[1, 1], m[2, 2] = mt[0], mt[1], mt[2]
    m[0, 1] = m[1, 0] = mt[3]
    m[0, 2] = m[2, 0] = mt[4]
    m[1, 2] = m[2, 1] = mt[5]
    comps = [m[1, 1], m[2, 2], m[0, 0], m[0, 2], m[0, 1], m[1, 2]]
    pat = np.zeros((nu_elem, 6, 25), dtype=np.complex128)
    for a in range(nu_elem):
        e = np.exp(1. * a * (-1j * phi))
        for d in range(6):
            pat[a, d] = e * comps[d] * weights
    return pat


# ------------------------------------------------------------- plain forward ---
def azimuthal_dt(sz, nr, vmax):
    """Stability bound of the azimuthal terms: the order-alpha stiffness grows like
    alpha v / s next to the axis, which Quad::computeDt (Quad.cpp:271-349) does not
    bound; min over off-axis points of s / ((nr // 2) v)."""
    s = np.asarray(sz)[..., 0, :]
    amax = max(1, int(nr) // 2)
    sp = s[s > 0]
    return float(np.min(sp) / (amax * vmax)) if sp.size else np.inf


def cartesian_model(nx=40, nz=40, width=100e3, height=100e3, nr=5, rho=2700.0, vp=5800.0,
                    vs=3460.0, source_depth=10e3, f0=1.0, nstations=20, courant=0.6, seed=0,
                    moment_scale=1e18, attenuation=None, record_interval=1, nr_aware_dt=False,
                    absorbing=False):
    """Plain forward case (the reference's CPU-runnable configuration).

    nr_aware_dt: also bound dt by the azimuthal terms next to the axis (azimuthal_dt);
    a uniform high nr on a fine axial mesh is unstable at the reference's dt."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h_s, h_z = width / nx, height / nz
    ne = nx * nz
    i = np.repeat(np.arange(nx), nz)
    j = np.tile(np.arange(nz), nx)
    s0, s1 = i * h_s, (i + 1) * h_s
    z0, z1 = -height + j * h_z, -height + (j + 1) * h_z
    nodal = np.stack([s0, z0, s1, z0, s1, z1, s0, z1], axis=1)
    axial = (i == 0).astype(np.uint8)
    geom, sz = geometry_batch(nodal, axial)
    pts, npts = structured_points(nx, nz)
    lam, mu = isotropic_moduli(rho, vp, vs)
    se_moduli = np.zeros((ne, 2, 25))
    se_moduli[:, 0, :] = lam
    se_moduli[:, 1, :] = mu
    mass = assemble_mass(pts, geom[:, 5, :], rho, npts)
    coords = np.zeros((npts, 2))
    coords[pts.ravel(), 0] = sz[:, 0, :].ravel()
    coords[pts.ravel(), 1] = sz[:, 1, :].ravel()
    sp_axial = (np.abs(coords[:, 0]) < 1e-9 * width).astype(np.uint8)
    # Quad::computeDt (Quad.cpp:329-345): quads on a Clayton boundary take half the step
    on_abc = (i == nx - 1) | (j == 0) if absorbing else np.zeros(ne, bool)
    dt_e = min(quad_dt(sz[e], vp) * (0.5 if on_abc[e] else 1.0) for e in range(ne))
    if nr_aware_dt:
        dt_e = min(dt_e, azimuthal_dt(sz, nr, vp))
    dt = round_dt(dt_e * courant)
    m = Model(dt=dt)
    m.sp_nr = np.full(npts, nr, np.int32)
    m.sp_mass = mass
    m.sp_axial = sp_axial
    m.sp_coords = coords
    m.se_nr = np.full(ne, nr, np.int32)
    m.se_pts = pts
    m.se_axial = axial
    m.se_geom = geom
    m.se_rheo = np.full(ne, L.AXG_ISO, np.int32)
    m.se_is3d = np.zeros(ne, np.uint8)
    m.se_mat_off = np.arange(ne, dtype=np.int64) * 50
    m.se_moduli = se_moduli.ravel()
    m.meta_rho = np.full((ne, 25), rho)
    if attenuation:
        sls = attenuation
        lam2, mu2, dl, dm = iso_with_attenuation(np.full((ne, 25), lam), np.full((ne, 25), mu),
                                                 sls["qkappa"], sls["qmu"], sls)
        se_moduli[:, 0, :], se_moduli[:, 1, :] = lam2, mu2
        m.se_moduli = se_moduli.ravel()
        m.se_att = np.full(ne, L.AXG_ATT_FULL, np.int32)
        am = np.stack([dl, dm], axis=1)
        m.se_att_off = np.arange(ne, dtype=np.int64) * 50
        m.se_att_moduli = am.ravel()
        a, b, g = att_alpha_beta_gamma(sls["w"], sls["y"], dt)
        m.nsls, m.att_alpha, m.att_beta, m.att_gamma = len(a), a, b, g
    # moment tensor on the axis at the given depth (Source::release)
    mt = rng.normal(0.0, moment_scale, 6)
    zsrc = -source_depth
    jsrc = int(min(nz - 1, max(0, math.floor((zsrc + height) / h_z - 1e-9))))
    esrc = 0 * nz + jsrc
    eta = 2.0 * (zsrc - z0[esrc]) / h_z - 1.0
    w = inplane_weights(-1.0, eta, True)
    pat = moment_pattern_axial(mt, w, nr // 2 + 1, True)
    hd = 1.0
    m.ms_elem = np.array([esrc], np.int32)
    m.ms_nu = np.array([pat.shape[0]], np.int32)
    m.ms_pat_off = np.array([0], np.int64)
    m.ms_pattern = pat.ravel()
    m.ms_stf = [STF(half_duration=hd, decay_factor=math.pi * f0 * hd, time_shift=0.0, derivative_order=2)]
    m.t0 = -2.5 * hd
    # receivers on the surface (z = 0), one azimuth
    st_e, st_w = [], []
    for k in range(1, nstations + 1):
        s = width * k / nstations
        ic = min(nx - 1, int(math.floor(s / h_s - 1e-9)))
        e = ic * nz + (nz - 1)
        xi = 2.0 * (s - s0[e]) / h_s - 1.0
        st_e.append(e)
        st_w.append(inplane_weights(xi, 1.0, bool(axial[e])))
    m.st_elem = np.array(st_e, np.int32)
    m.st_w = np.array(st_w)
    m.st_phi = np.zeros(nstations)
    m.st_interval = record_interval
    m.meta = {"workload": "cartesian %dx%d nr=%d" % (nx, nz, nr), "moment": mt.tolist(), "seed": seed}
    if absorbing:
        add_absorbing(m, nx, nz, width, height, rho, vp, vs)
    return m


def add_absorbing(m, nx, nz, width, height, rho=2700.0, vp=5800.0, vs=3460.0, sponge_frac=0.15,
                  sponge_gamma=None):
    """Clayton-Engquist 1-D coefficients on the outer (s = width) and bottom (z = -height)
    edges of a cartesian_model grid, and a Kosloff sponge whose gamma rises as cos^2 over the
    last sponge_frac of the domain (AbsorbingBoundary / ClaytonSolid1D / Sponge).

    area = GLL weight * half edge length * s (the axisymmetric line integral of the normal);
    theta = polar angle of the outward normal (pi/2 on the outer edge, pi at the bottom)."""
    wgll = np.array([0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1])
    h_s, h_z = width / nx, height / nz
    pts, _ = structured_points(nx, nz)
    # one dict per boundary key: normals of neighbouring elements add up per point
    right, bottom = {}, {}
    for e in range(nx * nz):
        i, j = divmod(e, nz)
        if i == nx - 1:
            for jp in range(5):
                p = int(pts[e, 4 * 5 + jp])
                right[p] = right.get(p, 0.0) + wgll[jp] * 0.5 * h_z * width
        if j == 0:
            for ip in range(5):
                p = int(pts[e, ip * 5 + 0])
                bottom[p] = bottom.get(p, 0.0) + wgll[ip] * 0.5 * h_s * max(m.sp_coords[p, 0], 0.0)
    cp = list(bottom) + list(right)
    area = list(bottom.values()) + list(right.values())
    theta = [math.pi] * len(bottom) + [math.pi / 2] * len(right)
    keep = [k for k in range(len(cp)) if area[k] > 0.0]
    n = len(keep)
    m.cl_solid = {"point": np.array([cp[k] for k in keep], np.int32), "rho_vp": np.full(n, rho * vp),
                  "rho_vs": np.full(n, rho * vs), "area": np.array([area[k] for k in keep]),
                  "theta": np.array([theta[k] for k in keep])}
    # sponge: distance into the layer along s and depth, normalised to [0, 1]
    span = sponge_frac * min(width, height)
    g0 = sponge_gamma if sponge_gamma is not None else 0.5 * vp / span
    ds = np.clip((m.sp_coords[:, 0] - (width - span)) / span, 0.0, 1.0)
    dz = np.clip(((-height + span) - m.sp_coords[:, 1]) / span, 0.0, 1.0)
    x = np.maximum(ds, dz)
    sel = np.nonzero(x > 0.0)[0].astype(np.int32)
    m.sponge_solid = (sel, g0 * np.sin(0.5 * math.pi * x[sel]) ** 2)
    return m


def add_ocean_load(m, nx, nz, width, rho_water=1020.0, depth_water=3000.0, tilt=0.0, seed=0):
    """MassOceanLoad1D on the surface points (z = 0) of a cartesian_model grid: ocean mass =
    rho_water * depth_water * area, area = GLL weight * half edge length * s (the
    axisymmetric line integral of the surface normal). The normal's polar angle is 0 (flat
    surface) plus, with tilt > 0, a seeded random angle in [0, tilt] per point, which makes
    the s-z coupling of the ocean-loaded mass non-zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    wgll = np.array([0.1, 49.0 / 90.0, 32.0 / 45.0, 49.0 / 90.0, 0.1])
    h_s = width / nx
    pts, _ = structured_points(nx, nz)
    area = {}
    for i in range(nx):
        e = i * nz + (nz - 1)
        for ip in range(5):
            p = int(pts[e, ip * 5 + 4])
            area[p] = area.get(p, 0.0) + wgll[ip] * 0.5 * h_s * max(m.sp_coords[p, 0], 0.0)
    keep = sorted(p for p in area if area[p] > 0.0)
    mo = np.array([rho_water * depth_water * area[p] for p in keep])
    th = rng.uniform(0.0, tilt, len(keep)) if tilt > 0 else np.zeros(len(keep))
    m.ocean_load = (np.array(keep, np.int32), mo, th)
    return m


def add_absorbing3d(m, rho=3300.0, vp=8000.0, vs=4500.0, pert=0.05, sponge_width=0.02, seed=0):
    """3-D absorbing boundaries on the outer surface of a spherical shell (points at the
    largest radius): ClaytonSolid3D conditions with rho vp and rho vs varying by +-pert over
    the nr slices of each point and a radial normal tilted towards phi by a small seeded
    angle per slice; and 3-D sponges (nr gammas, seeded variation over the slices) on the
    points within sponge_width of the outer radius. Synthetic: for parity of the 3-D
    boundary terms, not a calibrated absorbing layer."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r = np.hypot(m.sp_coords[:, 0], m.sp_coords[:, 1])
    rmax = r.max()
    surf = np.nonzero(r > rmax * (1 - 1e-9))[0].astype(np.int32)
    nr = np.asarray(m.sp_nr)
    off, rvp, rvs, area, nrm = [], [], [], [], []
    o = 0
    for p in surf:
        n = int(nr[p])
        off.append(o)
        o += n
        k = np.arange(n)
        wobble = 1.0 + pert * np.sin(2 * np.pi * k / n + rng.uniform(0, 2 * np.pi))
        rvp.append(rho * vp * wobble)
        rvs.append(rho * vs * wobble)
        area.append(np.full(n, 1e6 * (1.0 + m.sp_coords[p, 0] / rmax)))
        th = math.atan2(m.sp_coords[p, 0], m.sp_coords[p, 1])
        tilt = rng.uniform(-0.1, 0.1, n)
        v = np.stack([np.sin(th) * np.cos(tilt), np.sin(tilt), np.cos(th) * np.cos(tilt)], axis=1)
        nrm.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    m.cl3_solid = {"point": surf, "offset": np.array(off, np.int64), "rho_vp": np.concatenate(rvp),
                   "rho_vs": np.concatenate(rvs), "area": np.concatenate(area), "normal": np.concatenate(nrm)}
    near = np.nonzero(r > rmax * (1 - sponge_width))[0].astype(np.int32)
    goff, g = [], []
    o = 0
    for p in near:
        n = int(nr[p])
        goff.append(o)
        o += n
        x = (r[p] - rmax * (1 - sponge_width)) / (rmax * sponge_width)
        g.append(0.05 * x * (1.0 + 0.2 * rng.uniform(-1, 1, n)))
    m.sponge3d_solid = (near, np.array(goff, np.int64), np.concatenate(g))
    return m


def add_ocean_load3d(m, nx, nz, width, rho_water=1020.0, depth_water=3000.0, amp=0.2, tilt=0.2, seed=0):
    """MassOceanLoad3D on the surface points of a cartesian_model grid: the water depth varies
    by +-amp over the nr slices of each point (a seeded phase), and the unit normal tilts by a
    seeded angle of up to `tilt` towards s and phi per slice; area as in add_ocean_load."""
    rng = np.random.Generator(np.random.PCG64(seed))
    add_ocean_load(m, nx, nz, width, rho_water, depth_water)
    pts, mo1, _ = m.ocean_load
    m.ocean_load = None
    nr = np.asarray(m.sp_nr)
    off, mo, nrm = [], [], []
    o = 0
    for p, m0 in zip(pts, mo1):
        n = int(nr[p])
        off.append(o)
        o += n
        k = np.arange(n)
        mo.append(m0 * (1.0 + amp * np.sin(2 * np.pi * k / n + rng.uniform(0, 2 * np.pi))))
        a, b = rng.uniform(-tilt, tilt, n), rng.uniform(-tilt, tilt, n)
        v = np.stack([np.sin(a), np.sin(b), np.cos(a) * np.cos(b)], axis=1)
        nrm.append(v / np.linalg.norm(v, axis=1, keepdims=True))
    m.ocean_load3d = (np.asarray(pts, np.int32), np.array(off, np.int64), np.concatenate(mo), np.concatenate(nrm))
    return m


def add_prt_fluid(m, amp=0.05, three_d=False, seed=0, rtz=True):
    """add_prt's synthetic factors on every fluid element (3-D factors need 3-D fluid
    elements); with rtz, the polar angle of each element point (fe_theta of a spherical
    model) selects the RTZ frame."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ne = len(m.fe_nr)
    off, x3, xs = [], [], []
    o = 0
    for e in range(ne):
        ns = int(m.fe_nr[e]) if three_d else 1
        X0 = 1.0 + amp * rng.uniform(-1, 1, (ns, 25))
        X1 = amp * rng.uniform(-1, 1, (ns, 25))
        X2 = amp * rng.uniform(-1, 1, (ns, 25))
        X3 = 1.0 + amp * rng.uniform(-1, 1, (ns, 25))
        off.append(o)
        x3.append(1 if three_d else 0)
        xs.append(np.stack([X0, X1, X2, X3, 1.0 / (X0 * X3)]).ravel())
        o += 5 * ns * 25
    th = np.asarray(m.fe_theta) if rtz else None
    m.prt_fluid = {"element": np.arange(ne, dtype=np.int32), "offset": np.array(off, np.int64),
                   "is3d_prt": np.array(x3, np.uint8), "x": np.concatenate(xs), "theta": th}
    return m


def add_prt(m, elements=None, amp=0.05, three_d=False, seed=0):
    """Particle-relabelling factors on `elements` (default: every solid element): J^-1
    components X0 = 1 + a, X1 = b, X2 = c, X3 = 1 + d and |J| = 1 / (X0 X3), with a, b, c, d
    seeded and of size `amp` per point (and per slice with three_d, which needs 3-D
    elements). Synthetic: a smooth near-identity relabelling for parity of the PRT path."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ne = m.n_solid_elements
    el = np.arange(ne, dtype=np.int32) if elements is None else np.asarray(elements, np.int32)
    off, x3, xs = [], [], []
    o = 0
    for e in el:
        ns = int(m.se_nr[e]) if three_d else 1
        X0 = 1.0 + amp * rng.uniform(-1, 1, (ns, 25))
        X1 = amp * rng.uniform(-1, 1, (ns, 25))
        X2 = amp * rng.uniform(-1, 1, (ns, 25))
        X3 = 1.0 + amp * rng.uniform(-1, 1, (ns, 25))
        XJ = 1.0 / (X0 * X3)
        off.append(o)
        x3.append(1 if three_d else 0)
        xs.append(np.stack([X0, X1, X2, X3, XJ]).ravel())
        o += 5 * ns * 25
    m.prt = {"element": el, "offset": np.array(off, np.int64), "is3d_prt": np.array(x3, np.uint8),
             "x": np.concatenate(xs)}
    return m


def with_mass3d(m, amp=0.05, seed=0, exclude=()):
    """A copy of `m` whose solid points with nr >= 2 (except `exclude`) carry 3-D masses
    (Mass3D): the point's mass times (1 + amp * U(-1, 1)) per slice, seeded."""
    import copy
    rng = np.random.Generator(np.random.PCG64(seed))
    out = copy.copy(m)
    ex = set(int(p) for p in exclude)
    nr = np.asarray(m.sp_nr)
    mass = np.asarray(m.sp_mass, dtype=np.float64)
    mnr = np.ones(len(nr), np.int32)
    moff = np.zeros(len(nr), np.int64)
    vals = []
    o = 0
    for p in range(len(nr)):
        moff[p] = o
        if nr[p] >= 2 and p not in ex:
            mnr[p] = nr[p]
            vals.append(mass[p] * (1.0 + amp * rng.uniform(-1.0, 1.0, nr[p])))
            o += nr[p]
        else:
            vals.append(mass[p:p + 1])
            o += 1
    out.sp_mass_nr = mnr
    out.sp_mass_off = moff
    out.sp_mass = np.concatenate(vals)
    return out


# ---------------------------------------------------------- microbenchmark ---
def microbench_model(n_elem=200000, nr_max=64, seed=1, rheology="tiso", attenuation="full",
                     is3d=True, nsls=3, aspect=1.25, s_offset=1.0e6, h=2.0e3, axial_column=False,
                     nr_min=1, nr_choices=None):
    """Stiffness microbenchmark: non-axial structured quads with perturbed nodes,
    per-element nr log-uniform on [1, nr_max] (points take the minimum over their
    elements, so each element's nr is the maximum over its points). nr_choices: draw each
    element's nr uniformly from this list instead."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nz = max(1, int(round(math.sqrt(n_elem / aspect))))
    nx = max(1, int(math.ceil(n_elem / nz)))
    ne = nx * nz
    # perturbed node grid
    gs = np.arange(nx + 1) * h + s_offset
    gz = np.arange(nz + 1) * h - nz * h
    S, Z = np.meshgrid(gs, gz, indexing="ij")
    if axial_column:
        gs = gs - s_offset
        S, Z = np.meshgrid(gs, gz, indexing="ij")
    dS = rng.uniform(-0.1, 0.1, S.shape) * h
    if axial_column:
        dS[0, :] = 0.0
    S = S + dS
    Z = Z + rng.uniform(-0.1, 0.1, Z.shape) * h
    i = np.repeat(np.arange(nx), nz)
    j = np.tile(np.arange(nz), nx)
    nodal = np.stack([S[i, j], Z[i, j], S[i + 1, j], Z[i + 1, j], S[i + 1, j + 1], Z[i + 1, j + 1],
                      S[i, j + 1], Z[i, j + 1]], axis=1)
    axial = ((i == 0) & axial_column).astype(np.uint8)
    geom, sz = geometry_batch(nodal, axial)
    pts, npts = structured_points(nx, nz)
    # nr: log-uniform per element; points take the minimum over their elements
    enr = np.clip(np.rint(np.exp(rng.uniform(math.log(nr_min), math.log(nr_max), ne))),
                  nr_min, nr_max).astype(np.int32)
    if nr_choices is not None:
        enr = rng.choice(np.asarray(nr_choices, np.int32), ne)
        nr_max = int(np.max(nr_choices))
    pnr = np.full(npts, nr_max + 1, np.int32)
    np.minimum.at(pnr, pts.ravel(), np.repeat(enr, 25))
    enr = np.max(pnr[pts], axis=1).astype(np.int32)
    rho, vp, vs = 3300.0, 8000.0, 4500.0
    nsl = enr if is3d else np.ones(ne, np.int32)
    m = Model(dt=1.0)
    sls = default_sls(nsls)
    if rheology == "tiso":
        nmod = 5
    elif rheology == "iso":
        nmod = 2
    else:
        nmod = 21
    mat_off = np.zeros(ne, np.int64)
    att_off = np.zeros(ne, np.int64)
    sizes = nmod * nsl * 25
    mat_off[1:] = np.cumsum(sizes)[:-1]
    moduli = np.empty(int(np.sum(sizes)))
    npa = 4 if attenuation == "cg4" else 25
    att_mod = np.empty(int(np.sum(2 * nsl * npa))) if attenuation else None
    if attenuation:
        att_off[1:] = np.cumsum(2 * nsl * npa)[:-1]
    qmu = rng.uniform(80.0, 600.0, ne)
    A0, C0, L0 = rho * vp ** 2, rho * vp ** 2, rho * vs ** 2
    F0, N0 = A0 - 2 * L0, L0
    lam0, mu0 = isotropic_moduli(rho, vp, vs)
    tot = int(np.sum(nsl)) * 25
    # per (element, slice, point) perturbations, drawn in one batch
    elem_of = np.repeat(np.arange(ne), nsl * 25)
    if attenuation == "cg4":
        if not np.all(nsl == nsl[0]):
            raise ValueError("the CG4 workload uses one nr for all elements")
        wcg4 = weights_cg4(geom[:, 5, :])
    if rheology == "tiso":
        pert = 1.0 + rng.uniform(-0.1, 0.1, (5, tot))
        A, C, F, Lm, N = A0 * pert[0], C0 * pert[1], F0 * pert[2], L0 * pert[3], N0 * pert[4]
        if attenuation == "full":
            A, C, F, Lm, N, dl, dm = tiso_with_attenuation(A, C, F, Lm, N, 57823.0, qmu[elem_of], sls)
        elif attenuation == "cg4":
            shp = (ne, nsl[0], 25)
            A, C, F, Lm, N = [x.reshape(shp) for x in (A, C, F, Lm, N)]
            kp = (A * 4. + C + F * 4. - N * 4.) / 9.
            mu = (A + C - F * 2. + Lm * 6. + N * 5.) / 15.
            kp2, mu2, dl4, dm4 = cg4_correct(kp, mu, 57823.0, qmu[:, None, None], wcg4, sls)
            A = A - (kp + 4. / 3. * mu) + (kp2 + 4. / 3. * mu2)
            C = C - (kp + 4. / 3. * mu) + (kp2 + 4. / 3. * mu2)
            F = F - (kp - 2. / 3. * mu) + (kp2 - 2. / 3. * mu2)
            Lm = Lm - mu + mu2
            N = N - mu + mu2
            A, C, F, Lm, N = [x.ravel() for x in (A, C, F, Lm, N)]
        mods = [A, C, F, Lm, N]
    elif rheology == "iso":
        pert = 1.0 + rng.uniform(-0.1, 0.1, (2, tot))
        lam, mu = lam0 * pert[0], mu0 * pert[1]
        if attenuation == "full":
            lam, mu, dl, dm = iso_with_attenuation(lam, mu, 57823.0, qmu[elem_of], sls)
        elif attenuation == "cg4":
            shp = (ne, nsl[0], 25)
            lam, mu = lam.reshape(shp), mu.reshape(shp)
            kp = lam + (2. / 3.) * mu
            kp2, mu2, dl4, dm4 = cg4_correct(kp, mu, 57823.0, qmu[:, None, None], wcg4, sls)
            lam, mu = (kp2 - (2. / 3.) * mu2).ravel(), mu2.ravel()
        mods = [lam, mu]
    else:
        mods = aniso_moduli(rho, vp, vs, tot, rng)
        if attenuation:
            raise ValueError("anisotropic microbenchmark is built without attenuation")
    # scatter [element][slice][point] samples into [element][mod][slice][point]
    start = np.zeros(ne, np.int64)
    start[1:] = np.cumsum(nsl * 25)[:-1]
    local = np.arange(tot) - np.repeat(start, nsl * 25)
    for k, v in enumerate(mods):
        moduli[mat_off[elem_of] + k * (nsl[elem_of] * 25) + local] = v
    if attenuation == "full":
        att_mod[att_off[elem_of] + local] = dl
        att_mod[att_off[elem_of] + nsl[elem_of] * 25 + local] = dm
    elif attenuation == "cg4":
        half = nsl[0] * 4
        for e0 in range(ne):
            att_mod[att_off[e0]:att_off[e0] + half] = dl4[e0].ravel()
            att_mod[att_off[e0] + half:att_off[e0] + 2 * half] = dm4[e0].ravel()
    mass = assemble_mass(pts, geom[:, 5, :], rho, npts)
    vmax = vp * 1.1
    dt = round_dt(min(quad_dt(sz[e], vmax) for e in range(0, ne, max(1, ne // 2000))) * 0.6)
    m.dt = dt
    m.sp_nr = pnr
    m.sp_mass = mass
    coords = np.zeros((npts, 2))
    coords[pts.ravel(), 0] = sz[:, 0, :].ravel()
    coords[pts.ravel(), 1] = sz[:, 1, :].ravel()
    m.sp_coords = coords
    m.sp_axial = (np.abs(coords[:, 0]) < 1e-9 * h).astype(np.uint8) if axial_column else np.zeros(npts, np.uint8)
    m.se_nr = enr
    m.se_pts = pts
    m.se_axial = axial
    m.se_geom = geom
    m.se_rheo = np.full(ne, {"iso": L.AXG_ISO, "tiso": L.AXG_TISO, "aniso": L.AXG_ANISO}[rheology], np.int32)
    m.se_is3d = np.full(ne, 1 if is3d else 0, np.uint8)
    m.se_mat_off = mat_off
    m.se_moduli = moduli
    if attenuation:
        m.se_att = np.full(ne, L.AXG_ATT_FULL if attenuation == "full" else L.AXG_ATT_CG4, np.int32)
        m.se_att_off = att_off
        m.se_att_moduli = att_mod
        a, b, g = att_alpha_beta_gamma(sls["w"], sls["y"], dt)
        m.nsls, m.att_alpha, m.att_beta, m.att_gamma = len(a), a, b, g
    m.meta = {"workload": "microbench %d elements nr<=%d %s %s %s" %
              (ne, nr_max, rheology, "3D" if is3d else "1D", attenuation or "elastic"), "seed": seed}
    return m


def aniso_moduli(rho, vp, vs, n, rng, pert=0.05):
    """21 Cij: isotropic background plus a symmetric perturbation of relative size `pert`,
    kept positive definite; returns the 21 upper-triangle arrays (row-major)."""
    lam, mu = isotropic_moduli(rho, vp, vs)
    Ciso = np.zeros((6, 6))
    Ciso[:3, :3] = lam
    for k in range(3):
        Ciso[k, k] = lam + 2 * mu
        Ciso[3 + k, 3 + k] = mu
    R = rng.normal(0.0, 1.0, (n, 6, 6))
    R = 0.5 * (R + np.transpose(R, (0, 2, 1)))
    C = Ciso[None] + pert * (lam + 2 * mu) * R / 3.0
    iu = np.triu_indices(6)
    return [C[:, a, b] for a, b in zip(*iu)]


def blob_model(base, amp=0.05, fields=("mu", "rho"), center=None, radius=None, seed=0):
    """A copy of an isotropic 1-D Cartesian model with a seeded Gaussian blob of
    relative amplitude `amp` in mu and / or rho (the adjoint workload)."""
    import copy
    rng = np.random.Generator(np.random.PCG64(seed))
    m = copy.copy(base)
    ne = base.n_solid_elements
    coords = base.sp_coords[base.se_pts]                       # (ne, 25, 2)
    smax, zmin = coords[..., 0].max(), coords[..., 1].min()
    if center is None:
        center = (rng.uniform(0.3, 0.7) * smax, zmin * rng.uniform(0.3, 0.7))
    if radius is None:
        radius = 0.15 * smax
    d2 = (coords[..., 0] - center[0]) ** 2 + (coords[..., 1] - center[1]) ** 2
    blob = amp * np.exp(-d2 / (2 * radius ** 2))
    mods = base.se_moduli.reshape(ne, 2, 25).copy()
    lam, mu = mods[:, 0], mods[:, 1]
    rho = base.meta_rho.copy()
    if "mu" in fields:
        mu = mu * (1 + blob)
    if "rho" in fields:
        rho = rho * (1 + blob)
    m.se_moduli = np.stack([lam, mu], axis=1).ravel()
    m.meta_rho = rho
    m.sp_mass = assemble_mass(base.se_pts, base.se_geom[:, 5, :], rho, len(base.sp_nr))
    return m


def random_displacement(model, seed=2, solid=True):
    """Complex N(0,1)/(1+m) in mode m; mode 0 and Nyquist imaginary parts zero."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nr = np.asarray(model.sp_nr if solid else model.fp_nr)
    nu = nr // 2 + 1
    nd = 3 if solid else 1
    tot = int(np.sum(nu))
    mode = np.concatenate([np.arange(k) for k in nu]) if tot else np.zeros(0, int)
    u = (rng.normal(size=(tot, nd)) + 1j * rng.normal(size=(tot, nd))) / (1.0 + mode)[:, None]
    first = np.concatenate([[0], np.cumsum(nu)[:-1]]).astype(int)
    u[first, :] = u[first, :].real
    even = np.nonzero(nr % 2 == 0)[0]
    last = first[even] + nu[even] - 1
    u[last, :] = u[last, :].real
    return u.ravel()


# ------------------------------------------------------- spherical shell ---
def layered_background(seed=11, r_cmb=3480e3, r_fluid_top=3600e3, r_surface=6371e3, nlayers=6):
    """Seeded piecewise-linear 1-D table (radius -> rho, vp, vs): a fluid layer above
    the inner boundary, then `nlayers` solid layers whose end values are perturbed
    by 2 % around a smooth mantle-like trend."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rs = np.linspace(r_fluid_top, r_surface, nlayers + 1)
    x = (rs - r_fluid_top) / (r_surface - r_fluid_top)
    rho = (5.5e3 - 2.2e3 * x) * (1 + 0.02 * rng.uniform(-1, 1, x.size))
    vp = (13.7e3 - 5.7e3 * x) * (1 + 0.02 * rng.uniform(-1, 1, x.size))
    vs = (7.2e3 - 2.7e3 * x) * (1 + 0.02 * rng.uniform(-1, 1, x.size))
    fluid = {"r": np.array([r_cmb, r_fluid_top]), "rho": np.array([9.9e3, 9.9e3]),
             "vp": np.array([8.06e3, 8.0e3])}
    return {"solid": {"r": rs, "rho": rho, "vp": vp, "vs": vs}, "fluid": fluid}


def _interp(table, key, r):
    return np.interp(r, table["r"], table[key])


class GaussianField:
    """Isotropic Gaussian random field with Gaussian correlation of length L,
    by random Fourier features: f(x) = sigma sqrt(2/M) sum_m cos(k_m . x + p_m)."""

    def __init__(self, sigma, length, seed, nfeatures=24):
        rng = np.random.Generator(np.random.PCG64(seed))
        self.k = rng.normal(0.0, 1.0 / length, (nfeatures, 3))
        self.p = rng.uniform(0, 2 * np.pi, nfeatures)
        self.a = sigma * math.sqrt(2.0 / nfeatures)

    def __call__(self, x, y, z):
        # evaluated with torch's multi-threaded CPU kernels (the workloads sample the field at
        # up to ~1e9 (slice, point) positions), in float64
        import torch
        x, y, z = (torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)) for v in (x, y, z))
        shape = torch.broadcast_shapes(x.shape, y.shape, z.shape)
        out = torch.zeros(shape, dtype=torch.float64)
        for k, p in zip(self.k, self.p):
            t = x * float(k[0])
            t = t + y * float(k[1])
            t = t + z * float(k[2])
            out += torch.cos(t + float(p))
        return self.a * out.numpy()

    def ring_nr(self, s, z, nr_min, nr_max, energy=0.999, nsamp=512, chunk=4096):
        """The nr that resolves the field around the axis at each (s, z): the field sampled
        on the ring of radius s at height z (nsamp azimuths), its azimuthal power spectrum,
        and the smallest order M whose modes 1..M hold `energy` of the power above mode 0;
        nr = 2 M + 1, clipped to [nr_min, nr_max]."""
        s = np.asarray(s, np.float64).ravel()
        z = np.asarray(z, np.float64).ravel()
        phi = 2 * np.pi * np.arange(nsamp) / nsamp
        c, sn = np.cos(phi), np.sin(phi)
        out = np.empty(s.size, np.int32)
        for i0 in range(0, s.size, chunk):
            ss, zz = s[i0:i0 + chunk, None], z[i0:i0 + chunk, None]
            f = self(ss * c[None, :], ss * sn[None, :], zz)
            p = np.abs(np.fft.rfft(f, axis=1)[:, 1:]) ** 2
            cum = np.cumsum(p, axis=1)
            tot = np.maximum(cum[:, -1:], 1e-300)
            M = 1 + np.argmax(cum >= energy * tot, axis=1)
            out[i0:i0 + chunk] = np.clip(2 * M + 1, nr_min, nr_max)
        return out


def spherical_model(n_theta=96, n_solid_layers=24, n_fluid_layers=2, r_cmb=3480e3, r_fluid_top=3600e3,
                    r_surface=6371e3, nr_min=3, nr_max=128, dlnvs=0.02, corr_length=200e3, three_d=True,
                    q_mu=300.0, q_kappa=57823.0, attenuation="cg4", rheology="iso", period=20.0,
                    source_depth=100e3, nstations=20, courant=0.6, seed=12, nr_scale=1.0,
                    aniso_pert=0.05, record_interval=1, nr_from="field", nr_energy=0.99):
    """Half-annulus r in [r_cmb, r_surface], theta in [0, pi] (axis at both ends), with
    a fluid layer r in [r_cmb, r_fluid_top] (FluidElement, scalar potential) coupled to
    the solid above, spherical mapping, a seeded 1-D layered background and (three_d)
    a Gaussian random-field dlnVs sampled on each element's phi slices.
    Element nr (nr_from = "field"): the azimuthal bandwidth of the dlnVs field at the
    element centre -- the order that holds `nr_energy` of the field's power around the
    ring through that centre (GaussianField.ring_nr) -- clipped to [nr_min, nr_max] and
    rounded up to the reference's lucky numbers (7-smooth, or one factor 11 or 13);
    nr_from = "distance" takes nr = clip(round(nr_scale * pi s / L)) instead. Points take
    the minimum over their elements, and an element the maximum over its points.
    rheology 'aniso' carries 21 Cij: the isotropic background plus a seeded
    positive-definite perturbation of relative size aniso_pert."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bg = layered_background(seed, r_cmb, r_fluid_top, r_surface)
    r_edges = np.concatenate([np.linspace(r_cmb, r_fluid_top, n_fluid_layers + 1)[:-1],
                              np.linspace(r_fluid_top, r_surface, n_solid_layers + 1)])
    nl = n_fluid_layers + n_solid_layers
    t_edges = np.linspace(0.0, np.pi, n_theta + 1)
    nJ = 4 * nl + 1
    ne = n_theta * nl
    # element nodes; the south-axis column is rotated so that its axis edge is xi = -1
    nodal = np.zeros((ne, 8))
    axial = np.zeros(ne, np.uint8)
    pts = np.zeros((ne, 25), np.int64)
    ei = np.zeros(ne, np.int64)
    ej = np.zeros(ne, np.int64)
    ip = np.arange(5)
    for i in range(n_theta):
        for j in range(nl):
            e = i * nl + j
            ei[e], ej[e] = i, j
            t0_, t1_ = t_edges[i], t_edges[i + 1]
            r0_, r1_ = r_edges[j], r_edges[j + 1]
            sz = lambda t, r: (r * math.sin(t), r * math.cos(t))  # noqa: E731
            if i == n_theta - 1 and n_theta > 1:
                # nodes: (pi, r1) (t0, r1) (t0, r0) (pi, r0): curved outer = edge 0
                nodes = [sz(t1_, r1_), sz(t0_, r1_), sz(t0_, r0_), sz(t1_, r0_)]
                I = 4 * i + 4 - ip[:, None]
                J = 4 * j + 4 - ip[None, :]
                axial[e] = 1
            else:
                nodes = [sz(t0_, r0_), sz(t1_, r0_), sz(t1_, r1_), sz(t0_, r1_)]
                I = 4 * i + ip[:, None]
                J = 4 * j + ip[None, :]
                axial[e] = 1 if i == 0 else 0
            nodal[e] = np.array(nodes).ravel()
            pts[e] = (I * nJ + J).ravel()
    nodal[:, 0::2] = np.where(np.abs(nodal[:, 0::2]) < 1e-6, 0.0, nodal[:, 0::2])
    geom, szp = geometry_batch(nodal, axial, L.AXG_MAP_SPHERICAL)
    fluid_e = ej < n_fluid_layers
    # split global GLL points into solid and fluid sets
    gmax = (4 * n_theta + 1) * nJ
    sid = -np.ones(gmax, np.int64)
    fid = -np.ones(gmax, np.int64)
    sp_used = np.unique(pts[~fluid_e].ravel())
    fp_used = np.unique(pts[fluid_e].ravel())
    sid[sp_used] = np.arange(len(sp_used))
    fid[fp_used] = np.arange(len(fp_used))
    coords = np.zeros((gmax, 2))
    coords[pts.ravel(), 0] = szp[:, 0, :].ravel()
    coords[pts.ravel(), 1] = szp[:, 1, :].ravel()
    coords[:, 0] = np.where(np.abs(coords[:, 0]) < 1e-6, 0.0, coords[:, 0])
    field = GaussianField(dlnvs, corr_length, seed + 1)
    sc = np.mean(szp[:, 0, :], axis=1)
    if nr_from == "field":
        # element nr from the azimuthal spectrum of the dlnVs field at the element centre,
        # rounded up to the reference's lucky numbers (NrField::nextLuckyNumber) within nr_max
        from .preloop import next_lucky
        enr = field.ring_nr(sc, np.mean(szp[:, 1, :], axis=1), nr_min, nr_max, nr_energy)
        lucky = np.array([0] + [next_lucky(n) for n in range(1, nr_max + 1)])
        enr = np.where(lucky[enr] <= nr_max, lucky[enr], enr).astype(np.int32)
    else:
        # element nr from the distance to the axis
        enr = np.clip(np.rint(nr_scale * np.pi * sc / corr_length), nr_min, nr_max).astype(np.int32)
    pnr = np.full(gmax, nr_max + 1, np.int64)
    np.minimum.at(pnr, pts.ravel(), np.repeat(enr, 25))
    enr = np.max(pnr[pts], axis=1).astype(np.int32)
    sel_s, sel_f = np.nonzero(~fluid_e)[0], np.nonzero(fluid_e)[0]
    sls = default_sls(3, fmin=1.0 / (4 * period), fmax=4.0 / period)
    m = Model(dt=1.0)
    # ---- solid elements: moduli per point (1-D) or per (slice, point) (3-D)
    nss = enr[sel_s] if three_d else np.ones(len(sel_s), np.int32)
    nmod = {"iso": 2, "aniso": 21}[rheology]
    mat_off = np.zeros(len(sel_s), np.int64)
    mat_off[1:] = np.cumsum(nmod * nss * 25)[:-1]
    moduli = np.zeros(int(np.sum(nmod * nss * 25)))
    npa = 4 if attenuation == "cg4" else 25
    att_off = np.zeros(len(sel_s), np.int64)
    att_off[1:] = np.cumsum(2 * nss * npa)[:-1]
    att_mod = np.zeros(int(np.sum(2 * nss * npa))) if attenuation else None
    wcg4 = weights_cg4(geom[sel_s, 5, :]) if attenuation == "cg4" else None
    # background at every solid GLL point
    s_all, z_all = szp[sel_s, 0, :], szp[sel_s, 1, :]
    r_all = np.hypot(s_all, z_all)
    rho_pt = _interp(bg["solid"], "rho", r_all)
    vp_pt = _interp(bg["solid"], "vp", r_all)
    vs_pt = _interp(bg["solid"], "vs", r_all)
    vmax = float(np.max(vp_pt)) if len(sel_s) else 0.0
    # elements with one slice count at a time, in chunks of about 2M (slice, point) values:
    # moduli of shape (chunk, ns, 25)
    groups = []
    for ns in np.unique(nss):
        kall = np.nonzero(nss == ns)[0]
        step = max(1, (1 << 21) // (int(ns) * 25))
        groups += [(int(ns), kall[i:i + step]) for i in range(0, len(kall), step)]
    for ns, ks in groups:
        if three_d:
            phi = 2 * np.pi * np.arange(ns) / ns
            sg = s_all[ks][:, None, :]
            vs = vs_pt[ks][:, None, :] * (1.0 + field(sg * np.cos(phi)[None, :, None],
                                                      sg * np.sin(phi)[None, :, None], z_all[ks][:, None, :]))
        else:
            vs = vs_pt[ks][:, None, :]
        vp = np.broadcast_to(vp_pt[ks][:, None, :], vs.shape)
        rho = np.broadcast_to(rho_pt[ks][:, None, :], vs.shape)
        lam, mu = isotropic_moduli(rho, vp, vs)
        blk = np.arange(ns * 25)[None, :]
        if rheology == "aniso":
            C = aniso_moduli_from(lam, mu, rng, aniso_pert)
            for c in range(21):
                moduli[mat_off[ks][:, None] + c * ns * 25 + blk] = C[c].reshape(len(ks), ns * 25)
            continue
        if attenuation == "full":
            lam, mu, dl, dm = iso_with_attenuation(lam, mu, q_kappa, q_mu, sls)
            att_mod[att_off[ks][:, None] + blk] = dl.reshape(len(ks), ns * 25)
            att_mod[att_off[ks][:, None] + ns * 25 + blk] = dm.reshape(len(ks), ns * 25)
        elif attenuation == "cg4":
            kp = lam + (2. / 3.) * mu
            kp2, mu2, dl4, dm4 = cg4_correct(kp, np.array(mu), q_kappa, q_mu, wcg4[ks], sls)
            lam, mu = kp2 - (2. / 3.) * mu2, mu2
            b4 = np.arange(ns * 4)[None, :]
            att_mod[att_off[ks][:, None] + b4] = dl4.reshape(len(ks), ns * 4)
            att_mod[att_off[ks][:, None] + ns * 4 + b4] = dm4.reshape(len(ks), ns * 4)
        moduli[mat_off[ks][:, None] + blk] = np.asarray(lam).reshape(len(ks), ns * 25)
        moduli[mat_off[ks][:, None] + ns * 25 + blk] = np.asarray(mu).reshape(len(ks), ns * 25)
    # ---- fluid elements: K = 1 / rho (Material::createAcoustic), 1-D
    K = np.zeros((len(sel_f), 25))
    fmass_pt = np.zeros((len(sel_f), 25))
    for k, e in enumerate(sel_f):
        r_ = np.hypot(szp[e, 0, :], szp[e, 1, :])
        rho = _interp(bg["fluid"], "rho", r_)
        vp = _interp(bg["fluid"], "vp", r_)
        vmax = max(vmax, float(np.max(vp)))
        K[k] = 1.0 / rho
        fmass_pt[k] = 1.0 / (rho * vp ** 2)          # Material::getMass, fluid branch
    # ---- masses
    nsp, nfp = len(sp_used), len(fp_used)
    smass = np.zeros(nsp)
    np.add.at(smass, sid[pts[sel_s]].ravel(), (rho_pt * geom[sel_s, 5, :]).ravel())
    fmass = np.zeros(nfp)
    np.add.at(fmass, fid[pts[sel_f]].ravel(), (fmass_pt * geom[sel_f, 5, :]).ravel())
    # ---- solid-fluid coupling on r = r_fluid_top (Quad::setupGLL, computeNormal)
    normal = np.zeros((gmax, 2))
    wt = tables()
    for e in np.concatenate([sel_s, sel_f]):
        fl = fluid_e[e]
        j = ej[e]
        on = (fl and j == n_fluid_layers - 1) or ((not fl) and j == n_fluid_layers)
        if not on:
            continue
        rotated = (ei[e] == n_theta - 1 and n_theta > 1)
        # local edge on the interface: fluid top (r1), solid bottom (r0)
        outer = fl
        if not rotated:
            edge = 2 if outer else 0
        else:
            edge = 0 if outer else 2
        ed_pts = {0: [0, 5, 10, 15, 20], 2: [24, 19, 14, 9, 4]}[edge]
        J = _jacobians(nodal[e], bool(axial[e]))
        for q in ed_pts:
            ipol, jpol = q // 5, q % 5
            Jq = J[q]
            if edge == 0:
                n = np.array([Jq[1, 0], -Jq[0, 0]])
            else:
                n = np.array([-Jq[1, 0], Jq[0, 0]])
            n = n * (wt["wGLJ"][ipol] if axial[e] else wt["wGLL"][ipol])
            s_ = szp[e, 0, q]
            if axial[e]:
                xi = wt["pGLJ"][ipol]
                n = n * (Jq[0, 0] if ipol == 0 else s_ / (1. + xi))
            else:
                n = n * s_
            normal[pts[e, q]] += (n / 2.) if fl else (-n / 2.)
    iface = np.intersect1d(sp_used, fp_used)
    # ---- time step (Quad::computeDt with the solid-fluid factor 0.9, rounded)
    dts = [quad_dt(szp[e], vmax) for e in range(ne)]
    dt = round_dt(min(dts) * 0.9 * courant)
    m.dt = dt
    m.sp_nr = pnr[sp_used].astype(np.int32)
    m.sp_mass = smass
    m.sp_axial = (coords[sp_used, 0] == 0.0).astype(np.uint8)
    m.sp_coords = coords[sp_used]
    m.fp_nr = pnr[fp_used].astype(np.int32)
    m.fp_mass = fmass
    m.fp_axial = (coords[fp_used, 0] == 0.0).astype(np.uint8)
    m.fp_coords = coords[fp_used]
    m.fp_surface = np.zeros(nfp, np.uint8)
    m.se_nr = enr[sel_s]
    m.se_pts = sid[pts[sel_s]].astype(np.int32)
    m.se_axial = axial[sel_s]
    m.se_geom = geom[sel_s]
    m.se_rheo = np.full(len(sel_s), L.AXG_ANISO if rheology == "aniso" else L.AXG_ISO, np.int32)
    m.se_rtz = np.full(len(sel_s), 1 if rheology == "aniso" else 0, np.uint8)
    th = np.arctan2(szp[sel_s, 0, :], szp[sel_s, 1, :])
    m.se_theta = th
    m.se_is3d = np.full(len(sel_s), 1 if three_d else 0, np.uint8)
    m.se_mat_off = mat_off
    m.se_moduli = moduli
    if attenuation and rheology != "aniso":
        m.se_att = np.full(len(sel_s), L.AXG_ATT_CG4 if attenuation == "cg4" else L.AXG_ATT_FULL, np.int32)
        m.se_att_off = att_off
        m.se_att_moduli = att_mod
        a, b, g = att_alpha_beta_gamma(sls["w"], sls["y"], dt)
        m.nsls, m.att_alpha, m.att_beta, m.att_gamma = len(a), a, b, g
    m.fe_nr = enr[sel_f]
    m.fe_pts = fid[pts[sel_f]].astype(np.int32)
    m.fe_theta = np.arctan2(szp[sel_f, 0, :], szp[sel_f, 1, :])
    m.fe_axial = axial[sel_f]
    m.fe_geom = geom[sel_f]
    m.fe_is3d = np.zeros(len(sel_f), np.uint8)
    m.fe_mat_off = np.arange(len(sel_f), dtype=np.int64) * 25
    m.fe_moduli = K.ravel()
    m.sf_solid = sid[iface].astype(np.int32)
    m.sf_fluid = fid[iface].astype(np.int32)
    m.sf_nsu = normal[iface, 0]
    m.sf_nzu = normal[iface, 1]
    m.sf_nsa = normal[iface, 0]
    m.sf_nza = normal[iface, 1]
    m.sf_mass_fluid = fmass[fid[iface]]
    # ---- moment tensor on the north axis at the given depth, Ricker of the given period
    mt = rng.normal(0.0, 1e20, 6)
    r_src = r_surface - source_depth
    jsrc = int(np.searchsorted(r_edges, r_src) - 1)
    esrc = 0 * nl + jsrc
    eta = 2.0 * (r_src - r_edges[jsrc]) / (r_edges[jsrc + 1] - r_edges[jsrc]) - 1.0
    k_src = int(np.nonzero(sel_s == esrc)[0][0])
    w = inplane_weights(-1.0, eta, True)
    pat = moment_pattern_axial(mt, w, int(enr[esrc]) // 2 + 1, True)
    hd = period / 2.0
    m.ms_elem = np.array([k_src], np.int32)
    m.ms_nu = np.array([pat.shape[0]], np.int32)
    m.ms_pat_off = np.array([0], np.int64)
    m.ms_pattern = pat.ravel()
    m.ms_stf = [STF(half_duration=hd, decay_factor=math.pi * hd / period, time_shift=0.0,
                    derivative_order=2)]
    m.t0 = -2.5 * hd
    # ---- stations on the surface at theta in (0, pi)
    st_e, st_w = [], []
    for kk in range(1, nstations + 1):
        t = np.pi * kk / (nstations + 1)
        i = min(n_theta - 2, int(t / (np.pi / n_theta))) if n_theta > 1 else 0
        e = i * nl + (nl - 1)
        xi = 2.0 * (t - t_edges[i]) / (t_edges[i + 1] - t_edges[i]) - 1.0
        st_e.append(int(np.nonzero(sel_s == e)[0][0]))
        st_w.append(inplane_weights(xi, 1.0, bool(axial[e])))
    m.st_elem = np.array(st_e, np.int32)
    m.st_w = np.array(st_w)
    m.st_phi = np.zeros(nstations)
    m.st_interval = record_interval
    m.meta = {"workload": "spherical shell %dx%d (%d fluid layers) nr %d..%d %s %s" %
              (n_theta, nl, n_fluid_layers, int(enr.min()), int(enr.max()), rheology,
               "3D" if three_d else "1D"), "seed": seed}
    return m


def _jacobians(nodal, axial):
    """Jacobian d(s,z)/d(xi,eta) at the 25 points by central differences of the
    spherical map (used for the solid-fluid normals)."""
    t = tables()
    xn = t["pGLJ"] if axial else t["pGLL"]
    out = np.zeros((25, 2, 2))
    eps = 1e-6
    for ip in range(5):
        for jp in range(5):
            xi, eta = xn[ip], t["pGLL"][jp]
            cols = []
            for dx, de in ((eps, 0.0), (0.0, eps)):
                a = _sph_map(nodal, xi + dx, eta + de)
                b = _sph_map(nodal, xi - dx, eta - de)
                cols.append((a - b) / (2 * eps))
            out[ip * 5 + jp] = np.array(cols).T
    return out


def _sph_map(nodal, xi, eta):
    """Point of the spherical map (MappingSpherical::mapping) at (xi, eta)."""
    n = np.asarray(nodal).reshape(4, 2)
    r = np.hypot(n[:, 0], n[:, 1])
    if abs(r[0] - r[1]) < 1e-6 * r.max() and abs(r[2] - r[3]) < 1e-6 * r.max():
        co = 2 if r[2] > r[0] else 0
    else:
        co = 3 if r[3] > r[1] else 1
    Q = {0: np.array([[-1., 0.], [0., -1.]]), 1: np.array([[0., -1.], [1., 0.]]),
         2: np.eye(2), 3: np.array([[0., 1.], [-1., 0.]])}[co]
    nq = n @ Q.T
    rr = np.hypot(nq[:, 0], nq[:, 1])
    th = np.pi / 2 - np.arctan2(nq[:, 1], nq[:, 0])
    xq, eq = Q @ np.array([xi, eta])
    c = lambda p: p % 4  # noqa: E731
    r0, r2 = rr[c(co - 2)], rr[c(co)]
    t0, t1, t2, t3 = th[c(co - 2)], th[c(co - 1)], th[c(co)], th[c(co + 1)]
    if t3 - t2 > np.pi:
        t2 += 2 * np.pi
    if t2 - t3 > np.pi:
        t3 += 2 * np.pi
    if t0 - t1 > np.pi:
        t1 += 2 * np.pi
    if t1 - t0 > np.pi:
        t0 += 2 * np.pi
    t01 = ((1 - xq) * t0 + (1 + xq) * t1) * .5
    t32 = ((1 - xq) * t3 + (1 + xq) * t2) * .5
    r0m, r2p = (1 - eq) * r0 * .5, (1 + eq) * r2 * .5
    sz = np.array([r0m * np.sin(t01) + r2p * np.sin(t32), r0m * np.cos(t01) + r2p * np.cos(t32)])
    return Q.T @ sz


def aniso_moduli_from(lam, mu, rng, pert):
    """21 Cij per (slice, point): the isotropic tensor of (lam, mu) plus a seeded
    symmetric perturbation P = pert mu R / 3, whose 21 upper-triangle entries are drawn
    independently, zero-mean and uniform, with variance 1 on the diagonal and 1/2 off it
    (the variances of (G + G^T) / 2 for a standard normal G), checked positive definite.
    Returns the 21 upper-triangle arrays (row-major), each of the shape of lam."""
    lam = np.asarray(lam, np.float64)
    mu = np.asarray(mu, np.float64)
    shp = lam.shape
    lf, mf = lam.ravel(), mu.ravel()
    iu = list(zip(*np.triu_indices(6)))
    R = rng.random((21, lf.size))
    R -= 0.5
    R *= 2.0 * math.sqrt(3.0)            # U(-sqrt 3, sqrt 3): variance 1
    off = np.array([a != b for a, b in iu])
    R[off] *= math.sqrt(0.5)
    scale = pert * mf / 3.0
    # |P|_F below the isotropic tensor's smallest eigenvalue (mu, the shear Voigt term)
    # proves C positive definite; only the rest take an eigenvalue check
    fro2 = np.sum(np.where(off[:, None], 2.0, 1.0) * R * R, axis=0) * scale * scale
    out = []
    for k, (a, b) in enumerate(iu):
        base = np.zeros_like(lf)
        if a < 3 and b < 3:
            base = lf + 2 * mf if a == b else lf.copy()
        elif a == b:
            base = mf.copy()
        out.append(base + scale * R[k])
    unsure = np.nonzero(fro2 >= mf * mf * (1.0 - 1e-12))[0]
    if unsure.size:
        C = np.zeros((unsure.size, 6, 6))
        for k, (a, b) in enumerate(iu):
            C[:, a, b] = C[:, b, a] = out[k][unsure]
        if np.min(np.linalg.eigvalsh(C)) <= 0:
            raise ValueError("perturbed Cij not positive definite")
    return [x.reshape(shp) for x in out]


def ensemble_model(base, nsrc=64, seed=21, periods=(10.0, 40.0), moment_scale=1e20):
    """Batched ensemble: `nsrc` independent moment-tensor sources on the mesh of
    `base`, one wavefield each, all advanced in the same launches. Sources sit at
    seeded random (element, xi, eta) in non-axial solid elements with seeded
    tensors (drawn directly in the element's s, phi, z frame, i.e. after the
    Qzsp rotation of Mechanism::release) and Ricker wavelets with periods uniform
    in `periods`."""
    import copy
    rng = np.random.Generator(np.random.PCG64(seed))
    m = copy.copy(base)
    t = tables()
    cand = np.nonzero(base.se_axial == 0)[0]
    elems = rng.choice(cand, size=nsrc, replace=len(cand) < nsrc)
    pats, offs, nus, stfs = [], [], [], []
    o = 0
    t0 = 0.0
    for i, e in enumerate(elems):
        xi, eta = rng.uniform(-1, 1, 2)
        w = np.outer(lagrange(t["pGLL"], xi), lagrange(t["pGLL"], eta)).ravel()
        nu = int(base.se_nr[e]) // 2 + 1
        pat = moment_pattern_offaxis(rng.normal(0.0, moment_scale, 6), w, nu, phi=rng.uniform(0, 2 * np.pi))
        pats.append(pat.ravel())
        offs.append(o)
        nus.append(nu)
        o += pat.size
        period = rng.uniform(*periods)
        hd = period / 2.0
        stfs.append(STF(half_duration=hd, decay_factor=math.pi * hd / period, time_shift=0.0,
                        derivative_order=2))
        t0 = min(t0, -2.5 * hd)
    m.ms_elem = elems.astype(np.int32)
    m.ms_nu = np.array(nus, np.int32)
    m.ms_pat_off = np.array(offs, np.int64)
    m.ms_pattern = np.concatenate(pats)
    m.ms_stf = stfs
    m.ms_wave = np.arange(nsrc, dtype=np.int32)
    m.nwave = nsrc
    m.t0 = t0
    m.meta = dict(base.meta, workload=base.meta.get("workload", "") + " x %d sources" % nsrc)
    return m


def single_source(ens, i):
    """The i-th source of an ensemble model as its own one-wavefield model."""
    import copy
    m = copy.copy(ens)
    nu = int(ens.ms_nu[i])
    o = int(ens.ms_pat_off[i])
    m.ms_elem = ens.ms_elem[i:i + 1].copy()
    m.ms_nu = ens.ms_nu[i:i + 1].copy()
    m.ms_pat_off = np.zeros(1, np.int64)
    m.ms_pattern = ens.ms_pattern[o:o + nu * 150].copy()
    m.ms_stf = [ens.ms_stf[i]]
    m.ms_wave = None
    m.nwave = 1
    return m
