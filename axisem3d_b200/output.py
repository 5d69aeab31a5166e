"""Station output after the time loop: frame rotation, channels and the reference's three
file formats.

Rotation follows Station::rotateField (core/output/station-wise/station/Station.hpp:79-118)
with Station::rotate (Station.cpp): displacement is recorded in (s, phi, z); RTZ rotates
about the phi axis by the station's theta, ENZ further about the vertical by back azimuth +
90 degrees, xyz about the vertical by -phi; in Cartesian meshes spz already is RTZ.

Files follow StationIO_Ascii.cpp and StationIO_NetCDF.cpp under <output>/stations/<group>:
  ASCII_STATION  data_time.ascii, <network.name>.ascii (time x channel), list_channel.info
  ASCII_CHANNEL  data_time.ascii, dir_rank0/<channel>.ascii (time x station),
                 dir_rank0/list_station.info, rank_station.info
  NETCDF         axisem3d_synthetics.nc.rank0 with data_time, data_wave [station, channel,
                 time], list_channel, list_station (written as NetCDF-3, which the NetCDF
                 library reads like NetCDF-4)
Numbers are written with 16 significant digits for time and 8 (FP32 / mixed) or 16 (FP64)
for the wavefield, in blocks of buffer_size lines with right-aligned columns.
"""
from __future__ import annotations

import math
import os

import numpy as np


def _rotate(V, k, angle):
    """Station::rotate for 3-vectors (V: [..., 3]) about axis k."""
    i = k - 2 if k + 1 > 2 else k + 1
    j = k - 1 if k + 2 > 2 else k + 2
    c, s = np.cos(angle), np.sin(angle)
    vi = V[..., i].copy()
    V[..., i] = vi * c + V[..., j] * s
    V[..., j] = -vi * s + V[..., j] * c


def _rotate9(T, k, angle):
    """Station::rotate for 3 x 3 tensors stored as 9 (index 3 row + column): rows, then columns."""
    i = k - 2 if k + 1 > 2 else k + 1
    j = k - 1 if k + 2 > 2 else k + 2
    c, s = np.cos(angle), np.sin(angle)
    for n in range(3):
        I, J = i * 3 + n, j * 3 + n
        ti = T[..., I].copy()
        T[..., I] = ti * c + T[..., J] * s
        T[..., J] = -ti * s + T[..., J] * c
    for p in range(3):
        I, J = p * 3 + i, p * 3 + j
        ti = T[..., I].copy()
        T[..., I] = ti * c + T[..., J] * s
        T[..., J] = -ti * s + T[..., J] * c


# Voigt (0 5 4 / 5 1 3 / 4 3 2) <-> 3 x 3 (Station::rotate for 6-component fields)
_V2T = (0, 5, 4, 5, 1, 3, 4, 3, 2)
_T2V = (0, 4, 8, 5, 2, 1)


def _rotate6(S, k, angle):
    T = S[..., list(_V2T)].copy()
    _rotate9(T, k, angle)
    S[...] = T[..., list(_T2V)]


def rotate_field(f, frame, theta, baz, phi, cartesian):
    """Station::rotateField for a field recorded in (s, phi, z): f [station, time, D] with D = 3
    (vectors), 6 (Voigt tensors) or 9 (full tensors); returns a new array in the frame."""
    f = np.array(f, dtype=np.float64, copy=True)
    rot = {3: _rotate, 6: _rotate6, 9: _rotate9}[f.shape[-1]]
    th = np.asarray(theta)[:, None]
    bz = (np.asarray(baz) + math.pi * .5)[:, None]
    ph = np.asarray(phi)[:, None]
    if cartesian:
        if frame == "ENZ":
            rot(f, 2, bz)
        elif frame == "xyz":
            rot(f, 2, -ph)
    else:
        if frame == "RTZ":
            rot(f, 1, th)
        elif frame == "ENZ":
            rot(f, 1, th)
            rot(f, 2, bz)
        elif frame == "xyz":
            rot(f, 2, -ph)
    return f


def rotate_displacement(u_spz, frame, theta, baz, phi, cartesian):
    """u_spz: [station, time, 3] -> the requested frame (a new array)."""
    return rotate_field(u_spz, frame, theta, baz, phi, cartesian)


def strain_from_gradient(g):
    """computeGrad6 from computeGrad9 (GradientQuadrature.hpp:177-232): Voigt strain with
    engineering shear, E = (G0, G4, G8, G5 + G7, G2 + G6, G1 + G3)."""
    return np.stack([g[..., 0], g[..., 4], g[..., 8], g[..., 5] + g[..., 7], g[..., 2] + g[..., 6],
                     g[..., 1] + g[..., 3]], axis=-1)


def curl_from_gradient(g):
    """SolidElement::getCurlField (SolidElement.cpp:525-533): (G7 - G5, G2 - G6, G3 - G1)."""
    return np.stack([g[..., 7] - g[..., 5], g[..., 2] - g[..., 6], g[..., 3] - g[..., 1]], axis=-1)


def channel_data(u, channels):
    """Displacement channels of u [station, time, 3], already in the output frame ->
    [station, channel, time]."""
    cols = []
    for ch in channels:
        if ch == "U_NORM":
            cols.append(np.sqrt(np.sum(u * u, axis=2)))
        else:
            cols.append(u[:, :, int(ch[1]) - 1])
    return np.stack(cols, axis=1)


def group_channels(u_spz, g_spz, channels, frame, theta, baz, phi, cartesian):
    """[station, channel, time] of one group from the (s, phi, z) displacement [station,
    time, 3] and gradient [station, time, 9] (None when no G / E / R channel is asked)."""
    need = {c[0] for c in channels}
    f = {}
    if "U" in need:
        f["U"] = rotate_field(u_spz, frame, theta, baz, phi, cartesian)
    if "G" in need:
        f["G"] = rotate_field(g_spz, frame, theta, baz, phi, cartesian)
    if "E" in need:
        e = strain_from_gradient(g_spz)
        e[..., 3:] *= .5
        e = rotate_field(e, frame, theta, baz, phi, cartesian)
        e[..., 3:] *= 2.
        f["E"] = e
    if "R" in need:
        f["R"] = rotate_field(curl_from_gradient(g_spz), frame, theta, baz, phi, cartesian)
    cols = []
    for ch in channels:
        x = f[ch[0]]
        if ch in ("U_NORM", "R_NORM"):
            cols.append(np.sqrt(np.sum(x * x, axis=2)))
        elif ch == "G_I1":
            cols.append(x[:, :, 0] + x[:, :, 4] + x[:, :, 8])
        elif ch == "E_I1":
            cols.append(x[:, :, 0] + x[:, :, 1] + x[:, :, 2])
        elif ch == "E_J2":
            i1 = x[:, :, 0] + x[:, :, 1] + x[:, :, 2]
            i2 = (x[:, :, 0] * x[:, :, 1] + x[:, :, 1] * x[:, :, 2] + x[:, :, 2] * x[:, :, 0] -
                  x[:, :, 3] ** 2 - x[:, :, 4] ** 2 - x[:, :, 5] ** 2)
            cols.append(i1 * i1 / 3. - i2)
        elif ch[0] == "G":
            cols.append(x[:, :, (int(ch[1]) - 1) * 3 + int(ch[2]) - 1])
        elif ch[0] == "E":
            cols.append(x[:, :, {"11": 0, "22": 1, "33": 2, "23": 3, "31": 4, "12": 5}[ch[1:]]])
        else:
            cols.append(x[:, :, int(ch[1]) - 1])
    return np.stack(cols, axis=1)


def _write_blocks(path, rows, precision, block):
    """Rows of numbers in blocks of `block` lines, each block right-aligned to its widest entry."""
    with open(path, "w") as f:
        for b0 in range(0, len(rows), block):
            chunk = rows[b0:b0 + block]
            txt = [["%.*g" % (precision, v) for v in r] for r in chunk]
            w = max((len(x) for r in txt for x in r), default=0)
            for r in txt:
                f.write(" ".join(x.rjust(w) for x in r) + "\n")


def write_group(out_dir, group, times, data, wave_precision):
    """Write one station group; data: [station, channel, time]."""
    gdir = os.path.join(out_dir, "stations", group.name)
    os.makedirs(gdir, exist_ok=True)
    block = max(1, int(group.buffer_size))
    if group.fmt == "NETCDF":
        from scipy.io import netcdf_file
        fname = os.path.join(gdir, "axisem3d_synthetics.nc.rank0")
        nc = netcdf_file(fname, "w", version=2)
        nst, nch, nt = data.shape
        nc.createDimension("dim_time", nt)
        nc.createDimension("dim_station", nst)
        nc.createDimension("dim_channel", nch)
        lc = max(len(c) for c in group.channels)
        ls = max(len(k) for k in group.keys)
        nc.createDimension("dim_channel_str_length", lc)
        nc.createDimension("dim_station_str_length", ls)
        v = nc.createVariable("data_time", "d", ("dim_time",))
        v[:] = times
        v = nc.createVariable("data_wave", "f" if wave_precision <= 8 else "d",
                              ("dim_station", "dim_channel", "dim_time"))
        v[:] = data
        v = nc.createVariable("list_channel", "c", ("dim_channel", "dim_channel_str_length"))
        v[:] = np.array([list(c.ljust(lc, "\0")) for c in group.channels], "S1")
        v = nc.createVariable("list_station", "c", ("dim_station", "dim_station_str_length"))
        v[:] = np.array([list(k.ljust(ls, "\0")) for k in group.keys], "S1")
        nc.close()
        return
    _write_blocks(os.path.join(gdir, "data_time.ascii"), [[t] for t in times], 16, block)
    if group.fmt == "ASCII_STATION":
        for k, key in enumerate(group.keys):
            _write_blocks(os.path.join(gdir, key + ".ascii"), data[k].T.tolist(), wave_precision, block)
        with open(os.path.join(gdir, "list_channel.info"), "w") as f:
            for ch in group.channels:
                f.write(ch + "\n")
    else:
        rdir = os.path.join(gdir, "dir_rank0")
        os.makedirs(rdir, exist_ok=True)
        for c, ch in enumerate(group.channels):
            _write_blocks(os.path.join(rdir, ch + ".ascii"), data[:, c, :].T.tolist(), wave_precision, block)
        with open(os.path.join(rdir, "list_station.info"), "w") as f:
            for key in group.keys:
                f.write(key + "\n")
        with open(os.path.join(gdir, "rank_station.info"), "w") as f:
            f.write("MPI_RANK STATION_KEY STATION_INDEX_IN_RANK\n")
            for k, key in enumerate(group.keys):
                f.write("0 %s %d\n" % (key, k))


def group_records(group, nsteps, t0, dt, engine_interval):
    """(time steps, engine record rows) of one group (StationOutput::release :329-345)."""
    steps = [t for t in range(0, nsteps, group.interval)
             if group.tmin <= t0 + t * dt <= group.tmax]
    rows = [t // engine_interval for t in steps]
    return np.array(steps, np.int64), np.array(rows, np.int64)


# ------------------------------------------------------------ element groups ---
# Element-wise output (core/output/element-wise): ElementOpSolid::record (ElementOpSolid.cpp:48-80)
# takes the element's Fourier coefficients at the chosen GLL points to the output frame,
# ElementOp::recordToElem (ElementOp.hpp:26-68) lays them out as real rows (Fourier: row 0 the
# real part of order 0, rows 2 alpha - 1 and 2 alpha the real and imaginary parts of order
# alpha, cut at na = nr; azimuths: the series summed at each phi, 2 exp(i alpha phi) for
# alpha > 0), and ElementOp::dumpToIO (ElementOp.hpp:70-176) forms the channels on those rows.


def _rotate_complex(f, theta, cartesian):
    """(s, phi, z) -> RTZ of complex coefficients f [point, order, D] (theta per point):
    CoordTransformSpherical::transformSPZ_RTZ3 / 9 / 6 applied to real and imaginary parts;
    identity in a Cartesian mesh (CoordTransformCartesian)."""
    if cartesian:
        return f
    zero = np.zeros(len(theta))
    re = rotate_field(f.real, "RTZ", theta, zero, zero, False)
    im = rotate_field(f.imag, "RTZ", theta, zero, zero, False)
    return re + 1j * im


def element_fields(u, g, need, frame, theta, cartesian):
    """Fields of one set of elements in the output frame from the complex coefficients of the
    displacement u [point, order, 3] and gradient g [point, order, 9] (either may be None):
    SolidElement::getDisplField / getNablaField / getStrainField / getCurlField
    (SolidElement.cpp:396-546, the branch without particle relabelling)."""
    rtz = frame == "RTZ"
    out = {}
    if "U" in need:
        out["U"] = _rotate_complex(u, theta, cartesian) if rtz else u
    if "G" in need:
        out["G"] = _rotate_complex(g, theta, cartesian) if rtz else g
    if "E" in need:
        e = strain_from_gradient(g)
        if rtz and not cartesian:
            e = e.copy()
            e[..., 3:] *= .5
            e = _rotate_complex(e, theta, cartesian)
            e[..., 3:] *= 2.
        out["E"] = e
    if "R" in need:
        r = curl_from_gradient(g)
        out["R"] = _rotate_complex(r, theta, cartesian) if rtz else r
    return out


def fourier_rows(c, na, phis):
    """ElementOp::recordToElem: complex coefficients c [..., order, D] -> real rows
    [..., na, D] (Fourier layout when phis is empty, else the series at each azimuth)."""
    nu = c.shape[-2]
    if len(phis) == 0:
        rows = np.empty(c.shape[:-2] + (2 * nu - 1, c.shape[-1]))
        rows[..., 0, :] = c[..., 0, :].real
        rows[..., 1::2, :] = c[..., 1:, :].real
        rows[..., 2::2, :] = c[..., 1:, :].imag
        return rows[..., :na, :]
    al = np.arange(nu)
    z = np.where(al == 0, 1.0, 2.0)[None, :] * np.exp(1j * np.outer(np.asarray(phis), al))   # [phi, order]
    return np.real(np.einsum("pa,...ad->...pd", z, c))


def element_channels(rows, channels):
    """ElementOp::dumpToIO on rows {field: [..., na, D]} -> [..., na, channel]. As in the
    reference's element output, G_I1 adds the first three gradient components and E_J2 takes
    I1^2 / 3 - (E11 E22 + E22 E33 + E33 E11) + (E23 E31 + E31 E12 + E12 E23)."""
    cols = []
    for ch in channels:
        x = rows[ch[0]]
        if ch in ("U_NORM", "R_NORM"):
            cols.append(np.sqrt(np.sum(x * x, axis=-1)))
        elif ch in ("G_I1", "E_I1"):
            cols.append(x[..., 0] + x[..., 1] + x[..., 2])
        elif ch == "E_J2":
            i1 = x[..., 0] + x[..., 1] + x[..., 2]
            cols.append(i1 * i1 / 3. - (x[..., 0] * x[..., 1] + x[..., 1] * x[..., 2] + x[..., 2] * x[..., 0]) +
                        (x[..., 3] * x[..., 4] + x[..., 4] * x[..., 5] + x[..., 5] * x[..., 3]))
        elif ch[0] == "G":
            cols.append(x[..., (int(ch[1]) - 1) * 3 + int(ch[2]) - 1])
        elif ch[0] == "E":
            cols.append(x[..., {"11": 0, "22": 1, "33": 2, "23": 3, "31": 4, "12": 5}[ch[1:]]])
        else:
            cols.append(x[..., int(ch[1]) - 1])
    return np.stack(cols, axis=-1)


class ElementGroupWriter:
    """ElementIO_NetCDF (core/output/element-wise/io/ElementIO_NetCDF.cpp:14-249): the file
    <output>/elements/<group>/axisem3d_synthetics.nc.rank0 with data_time [dim_time], one
    data_wave__NaG=<nag> [dim_element__NaG=<nag>, dim_na__NaG=<nag>, dim_GLL, dim_channel,
    dim_time] per na-grid value, list_channel, list_element__NaG=<nag> (element tags),
    list_na_grid, list_element_na [dim_element, 5] and list_element_coords [dim_element,
    dim_GLL, 2]. No file when the group has no element. Rows at and above an element's na in
    its na-grid block are zero."""

    def __init__(self, out_dir, group, wave_dtype):
        from .ncwrite import NC3File
        self.group = group
        self.line = 0
        self.nc = None
        ne = len(group.elems)
        if ne == 0:
            return
        gdir = os.path.join(out_dir, "elements", group.name)
        os.makedirs(gdir, exist_ok=True)
        nc = NC3File(os.path.join(gdir, "axisem3d_synthetics.nc.rank0"))
        nt, npnts, nch = group.nrec, group.npnts, len(group.channels)
        nc.add("data_time", [("dim_time", nt)], np.float64)
        self.members = []
        for nag in group.na_grid:
            sel = np.nonzero(group.elem_na[:, 2] == nag)[0]
            self.members.append(sel)
            s = "%d" % nag
            nc.add("data_wave__NaG=" + s, [("dim_element__NaG=" + s, len(sel)), ("dim_na__NaG=" + s, int(nag)),
                                            ("dim_GLL", npnts), ("dim_channel", nch), ("dim_time", nt)], wave_dtype)
        lc = max(len(c) for c in group.channels)
        nc.add("list_channel", [("dim_channel", nch), ("dim_channel_str_length", lc)], "S1")
        for nag, sel in zip(group.na_grid, self.members):
            s = "%d" % nag
            nc.add("list_element__NaG=" + s, [("dim_element__NaG=" + s, len(sel))], np.int32)
        nc.add("list_na_grid", [("dim_na_grid", len(group.na_grid))], np.int32)
        nc.add("list_element_na", [("dim_element", ne), ("dim_5", 5)], np.int32)
        nc.add("list_element_coords", [("dim_element", ne), ("dim_GLL", npnts), ("dim_2", 2)], np.float64)
        nc.create()
        nc.var("list_channel")[:] = np.array([list(c.ljust(lc, "\0")) for c in group.channels], "S1")
        for nag, sel in zip(group.na_grid, self.members):
            nc.var("list_element__NaG=%d" % nag)[:] = group.tags[sel]
        nc.var("list_na_grid")[:] = group.na_grid
        nc.var("list_element_na")[:] = group.elem_na
        nc.var("list_element_coords")[:] = group.coords
        nc.flush()
        self.nc = nc

    def write(self, times, data):
        """times [b]; data: per element [na, npnts, channel, b] (a list in group order)."""
        b = len(times)
        if self.nc is None or b == 0:
            return
        g = self.group
        t0 = self.line
        self.nc.var("data_time")[t0:t0 + b] = times
        for nag, sel in zip(g.na_grid, self.members):
            blk = np.zeros((len(sel), int(nag), g.npnts, len(g.channels), b))
            for i, k in enumerate(sel):
                na = int(g.na[k])
                blk[i, :na] = data[k]
            self.nc.var("data_wave__NaG=%d" % nag)[..., t0:t0 + b] = blk
        self.line += b
        if g.flush:
            self.nc.flush()

    def close(self):
        if self.nc is not None:
            self.nc.close()
            self.nc = None
