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
