"""Writes small Exodus meshes and input directories for the preloop tests.

The meshes follow the salvus-mesher layout that ExodusMesh.cpp reads (connect1, coordx/y,
ss_names / elem_ss<i> / side_ss<i>, name_elem_var / vals_elem_var<i>eb1, name_glo_var /
vals_glo_var, info_records, discontinuities, ellipticity) and are written as NetCDF-3 with
scipy, which the NetCDF library reads like the mesher's NetCDF-4 files. They are generated
at test time; nothing here reads the reference.

cartesian_box() describes the same box as axisem3d_b200.meshgen.cartesian_model with z shifted
up by `surface` (a Cartesian Exodus mesh carries its depth as z below the surface radius), so
the model the preloop builds from it can be compared with the one meshgen builds directly.
"""
import math
import os

import numpy as np


def _strings(nc, var, dim_n, dim_len, values, length):
    v = nc.createVariable(var, "c", (dim_n, dim_len))
    v[:] = np.array([list(s.ljust(length, "\0")[:length]) for s in values], "S1")


def write_exodus(path, nodes, quads, side_sets, elem_vars, glob_vars, records, discontinuities,
                 ellipticity=None, name_len=33):
    """nodes [n, 2] (s, z); quads [q, 4] 0-based; side_sets {name: (elems, sides)} 0-based;
    elem_vars {name: [q]}; glob_vars {name: value}; records ["key = value", ...]."""
    from scipy.io import netcdf_file
    nc = netcdf_file(path, "w", version=2)
    nq, nn = len(quads), len(nodes)
    nc.createDimension("len_string", name_len)
    nc.createDimension("len_name", name_len)
    nc.createDimension("len_line", 81)
    nc.createDimension("num_nodes", nn)
    nc.createDimension("num_elem", nq)
    nc.createDimension("num_el_blk", 1)
    nc.createDimension("num_el_in_blk1", nq)
    nc.createDimension("num_nod_per_el1", 4)
    nc.createDimension("num_dim", 2)
    c = nc.createVariable("connect1", "i", ("num_el_in_blk1", "num_nod_per_el1"))
    c[:] = np.asarray(quads, np.int32) + 1
    x = nc.createVariable("coordx", "d", ("num_nodes",))
    x[:] = nodes[:, 0]
    y = nc.createVariable("coordy", "d", ("num_nodes",))
    y[:] = nodes[:, 1]
    names = list(side_sets)
    nc.createDimension("num_side_sets", len(names))
    _strings(nc, "ss_names", "num_side_sets", "len_name", names, name_len)
    for i, name in enumerate(names):
        el, sd = side_sets[name]
        nc.createDimension("num_side_ss%d" % (i + 1), len(el))
        v = nc.createVariable("elem_ss%d" % (i + 1), "i", ("num_side_ss%d" % (i + 1),))
        v[:] = np.asarray(el, np.int32) + 1
        v = nc.createVariable("side_ss%d" % (i + 1), "i", ("num_side_ss%d" % (i + 1),))
        v[:] = np.asarray(sd, np.int32) + 1
    ev = list(elem_vars)
    nc.createDimension("num_elem_var", len(ev))
    nc.createDimension("time_step", 1)
    _strings(nc, "name_elem_var", "num_elem_var", "len_name", ev, name_len)
    for i, name in enumerate(ev):
        v = nc.createVariable("vals_elem_var%deb1" % (i + 1), "d", ("time_step", "num_el_in_blk1"))
        v[:] = np.asarray(elem_vars[name], np.float64)[None, :]
    gv = list(glob_vars)
    nc.createDimension("num_glo_var", len(gv))
    _strings(nc, "name_glo_var", "num_glo_var", "len_name", gv, name_len)
    v = nc.createVariable("vals_glo_var", "d", ("time_step", "num_glo_var"))
    v[:] = np.array([[glob_vars[k] for k in gv]])
    nc.createDimension("num_info", len(records))
    _strings(nc, "info_records", "num_info", "len_line", records, 81)
    nc.createDimension("num_disc", len(discontinuities))
    v = nc.createVariable("discontinuities", "d", ("num_disc",))
    v[:] = discontinuities
    if ellipticity is not None:
        e = np.asarray(ellipticity, np.float64)
        nc.createDimension("ellip_rows", 2)
        nc.createDimension("ellip_cols", e.shape[1])
        v = nc.createVariable("ellipticity", "d", ("ellip_rows", "ellip_cols"))
        v[:] = e
    nc.close()


def cartesian_box(nx, nz, width, height, rho, vp, vs, surface=6371e3, storage="element_nodes",
                  attenuation=None, minimum_period=1.0):
    """The quads of meshgen.cartesian_model (element e = i * nz + j) as an Exodus description."""
    gs = np.linspace(0.0, width, nx + 1)
    gz = surface - height + np.linspace(0.0, height, nz + 1)
    node = lambda i, j: i * (nz + 1) + j                          # noqa: E731
    nodes = np.array([[gs[i], gz[j]] for i in range(nx + 1) for j in range(nz + 1)])
    quads, left, right, bottom, top = [], [], [], [], []
    for i in range(nx):
        for j in range(nz):
            e = len(quads)
            quads.append([node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)])
            if i == 0:
                left.append(e)
            if i == nx - 1:
                right.append(e)
            if j == 0:
                bottom.append(e)
            if j == nz - 1:
                top.append(e)
    nq = len(quads)
    sides = {"x0": (left, [3] * len(left)), "x1": (right, [1] * len(right)),
             "y0": (bottom, [0] * len(bottom)), "y1": (top, [2] * len(top))}
    ev = {"element_type": np.ones(nq), "fluid": np.zeros(nq)}
    props = {"RHO": rho, "VP": vp, "VS": vs}
    gv = {"minimum_period": minimum_period, "radius": surface}
    if attenuation is not None:
        props["QMU"] = attenuation["qmu"]
        props["QKAPPA"] = attenuation["qkappa"]
        gv.update({"nr_lin_solids": len(attenuation["w"]), "f_min": attenuation["fmin"],
                   "f_max": attenuation["fmax"], "f_ref": attenuation["fref"]})
        for i, (w, y) in enumerate(zip(attenuation["w"], attenuation["y"])):
            gv["w_%d" % i] = w
            gv["y_%d" % i] = y
    for k, v in props.items():
        if storage == "element_nodes":
            for n in range(4):
                ev["%s_%d" % (k, n)] = np.full(nq, v)
        else:
            ev[k] = np.full(nq, v)
    return dict(nodes=nodes, quads=np.array(quads), side_sets=sides, elem_vars=ev, glob_vars=gv,
                records=["crdsys = cartesian", "model = fixture_box"],
                discontinuities=np.array([surface - height, surface]))


def spherical_shell(n_theta, r_edges, n_fluid, layers, storage="elements", attenuation=None,
                    minimum_period=20.0, discontinuities=None):
    """Half annulus theta in [0, pi] (the axis at both ends) between r_edges[0] and r_edges[-1],
    spherical quads (element_type 0); the first n_fluid layers are fluid. layers: per radial
    layer dict(RHO=, VP=, VS=[, QMU=, QKAPPA=]). The south axis column lists its nodes in the
    order of the other columns, so its axis edge is side 1 and the reader rotates it."""
    nl = len(r_edges) - 1
    t = np.linspace(0.0, np.pi, n_theta + 1)
    node = lambda i, j: i * (nl + 1) + j                          # noqa: E731
    nodes = np.array([[r_edges[j] * math.sin(t[i]), r_edges[j] * math.cos(t[i])]
                      for i in range(n_theta + 1) for j in range(nl + 1)])
    nodes[:, 0] = np.where(np.abs(nodes[:, 0]) < 1e-6, 0.0, nodes[:, 0])
    quads, ax_e, ax_s, bot, top, sf_e, sf_s = [], [], [], [], [], [], []
    for i in range(n_theta):
        for j in range(nl):
            e = len(quads)
            quads.append([node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)])
            if i == 0:
                ax_e.append(e)
                ax_s.append(3)
            if i == n_theta - 1:
                ax_e.append(e)
                ax_s.append(1)
            if j == 0:
                bot.append(e)
            if j == nl - 1:
                top.append(e)
            if n_fluid and j == n_fluid - 1:
                sf_e.append(e)
                sf_s.append(2)
            if n_fluid and j == n_fluid:
                sf_e.append(e)
                sf_s.append(0)
    nq = len(quads)
    sides = {"r0": (bot, [0] * len(bot)), "r1": (top, [2] * len(top)), "t0": (ax_e, ax_s)}
    if n_fluid:
        sides["solid_fluid_boundary"] = (sf_e, sf_s)
    lay = np.array([j for i in range(n_theta) for j in range(nl)])
    ev = {"element_type": np.zeros(nq), "fluid": (lay < n_fluid).astype(float)}
    keys = [k for k in layers[0] if attenuation is not None or k not in ("QMU", "QKAPPA")]
    for k in keys:
        vals = np.array([layers[j][k] for j in lay], np.float64)
        if storage == "element_nodes":
            for n in range(4):
                ev["%s_%d" % (k, n)] = vals
        else:
            ev[k] = vals
    gv = {"minimum_period": minimum_period, "radius": r_edges[-1]}
    if attenuation is not None:
        gv.update({"nr_lin_solids": len(attenuation["w"]), "f_min": attenuation["fmin"],
                   "f_max": attenuation["fmax"], "f_ref": attenuation["fref"]})
        for i, (w, y) in enumerate(zip(attenuation["w"], attenuation["y"])):
            gv["w_%d" % i] = w
            gv["y_%d" % i] = y
    discs = discontinuities if discontinuities is not None else [r_edges[0], r_edges[-1]]
    return dict(nodes=nodes, quads=np.array(quads), side_sets=sides, elem_vars=ev, glob_vars=gv,
                records=["crdsys = spherical", "model = fixture_shell"],
                discontinuities=np.array(discs, np.float64),
                ellipticity=np.array([[0.0, 1.0], [1.0, 1.0]]))


MODEL_YAML = """model1D:
    exodus_mesh: {mesh}
geodesy:
    lat_lon_north_pole_mesh: SOURCE
    flattening_on_surface: {flattening}
absorbing_boundary:
    boundaries: [{boundaries}]
    enable_Clayton_Enquist: {clayton}
    Kosloff_Kosloff:
        enable: {sponge}
        relative_spans: [{spans}]
        gamma_expr_solid: 1.1 / T0 * (VS / VP)^2 * exp(-0.04 * SPAN / (VP * T0))
        gamma_expr_fluid: 0.88 / T0 * exp(-0.04 * SPAN / (VP * T0))
attenuation: {attenuation}
list_of_3D_models: []
"""

NR_YAML = """type_Nr: CONSTANT
bound_Nr_by_inplane: {bound}
constant: {nr}
"""

SOURCE_YAML = """time_axis:
    record_length: {record_length}
    enforced_dt: NONE
    Courant_number: {courant}
    integrator: NEWMARK
list_of_sources:
    - the_source:
        location:
            latitude_longitude: [90., 0.]
            depth: {depth}
            ellipticity: false
            depth_below_solid_surface: true
            undulated_geometry: false
        mechanism:
            type: MOMENT_TENSOR
            data: [{mt}]
            unit: 1.
        source_time_function:
            class_name: GaussianSTF
            half_duration: {hdur}
            decay_factor: {decay}
            time_shift: 0.
            use_derivative_integral: {order}
"""

OUTPUT_YAML = """list_of_station_groups:
    - {group}:
        locations:
            station_file: STATIONS.txt
            horizontal_x1_x2: {horizontal}
            vertical_x3: DEPTH
            ellipticity: false
            depth_below_solid_surface: true
            undulated_geometry: false
        wavefields:
            coordinate_frame: {frame}
            medium: SOLID
            channels: [U]
        temporal:
            sampling_period: {period}
            time_window: FULL
        file_options:
            format: {fmt}
            buffer_size: 100
            flush: true
list_of_element_groups: []
"""

ADVANCED_YAML = """verbose:
    channel: STDOUT
    level: ESSENTIAL
    warnings: true
    loop_info_interval: 1000
    stability_interval: 1
develop:
    diagnose_preloop: false
    max_num_time_steps: {max_steps}
    time_limit_for_fftw_planning: 60.
    fftw_lucky_numbers: {lucky}
"""


def write_inputs(d, mesh_desc, nr=5, depth=10e3, mt=(1e18, 0, 0, 0, 0, 0), hdur=1.0, decay=math.pi,
                 order="RICKER", courant=0.6, record_length=1.0, stations=(), horizontal="DISTANCE_AZIMUTH",
                 frame="spz", period="DT", fmt="ASCII_STATION", attenuation="NONE", boundaries=(),
                 clayton=False, sponge=False, spans=(), max_steps=0, lucky=False, bound_nr=False,
                 flattening="SPHERE"):
    """A complete input directory: the mesh, the five inparam files and STATIONS.txt.
    stations: (name, network, x1, x2, depth) rows."""
    os.makedirs(d, exist_ok=True)
    write_exodus(os.path.join(d, "mesh.e"), **mesh_desc)
    files = {
        "model": MODEL_YAML.format(mesh="mesh.e", flattening=flattening, boundaries=", ".join(boundaries),
                                   clayton=str(clayton).lower(), sponge=str(sponge).lower(),
                                   spans=", ".join("%g" % s for s in spans) or ".05", attenuation=attenuation),
        "nr": NR_YAML.format(bound=str(bound_nr).lower(), nr=nr),
        "source": SOURCE_YAML.format(record_length=record_length, courant=courant, depth=depth,
                                     mt=", ".join("%.17g" % v for v in mt), hdur=hdur, decay="%.17g" % decay,
                                     order=order),
        "output": OUTPUT_YAML.format(group="receivers", horizontal=horizontal, frame=frame, period=period,
                                     fmt=fmt) if stations else "list_of_station_groups: []\n"
                                                                  "list_of_element_groups: []\n",
        "advanced": ADVANCED_YAML.format(max_steps=max_steps, lucky=str(lucky).lower()),
    }
    for k, v in files.items():
        with open(os.path.join(d, "inparam.%s.yaml" % k), "w") as f:
            f.write(v)
    with open(os.path.join(d, "STATIONS.txt"), "w") as f:
        f.write("# name network x1 x2 elevation depth\n")
        for name, net, x1, x2, dep in stations:
            f.write("%s %s %.17g %.17g 0.0 %.17g\n" % (name, net, x1, x2, dep))
    return d


def write_grid_v3d(path, coords, data, order):
    """A StructuredGridV3D NetCDF-3 file: coords {name: values} (in the model's coordinate
    order), data {name: array over the coords in that order}, stored with its axes permuted
    to `order` (names of the coords in file order)."""
    from scipy.io import netcdf_file
    nc = netcdf_file(path, "w", version=2)
    names = list(coords)
    for n in names:
        nc.createDimension(n, len(coords[n]))
        v = nc.createVariable(n, "d", (n,))
        v[:] = coords[n]
    perm = [names.index(n) for n in order]
    for k, a in data.items():
        v = nc.createVariable(k, "d", tuple(order))
        v[:] = np.transpose(np.asarray(a, np.float64), perm)
    nc.close()


def model3d_yaml(name, fname, horizontal, vertical, nc_vars, data_rank, props, length_unit="km",
                 angle_unit="degree", depth_solid="true", ellipticity="false", whole_element="false"):
    """One list_of_3D_models entry; props: (key, nc_var, factor, reference_kind) rows."""
    lines = ["    - %s:" % name, "        activated: true", "        class_name: StructuredGridV3D",
             "        nc_data_file: %s" % fname, "        coordinates:",
             "            horizontal: %s" % horizontal, "            vertical: %s" % vertical,
             "            ellipticity: %s" % ellipticity,
             "            depth_below_solid_surface: %s" % depth_solid,
             "            nc_variables: [%s]" % ", ".join(nc_vars),
             "            data_rank: [%s]" % ", ".join(str(r) for r in data_rank),
             "            length_unit: %s" % length_unit, "            angle_unit: %s" % angle_unit,
             "            undulated_geometry: false", "            whole_element_inplane: %s" % whole_element,
             "        properties:"]
    for key, var, factor, kind in props:
        lines += ["            - %s:" % key, "                nc_var: %s" % var,
                  "                factor: %r" % factor, "                reference_kind: %s" % kind]
    lines.append("        store_grid_only_on_leaders: true")
    return "\n".join(lines) + "\n"


def geometric_yaml(name, fname, horizontal, vertical, nc_vars, data_rank, var, interface, lo, hi, factor=1.0,
                   length_unit="m", angle_unit="radian", depth_solid="false", ellipticity="false"):
    """One StructuredGridG3D entry of list_of_3D_models (undulation map between lo and hi)."""
    return "\n".join([
        "    - %s:" % name, "        activated: true", "        class_name: StructuredGridG3D",
        "        nc_data_file: %s" % fname, "        coordinates:",
        "            horizontal: %s" % horizontal, "            vertical: %s" % vertical,
        "            ellipticity: %s" % ellipticity, "            depth_below_solid_surface: %s" % depth_solid,
        "            nc_variables: [%s]" % ", ".join(nc_vars),
        "            data_rank: [%s]" % ", ".join(str(r) for r in data_rank),
        "            length_unit: %s" % length_unit, "            angle_unit: %s" % angle_unit,
        "        undulation_range:", "            interface: %r" % interface, "            min_max: [%r, %r]" % (lo, hi),
        "        undulation_data:", "            nc_var: %s" % var, "            factor: %r" % factor,
        "        store_grid_only_on_leaders: true"]) + "\n"


def ocean_yaml(name, fname, horizontal, nc_vars, data_rank, var, factor=1.0, length_unit="m",
               angle_unit="radian", ellipticity="false"):
    """One StructuredGridO3D entry of list_of_3D_models (sum of rho * depth)."""
    return "\n".join([
        "    - %s:" % name, "        activated: true", "        class_name: StructuredGridO3D",
        "        nc_data_file: %s" % fname, "        coordinates:",
        "            horizontal: %s" % horizontal, "            ellipticity: %s" % ellipticity,
        "            nc_variables: [%s]" % ", ".join(nc_vars),
        "            data_rank: [%s]" % ", ".join(str(r) for r in data_rank),
        "            length_unit: %s" % length_unit, "            angle_unit: %s" % angle_unit,
        "        data_sum_rho_depth:", "            nc_var: %s" % var, "            factor: %r" % factor,
        "        store_grid_only_on_leaders: true"]) + "\n"


def ellipticity_yaml(name):
    return "    - %s:\n        activated: true\n        class_name: Ellipticity\n" % name


def add_3d_models(d, entries):
    """Replace the empty list_of_3D_models of an input directory by the given entries."""
    p = os.path.join(d, "inparam.model.yaml")
    with open(p) as f:
        txt = f.read()
    with open(p, "w") as f:
        f.write(txt.replace("list_of_3D_models: []", "list_of_3D_models:\n" + "".join(entries)))


ELEMENT_GROUP_YAML = """    - {name}:
        elements:
            horizontal_range: [{hmin!r}, {hmax!r}]
            vertical_range: [{vmin!r}, {vmax!r}]
        inplane:
            edge_dimension: {edge_dim}
            edge_position: {edge_pos!r}
            GLL_points_one_edge: {gll}
        azimuthal:
            phi_list: [{phis}]
            lat_lon_list: [{latlon}]
            na_space: {na_space}
        wavefields:
            coordinate_frame: {frame}
            medium: SOLID
            channels: [{channels}]
        temporal:
            sampling_period: {period}
            time_window: {window}
        file_options:
            buffer_size: {buffer}
            flush: true
"""


def add_element_groups(d, groups):
    """Replace list_of_element_groups in d/inparam.output.yaml; groups: dicts with the keys of
    ELEMENT_GROUP_YAML (defaults: whole mesh, BOTH, FULL, Fourier, spz, [U], DT, FULL)."""
    base = dict(hmin=-1e30, hmax=1e30, vmin=-1e30, vmax=1e30, edge_dim="BOTH", edge_pos=0.0, gll="FULL",
                phis="", latlon="", na_space=1, frame="spz", channels="U", period="DT", window="FULL",
                buffer=100)
    txt = "list_of_element_groups:\n" + "".join(ELEMENT_GROUP_YAML.format(**dict(base, **g)) for g in groups)
    p = os.path.join(d, "inparam.output.yaml")
    with open(p) as f:
        cur = f.read()
    i = cur.index("list_of_element_groups:")
    with open(p, "w") as f:
        f.write(cur[:i] + txt)
