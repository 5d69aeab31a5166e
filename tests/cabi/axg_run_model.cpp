// axg_run_model.cpp -- a C++ caller of the engine's C ABI that includes nothing of the project
// but include/axg.h and links libaxg.so: the way the reference's time loop (a C++ program) binds
// the drop-in. It reads a model dump (named arrays written by tests/test_cabi.py), builds the
// axg_* structs from it, runs the time loop through the ABI and writes the displacement field
// and the seismograms back as raw doubles.
//
//   axg_run_model <dump> <precision 0|1|2> <nsteps> <out prefix> [deterministic 0|1]
//
// Dump format: repeated records of [u32 name length][name][u8 type][u64 count][data], type
// 'd' = double, 'i' = int32, 'l' = int64, 'b' = uint8.
#include "axg.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

namespace {

struct Array {
    char type = 0;
    std::vector<unsigned char> bytes;
    template <class X> const X *as() const { return bytes.empty() ? nullptr : reinterpret_cast<const X *>(bytes.data()); }
    template <class X> size_t count() const { return bytes.size() / sizeof(X); }
};

std::map<std::string, Array> read_dump(const char *path) {
    std::map<std::string, Array> out;
    FILE *f = std::fopen(path, "rb");
    if (!f) { std::perror(path); std::exit(2); }
    for (;;) {
        uint32_t len;
        if (std::fread(&len, 4, 1, f) != 1) break;
        std::string name(len, '\0');
        uint8_t type;
        uint64_t n;
        if (std::fread(&name[0], 1, len, f) != len || std::fread(&type, 1, 1, f) != 1 || std::fread(&n, 8, 1, f) != 1) {
            std::fprintf(stderr, "truncated dump\n");
            std::exit(2);
        }
        const size_t w = type == 'd' || type == 'l' ? 8 : type == 'i' ? 4 : 1;
        Array a;
        a.type = (char)type;
        a.bytes.resize(n * w);
        if (n && std::fread(a.bytes.data(), w, n, f) != n) { std::fprintf(stderr, "truncated dump\n"); std::exit(2); }
        out[name] = std::move(a);
    }
    std::fclose(f);
    return out;
}

void check(axg_solver *h, int rc, const char *what) {
    if (rc != AXG_OK) {
        std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, axg_last_error(h));
        std::exit(1);
    }
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 5 && argc != 6) {
        std::fprintf(stderr, "usage: %s <dump> <precision> <nsteps> <out prefix> [deterministic]\n", argv[0]);
        return 2;
    }
    auto d = read_dump(argv[1]);
    auto get = [&](const char *k) -> const Array & {
        auto it = d.find(k);
        if (it == d.end()) { std::fprintf(stderr, "missing %s\n", k); std::exit(2); }
        return it->second;
    };

    axg_config cfg = {};
    cfg.precision = std::atoi(argv[2]);
    cfg.device = 0;
    cfg.dt = get("dt").as<double>()[0];
    cfg.t0 = get("t0").as<double>()[0];
    cfg.nsls = 0;
    cfg.compensated = 1;
    cfg.nwave = 1;
    cfg.deterministic = argc == 6 ? std::atoi(argv[5]) : 0;
    axg_solver *h = nullptr;
    check(nullptr, axg_create(&cfg, &h), "axg_create");

    axg_solid_points sp = {};
    sp.count = (int32_t)get("sp_nr").count<int32_t>();
    sp.nr = get("sp_nr").as<int32_t>();
    sp.mass = get("sp_mass").as<double>();
    sp.axial = get("sp_axial").as<uint8_t>();
    check(h, axg_set_solid_points(h, &sp), "axg_set_solid_points");

    axg_solid_elements se = {};
    se.count = (int32_t)get("se_nr").count<int32_t>();
    se.nr = get("se_nr").as<int32_t>();
    se.points = get("se_pts").as<int32_t>();
    se.axial = get("se_axial").as<uint8_t>();
    se.geometry = get("se_geom").as<double>();
    se.rheology = get("se_rheo").as<int32_t>();
    se.mat_offset = get("se_mat_off").as<int64_t>();
    se.moduli = get("se_moduli").as<double>();
    check(h, axg_set_solid_elements(h, &se), "axg_set_solid_elements");

    const Array &stf_a = get("ms_stf");       // [count][4]: half duration, decay, shift, order
    const size_t nsrc = get("ms_elem").count<int32_t>();
    std::vector<axg_stf> stf(nsrc);
    for (size_t i = 0; i < nsrc; i++) {
        const double *s = stf_a.as<double>() + 4 * i;
        stf[i] = {s[0], s[1], s[2], (int32_t)s[3]};
    }
    axg_moment_sources ms = {};
    ms.count = (int32_t)nsrc;
    ms.element = get("ms_elem").as<int32_t>();
    ms.nu = get("ms_nu").as<int32_t>();
    ms.pattern_offset = get("ms_pat_off").as<int64_t>();
    ms.pattern = get("ms_pattern").as<double>();
    ms.stf = stf.data();
    check(h, axg_set_moment_sources(h, &ms), "axg_set_moment_sources");

    axg_stations st = {};
    st.count = (int32_t)get("st_elem").count<int32_t>();
    st.element = get("st_elem").as<int32_t>();
    st.weights = get("st_w").as<double>();
    st.phi = get("st_phi").as<double>();
    check(h, axg_set_stations(h, &st, 1), "axg_set_stations");
    check(h, axg_finalize(h), "axg_finalize");

    const int nsteps = std::atoi(argv[3]);
    check(h, axg_run(h, nsteps, 1), "axg_run");

    int64_t n = 0;
    check(h, axg_field_size(h, 1, &n), "axg_field_size");
    std::vector<double> u(2 * (size_t)n);
    check(h, axg_get_field(h, 1, AXG_FIELD_DISPL, u.data()), "axg_get_field");
    int32_t nrec = 0;
    check(h, axg_get_seismograms(h, nullptr, &nrec), "axg_get_seismograms");
    std::vector<double> seis((size_t)nrec * st.count * 3);
    if (nrec) check(h, axg_get_seismograms(h, seis.data(), &nrec), "axg_get_seismograms");
    check(h, axg_destroy(h), "axg_destroy");

    const std::string pre = argv[4];
    FILE *f = std::fopen((pre + ".displ").c_str(), "wb");
    std::fwrite(u.data(), sizeof(double), u.size(), f);
    std::fclose(f);
    f = std::fopen((pre + ".seis").c_str(), "wb");
    std::fwrite(seis.data(), sizeof(double), seis.size(), f);
    std::fclose(f);
    std::printf("ok %lld %d\n", (long long)n, nrec);
    return 0;
}
