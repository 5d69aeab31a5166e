// engine.hpp -- host-side engine interface behind the C ABI (include/axg.h).
#pragma once

#include "../../include/axg.h"

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <map>
#include <algorithm>

namespace axg {

// error carrying one of the AXG_E_* codes; the message follows the reference's
// "Class::method || message" convention
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ------------------------------------------------------------- host model ---
struct HostPoints {
    int count = 0, ndim = 3;
    std::vector<int> nr, mass_nr;
    std::vector<int64_t> mass_off;
    std::vector<double> mass;
    std::vector<uint8_t> axial, surface;
};

struct HostSolidElements {
    int count = 0;
    std::vector<int> nr, pts, rheo, att;
    std::vector<uint8_t> axial, rtz, is3d;
    std::vector<double> geom, theta;
    std::vector<int64_t> mat_off, att_off;
    std::vector<double> moduli, att_moduli;
    std::vector<uint8_t> part;   // axg_set_element_parts: 0 / 1 per element, empty = all 0
};

struct HostFluidElements {
    int count = 0;
    std::vector<int> nr, pts;
    std::vector<uint8_t> axial, is3d;
    std::vector<double> geom;
    std::vector<int64_t> mat_off;
    std::vector<double> moduli;
    std::vector<uint8_t> part;
};

struct HostCoupling {
    int count = 0;
    std::vector<int> sp, fp;
    std::vector<double> nsu, nzu, nsa, nza, mf;
};

// StreamSTF / NetCDF_STF table (core/source/elem_src/stf/StreamSTF.cpp, NetCDF_STF.cpp)
struct HostStfTable {
    std::vector<double> t, v;
    int padding = 0;               // 0: out of range is an error; 1: left / right values
    double left = 0, right = 0;
    int pad_first = 0;             // NetCDF_STF: padding tested before the interpolation
};

// StreamSTF::getValue / NetCDF_STF::getValue with vector_tools::linearInterpSorted (range x
// 1e-12 tolerance): samples in Real, combined in double, cast to Real
template <class T>
inline T stf_table_value(const HostStfTable &tb, double time) {
    const size_t n = tb.t.size();
    if (tb.pad_first && tb.padding) {
        if (time < tb.t.front()) return (T)tb.left;
        if (time > tb.t.back()) return (T)tb.right;
    }
    const double tol = (tb.t.back() - tb.t.front()) * 1e-12;
    if (time < tb.t.front() - tol || time > tb.t.back() + tol) {
        if (!tb.padding)
            throw Error(AXG_E_ARG, "StreamSTF::getValue || Time is out of range with padding disabled.");
        return (T)(time < tb.t.front() ? tb.left : tb.right);
    }
    size_t i1 = (size_t)(std::upper_bound(tb.t.begin(), tb.t.end(), time) - tb.t.begin());
    if (i1 == 0) i1++;
    else if (i1 == n) i1--;
    const size_t i0 = i1 - 1;
    const double f1 = (time - tb.t[i0]) / (tb.t[i1] - tb.t[i0]), f0 = 1. - f1;
    return (T)(f0 * (double)(T)tb.v[i0] + f1 * (double)(T)tb.v[i1]);
}

struct HostCoupling3D {
    int count = 0;
    std::vector<int> sp, fp;
    std::vector<int64_t> off;
    std::vector<double> nu3, na3;    // [n][3] unassembled normal, assembled normal / fluid mass
};

struct HostSources {
    int count = 0;
    std::vector<int> elem, nu, wave;
    std::vector<int64_t> pat_off;
    std::vector<double> pattern;   // (re, im) pairs
    std::vector<axg_stf> stf;
    std::map<int, HostStfTable> table;   // sources whose STF is a table
};

struct HostStations {
    int count = 0, interval = 1;
    int gradient = 0;               // also record the 9-component displacement gradient
    std::vector<int> elem;
    std::vector<double> w, phi;
};

struct HostClayton {
    int count = 0;
    std::vector<int> pt;
    std::vector<double> rvp, rvs, area, theta;
};

struct HostClayton3D {
    int count = 0;
    std::vector<int> pt;
    std::vector<int64_t> off;
    std::vector<double> rvp, rvs, area, normal;
};

struct HostSponge3D {
    int count = 0;
    std::vector<int> pt;
    std::vector<int64_t> off;
    std::vector<double> gamma;
};

struct HostPrt {
    int count = 0;
    std::vector<int> elem;
    std::vector<int64_t> off;
    std::vector<uint8_t> x3d;
    std::vector<double> x;       // per element from off: [5][nslice][25] X0..X3, |J|
    std::vector<double> theta;   // fluid elements: [count][25] theta of the RTZ frame (empty: none)
};

struct HostScanning {
    bool enabled = false;
    double tol_fourier_h1 = 0, rel_tol_h1 = 0, abs_tol_h1 = 0;
    int max_peaks = 1, interval = 1;
    bool all_solid = false, all_fluid = false;
    std::vector<int> solid_pts, fluid_pts;
};

struct HostOcean {
    int count = 0;
    std::vector<int> pt;
    std::vector<double> mass_ocean, theta;
};

struct HostOcean3D {
    int count = 0;
    std::vector<int> pt;
    std::vector<int64_t> off;
    std::vector<double> mass_ocean, normal;
};

struct HostSponge {
    int count = 0;
    std::vector<int> pt;
    std::vector<double> gamma;
};

struct HostModel {
    HostClayton cl_s, cl_f;
    HostClayton3D cl3_s, cl3_f;
    HostSponge3D sg3_s, sg3_f;
    HostOcean ocean;
    HostOcean3D ocean3;
    HostScanning scan;
    HostPrt prt, prt_f;
    HostSponge sg_s, sg_f;
    HostPoints sp, fp;
    HostSolidElements se;
    HostFluidElements fe;
    HostCoupling sf;
    HostCoupling3D sf3;
    HostSources ms, fs, ps;          // moment, force, fluid pressure
    HostStations st;
};

// ------------------------------------------------------------ engine API ---
class EngineBase {
public:
    virtual ~EngineBase() = default;
    virtual void finalize(const HostModel &m) = 0;
    virtual void apply_sources(int tstep) = 0;
    virtual void compute_stiffness() = 0;
    virtual void compute_stiffness_part(int part) = 0;   // the buckets of one element part
    virtual void bc_before() = 0;
    virtual void point_stage(int mask) = 0;   // 1 = BC after assembly, 2 = 1/M, 4 = Newmark
    virtual void record(int tstep) = 0;
    virtual void run(int nsteps, bool graph) = 0;
    virtual int step() const = 0;
    virtual int64_t field_size(int solid) const = 0;
    virtual void get_field(int solid, int which, double *out) = 0;
    virtual void set_field(int solid, int which, const double *in) = 0;
    virtual int64_t field_raw_bytes(int solid, int which) const = 0;
    virtual void set_field_raw(int solid, int which, const void *host, int64_t bytes) = 0;
    virtual void get_field_raw(int solid, int which, void *host, int64_t bytes) = 0;
    virtual int get_seismograms(double *out) = 0;
    virtual int get_station_gradients(double *out) = 0;
    virtual void set_element_record(int n, const int *elem, const int *gll, const int *kind, int interval,
                                    int ring) = 0;
    virtual int64_t element_record_words() const = 0;
    virtual void get_element_records(int rec_first, int nrec, double *out) = 0;
    virtual void synchronize() = 0;
    virtual int64_t launches() const = 0;
    virtual void set_timing(bool on) = 0;
    virtual void stiffness_time(double *ms, int64_t *n) = 0;
    virtual void stiffness_cost(double *bytes, double *flops) const = 0;
    virtual double point_cost() const = 0;
    virtual void set_stream(void *stream) = 0;
    virtual void set_team_override(int nr_class, int team) = 0;
    virtual int bucket_count() const = 0;
    virtual void forward_checkpointed(int nsteps, int interval) = 0;
    virtual void adjoint_run(const double *seis_adj, double *grad_mod, double *grad_mass,
                             double *grad_u0, double *grad_v0) = 0;
    // per-slice sensitivities of the next adjoint runs (3-D parameterisation)
    virtual void set_adjoint_slices(bool on) = 0;
    virtual void get_adjoint_slices(double *grad_mod_slices, double *grad_mass_slices) = 0;
    // -K x added to f (device pointers, one wavefield), SLS memory in `scratch` (cap bytes,
    // cleared here); queues work on the handle's stream and allocates nothing
    virtual void stiffness_noalloc(const void *sx, void *sf, const void *fx, void *ff, void *scratch,
                                   size_t cap) = 0;
    virtual int device() const = 0;
    // boundary-stiffness exchange: n complex stiffness values at device slots <-> device buffer
    virtual void gather_stiffness(int solid, int64_t n, const int64_t *slots, void *buf) = 0;
    virtual void scatter_add_stiffness(int solid, int64_t n, const int64_t *slots, const void *buf) = 0;
    // Point::reportScanningNr per point (-1: not scanned)
    virtual void scanning_nr(int32_t *solid_nr, int32_t *fluid_nr) = 0;
};

// device address of the library's fixed no-allocation scratch on `device` (looked up
// once per device; noalloc.cu)
void *noalloc_scratch(int device);

std::unique_ptr<EngineBase> make_engine_fp32(const axg_config &cfg);
std::unique_ptr<EngineBase> make_engine_fp64(const axg_config &cfg);
std::unique_ptr<EngineBase> make_engine_mixed(const axg_config &cfg);

// spectral tables (nPol = 4), derived from their definitions (spectral.cpp)
struct SpectralTables {
    double xGLL[5], xGLJ[5], wGLL[5], wGLJ[5];
    double G_GLL[25], G_GLJ[25];   // G(j, i) = l_j'(x_i), row-major, rounded to 12 decimals
};
const SpectralTables &spectral_tables();

}  // namespace axg
