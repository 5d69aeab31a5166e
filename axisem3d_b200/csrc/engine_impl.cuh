// engine_impl.cuh -- the templated engine: device layout, buckets, step launch
// sequence and CUDA-graph capture. Instantiated once per precision in
// engine_fp32.cu, engine_fp64.cu and engine_mixed.cu.
//
// Precision parameters:
//   T   element stiffness, point stiffness/acceleration
//   AT  attenuation memory variables (state and recursion)
//   D   Newmark displacement/velocity storage
#pragma once

#include "engine.hpp"
#include "adjoint_kernel.cuh"
#include "fluid_kernel.cuh"
#include "point_kernels.cuh"
#include "prt_kernel.cuh"
#include "solid_kernel.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

namespace axg {

#define AXG_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            throw Error(e_ == cudaErrorMemoryAllocation ? AXG_E_NOMEM : AXG_E_CUDA,          \
                        std::string("Engine::" ) + __func__ + " || " + #call + " || " +      \
                            cudaGetErrorString(e_));                                         \
    } while (0)

// owning device buffer
template <class X>
struct DBuf {
    X *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { if (p) cudaFree(p); }
    void alloc(size_t count) {
        if (p) { cudaFree(p); p = nullptr; }
        n = count;
        if (count) AXG_CUDA(cudaMalloc(&p, count * sizeof(X)));
    }
    void zero(cudaStream_t s) { if (n) AXG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(X), s)); }
    void upload(const std::vector<X> &h) {
        alloc(h.size());
        if (n) AXG_CUDA(cudaMemcpy(p, h.data(), n * sizeof(X), cudaMemcpyHostToDevice));
    }
};

// team size per nr class and the nr class boundaries
constexpr int kNrClasses = 5;
inline int nr_class(int nr) { return nr <= 3 ? 0 : nr <= 9 ? 1 : nr <= 25 ? 2 : nr <= 64 ? 3 : 4; }
// smallest nr of a 3-D element that takes the slice FFTs instead of the direct sums (0 = never)
#ifndef AXG_FFT_MIN_NR
#define AXG_FFT_MIN_NR 65
#endif

inline int default_team(int cls) {
    static const int t[kNrClasses] = {32, 64, 128, 256, 256};
    return t[cls];
}

template <class T>
std::vector<T> twiddle_pool(const std::vector<int> &nrs, int nr_max, std::vector<int> &off) {
    // for each nr: cos(2 pi j / nr), j < nr, then sin; exact on the quarter points
    std::vector<T> pool;
    off.assign(nr_max + 2, 0);
    std::vector<char> need(nr_max + 1, 0);
    for (int n : nrs) need[n] = 1;
    for (int n = 1; n <= nr_max; n++) {
        off[n] = (int)pool.size();
        if (!need[n]) continue;
        for (int j = 0; j < n; j++) {
            double a = 2.0 * M_PI * j / n, c = std::cos(a);
            if (4 * j == n || 4 * j == 3 * n) c = 0; else if (2 * j == n) c = -1;
            pool.push_back((T)c);
        }
        for (int j = 0; j < n; j++) {
            double a = 2.0 * M_PI * j / n, s = std::sin(a);
            if (4 * j == n) s = 1; else if (2 * j == n) s = 0; else if (4 * j == 3 * n) s = -1;
            pool.push_back((T)s);
        }
    }
    off[nr_max + 1] = (int)pool.size();
    if (pool.empty()) pool.push_back((T)0);
    return pool;
}

template <class T, class AT, class D, bool COMP>
class Engine final : public EngineBase {
    using C = cx_t<T>;
    using CD = cx_t<D>;

    struct PointDev {
        int n = 0, ndim = 3, total = 0, n3d = 0, nr_max = 1;
        std::vector<int> h_off, h_nu, h_nr;
        std::vector<uint8_t> h_flags;
        DBuf<int> off, nu, nr, mode_pt, pt3d;
        DBuf<uint8_t> flags;
        DBuf<T> inv1, inv3;
        DBuf<int64_t> im_off;
        DBuf<C> stiff, accel, displ_elem;
        DBuf<CD> displ, veloc;
        DBuf<cx_t<float>> cd, cv;
    };

    // per-slice absorbing-boundary data (3-D Clayton, 3-D sponge) of one point set
    struct Abc3D {
        int n = 0;
        DBuf<int> pt, first;
        DBuf<int64_t> coff;
        DBuf<T> c;
    };
    struct SolidBucket {
        int rheo, att, is3d, rtz, cls, team, tpc, qc, nr_max, n, grid = 1;
        int part = 0;   // element part (axg_set_element_parts)
        int mt = 1;   // Fourier modes per tile of the gather / gradient and the quadrature
        int fft = 0;  // 3-D elements of nr >= AXG_FFT_MIN_NR take the slice FFTs
        int ahead = 0;   // L2 prefetch distance in elements (AXG_PREFETCH_AHEAD waves), 0 = off
        size_t team_bytes;
        DBuf<int> nr, pts;
        DBuf<uint8_t> axial;
        DBuf<T> geom, trig, mod, attmod;
        DBuf<int64_t> mod_off, att_off, state_off;
        double bytes = 0, flops = 0;
        void (*kernel)(const SolidArgs<T, AT>, int, int, int, int, size_t) = nullptr;
        // particle relabelling (undulated geometry): its own kernel and factors
        int prt = 0;
        DBuf<T> xpool;
        DBuf<int64_t> xoff;
        DBuf<uint8_t> x3d;
        void (*pkernel)(const PrtArgs<T, AT>, int, int, int, size_t) = nullptr;
    };
    struct FluidBucket {
        int is3d, cls, team, tpc, nr_max, n, prt = 0;
        int part = 0;
        DBuf<T> xpool, trig;
        DBuf<int64_t> xoff;
        DBuf<uint8_t> x3d;
        size_t team_bytes;
        DBuf<int> nr, pts;
        DBuf<uint8_t> axial;
        DBuf<T> geom, K;
        DBuf<int64_t> K_off;
        double bytes = 0, flops = 0;
        void (*kernel)(const FluidArgs<T>, int, int, size_t) = nullptr;
    };

public:
    explicit Engine(const axg_config &c) : cfg_(c) {
        nwave_ = std::max(1, cfg_.nwave);
        AXG_CUDA(cudaSetDevice(cfg_.device));
        AXG_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
        stream_ = own_stream_;
        AXG_CUDA(cudaGetDeviceProperties(&prop_, cfg_.device));
        for (int i = 0; i < kNrClasses; i++) team_override_[i] = 0;
    }
    ~Engine() override {
        if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (own_stream_) cudaStreamDestroy(own_stream_);
    }

    // ------------------------------------------------------------ finalize ---
    void finalize(const HostModel &m) override {
        model_ = m;
        const SpectralTables &st = spectral_tables();
        std::vector<T> g(50);
        for (int i = 0; i < 25; i++) { g[i] = (T)st.G_GLL[i]; g[25 + i] = (T)st.G_GLJ[i]; }
        gmat_.upload(g);
        build_points(m.sp, sp_, true);
        build_points(m.fp, fp_, false);
        build_ocean(m);
        // twiddles for every nr in use (3-D elements and Mass3D points)
        std::vector<int> nrs;
        int nrmax = 1;
        for (int i = 0; i < m.se.count; i++) {
            nrmax = std::max(nrmax, m.se.nr[i]);
            if (m.se.is3d.size() && m.se.is3d[i]) nrs.push_back(m.se.nr[i]);
        }
        for (int i = 0; i < m.fe.count; i++) {
            nrmax = std::max(nrmax, m.fe.nr[i]);
            if (m.fe.is3d.size() && m.fe.is3d[i]) nrs.push_back(m.fe.nr[i]);
        }
        for (const HostPoints *hp : {&m.sp, &m.fp})
            for (int p = 0; p < hp->count; p++) {
                nrmax = std::max(nrmax, hp->nr[p]);
                if (hp->mass_nr.size() && hp->mass_nr[p] > 1) nrs.push_back(hp->nr[p]);
            }
        // and the points of 3-D absorbing boundaries
        for (int i = 0; i < m.cl3_s.count; i++) nrs.push_back(m.sp.nr[m.cl3_s.pt[i]]);
        for (int i = 0; i < m.cl3_f.count; i++) nrs.push_back(m.fp.nr[m.cl3_f.pt[i]]);
        for (int i = 0; i < m.sg3_s.count; i++) nrs.push_back(m.sp.nr[m.sg3_s.pt[i]]);
        for (int i = 0; i < m.sg3_f.count; i++) nrs.push_back(m.fp.nr[m.sg3_f.pt[i]]);
        for (int i = 0; i < m.ocean3.count; i++) nrs.push_back(m.sp.nr[m.ocean3.pt[i]]);
        for (int i = 0; i < m.sf3.count; i++) nrs.push_back(m.sp.nr[m.sf3.sp[i]]);
        std::vector<int> twoff;
        tw_.upload(twiddle_pool<T>(nrs, nrmax, twoff));
        tw_off_.upload(twoff);
        build_solid_buckets(m.se);
        build_fluid_buckets(m.fe);
        if (cfg_.autotune && !cfg_.plain) autotune();
        build_coupling(m.sf);
        build_coupling3d(m);
        build_abc(m);
        build_scanning(m);
        build_sources(m.ms, m.fs);
        build_pressure_sources(m.ps);
        build_stations(m.st);
        step_dev_.alloc(1);
        step_dev_.zero(stream_);
        nonfinite_.alloc(1);
        nonfinite_.zero(stream_);
        AXG_CUDA(cudaEventCreate(&ev0_));
        AXG_CUDA(cudaEventCreate(&ev1_));
        AXG_CUDA(cudaStreamSynchronize(stream_));
        finalized_ = true;
    }

    // ------------------------------------------------------------ hooks ---
    void apply_sources(int tstep) override {
        need();
        if (tstep < 0) throw Error(AXG_E_ARG, "Domain::applySources || negative time step.");
        ensure_capacity(tstep + 1);   // the STF table must cover this step
        set_step(tstep);
        launch_sources();
    }
    void compute_stiffness() override { need(); launch_stiffness(); }
    void compute_stiffness_part(int part) override {
        need();
        if (part < 0 || part > 1) throw Error(AXG_E_ARG, "axg_compute_stiffness_part || part must be 0 or 1.");
        launch_stiffness(part);
    }
    void bc_before() override { need(); launch_clayton(); launch_coupling(); }
    void point_stage(int mask) override { need(); launch_points(mask); }
    void record(int tstep) override {
        need();
        if (tstep < 0) throw Error(AXG_E_ARG, "Domain::recordOutput || negative time step.");
        ensure_capacity(tstep + 1);
        set_step(tstep);
        launch_stations();
        launch_element_record();
        launch_scan();
    }

    void run(int nsteps, bool graph) override {
        need();
        if (nsteps <= 0) return;
        ensure_capacity(step_ + nsteps);
        set_step(step_);
        if (timing_) {
            for (int i = 0; i < nsteps; i++) {
                launch_step();
                AXG_CUDA(cudaEventSynchronize(ev1_));
                float ms = 0;
                AXG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
                time_ms_ += ms;
                time_n_ += 1;
            }
        } else if (graph && !cfg_.plain) {
            if (!graph_exec_) capture();
            for (int i = 0; i < nsteps; i++) {
                AXG_CUDA(cudaGraphLaunch(graph_exec_, stream_));
                launches_ += kernels_per_step_;
            }
        } else {
            for (int i = 0; i < nsteps; i++) launch_step();
        }
        step_ += nsteps;
        if (cfg_.stability_interval > 0) check_finite();
    }
    int step() const override { return step_; }

    // ------------------------------------------------------------- fields ---
    int64_t field_size(int solid) const override {
        const PointDev &P = solid ? sp_ : fp_;
        return (int64_t)P.total * P.ndim * nwave_;
    }
    void get_field(int solid, int which, double *out) override {
        need();
        PointDev &P = solid ? sp_ : fp_;
        size_t n = (size_t)P.total * P.ndim * nwave_;
        if (!n) return;
        AXG_CUDA(cudaStreamSynchronize(stream_));
        if (which == AXG_FIELD_DISPL || which == AXG_FIELD_VELOC) {
            std::vector<CD> h(n);
            AXG_CUDA(cudaMemcpy(h.data(), which == AXG_FIELD_DISPL ? P.displ.p : P.veloc.p,
                                n * sizeof(CD), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; i++) { out[2 * i] = (double)h[i].x; out[2 * i + 1] = (double)h[i].y; }
        } else {
            std::vector<C> h(n);
            AXG_CUDA(cudaMemcpy(h.data(), which == AXG_FIELD_STIFF ? P.stiff.p : P.accel.p,
                                n * sizeof(C), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; i++) { out[2 * i] = (double)h[i].x; out[2 * i + 1] = (double)h[i].y; }
        }
    }
    void set_field(int solid, int which, const double *in) override {
        need();
        PointDev &P = solid ? sp_ : fp_;
        size_t n = (size_t)P.total * P.ndim * nwave_;
        if (!n) return;
        AXG_CUDA(cudaStreamSynchronize(stream_));
        if (which == AXG_FIELD_DISPL || which == AXG_FIELD_VELOC) {
            std::vector<CD> h(n);
            for (size_t i = 0; i < n; i++) h[i] = mk<D>((D)in[2 * i], (D)in[2 * i + 1]);
            AXG_CUDA(cudaMemcpy(which == AXG_FIELD_DISPL ? P.displ.p : P.veloc.p, h.data(),
                                n * sizeof(CD), cudaMemcpyHostToDevice));
            if (which == AXG_FIELD_DISPL && P.displ_elem.p) {
                std::vector<C> hf(n);
                for (size_t i = 0; i < n; i++) hf[i] = mk<T>((T)h[i].x, (T)h[i].y);
                AXG_CUDA(cudaMemcpy(P.displ_elem.p, hf.data(), n * sizeof(C), cudaMemcpyHostToDevice));
            }
            if (COMP) {
                if (which == AXG_FIELD_DISPL) P.cd.zero(stream_); else P.cv.zero(stream_);
            }
        } else {
            std::vector<C> h(n);
            for (size_t i = 0; i < n; i++) h[i] = mk<T>((T)in[2 * i], (T)in[2 * i + 1]);
            AXG_CUDA(cudaMemcpy(which == AXG_FIELD_STIFF ? P.stiff.p : P.accel.p, h.data(),
                                n * sizeof(C), cudaMemcpyHostToDevice));
        }
        AXG_CUDA(cudaStreamSynchronize(stream_));
    }
    int64_t field_raw_bytes(int solid, int which) const override {
        const PointDev &P = solid ? sp_ : fp_;
        size_t n = (size_t)P.total * P.ndim * nwave_;
        bool dv = which == AXG_FIELD_DISPL || which == AXG_FIELD_VELOC;
        return (int64_t)(n * (dv ? sizeof(CD) : sizeof(C)));
    }
    void *field_ptr(PointDev &P, int which) {
        switch (which) {
            case AXG_FIELD_DISPL: return P.displ.p;
            case AXG_FIELD_VELOC: return P.veloc.p;
            case AXG_FIELD_STIFF: return P.stiff.p;
            default: return P.accel.p;
        }
    }
    void set_field_raw(int solid, int which, const void *host, int64_t bytes) override {
        need();
        if (bytes != field_raw_bytes(solid, which))
            throw Error(AXG_E_ARG, "axg_set_field_raw || byte count mismatch.");
        PointDev &P = solid ? sp_ : fp_;
        if (!bytes) return;
        AXG_CUDA(cudaMemcpyAsync(field_ptr(P, which), host, bytes, cudaMemcpyHostToDevice, stream_));
        if (which == AXG_FIELD_DISPL && P.displ_elem.p) {
            size_t n = (size_t)P.total * P.ndim * nwave_;
            narrow_kernel<T, D><<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(P.displ.p, P.displ_elem.p, n);
            post_launch();
        }
        if (COMP) {
            if (which == AXG_FIELD_DISPL) P.cd.zero(stream_);
            if (which == AXG_FIELD_VELOC) P.cv.zero(stream_);
        }
    }
    void get_field_raw(int solid, int which, void *host, int64_t bytes) override {
        need();
        if (bytes != field_raw_bytes(solid, which))
            throw Error(AXG_E_ARG, "axg_get_field_raw || byte count mismatch.");
        PointDev &P = solid ? sp_ : fp_;
        if (!bytes) return;
        AXG_CUDA(cudaMemcpyAsync(host, field_ptr(P, which), bytes, cudaMemcpyDeviceToHost, stream_));
    }
    int get_seismograms(double *out) override {
        need();
        AXG_CUDA(cudaStreamSynchronize(stream_));
        int nrec = 0;
        if (st_n_ > 0) nrec = std::min(seis_cap_, (step_ + st_interval_ - 1) / st_interval_);
        if (out && nrec > 0)
            AXG_CUDA(cudaMemcpy(out, seis_.p, (size_t)nrec * nwave_ * st_n_ * 3 * sizeof(double),
                                cudaMemcpyDeviceToHost));
        return nrec;
    }
    int get_station_gradients(double *out) override {
        need();
        if (!model_.st.gradient)
            throw Error(AXG_E_ARG, "StationSolid::record || station gradients were not requested "
                                   "(axg_set_station_gradient before axg_finalize).");
        AXG_CUDA(cudaStreamSynchronize(stream_));
        int nrec = 0;
        if (st_n_ > 0) nrec = std::min(seis_cap_, (step_ + st_interval_ - 1) / st_interval_);
        if (out && nrec > 0)
            AXG_CUDA(cudaMemcpy(out, seis_grad_.p, (size_t)nrec * nwave_ * st_n_ * 9 * sizeof(double),
                                cudaMemcpyDeviceToHost));
        return nrec;
    }
    // ----------------------------------------------------- element output ---
    void set_element_record(int n, const int *elem, const int *gll, const int *kind, int interval,
                            int ring) override {
        need();
        if (n < 0 || interval < 1 || ring < 1 || (n && (!elem || !gll || !kind)))
            throw Error(AXG_E_ARG, "ElementOpGroup::ElementOpGroup || bad element-record arguments.");
        const HostSolidElements &h = model_.se;
        std::vector<int64_t> off(std::max(n, 1), 0);
        int64_t words = 0;
        bool grad = false;
        for (int i = 0; i < n; i++) {
            if (elem[i] < 0 || elem[i] >= h.count || gll[i] < 0 || gll[i] > 24 || kind[i] < 0 || kind[i] > 1)
                throw Error(AXG_E_ARG, "ElementOpSolid::ElementOpSolid || element, GLL point or kind out of range.");
            off[i] = words;
            words += (int64_t)(h.nr[elem[i]] / 2 + 1) * (kind[i] ? 9 : 3);
            grad = grad || kind[i] == 1;
        }
        if (grad)
            for (int i = 0; i < model_.prt.count; i++)
                for (int k = 0; k < n; k++)
                    if (kind[k] == 1 && elem[k] == model_.prt.elem[i])
                        throw Error(AXG_E_ARG, "SolidElement::getNablaField || gradient output of an "
                                               "element under particle relabelling is not supported.");
        AXG_CUDA(cudaStreamSynchronize(stream_));
        er_n_ = n; er_words_ = words; er_interval_ = interval; er_ring_ = ring;
        er_elem_.upload(std::vector<int>(elem, elem + n));
        er_gll_.upload(std::vector<int>(gll, gll + n));
        er_kind_.upload(std::vector<int>(kind, kind + n));
        er_off_.upload(off);
        er_out_.alloc((size_t)ring * nwave_ * (size_t)std::max<int64_t>(words, 1));
        er_out_.zero(stream_);
        if (n) upload_elem_tables(grad);
        AXG_CUDA(cudaStreamSynchronize(stream_));
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    }
    int64_t element_record_words() const override { return er_words_; }
    void get_element_records(int rec_first, int nrec, double *out) override {
        need();
        if (!er_n_) throw Error(AXG_E_STATE, "ElementOpGroup::dumpToFile || no element record was set.");
        const int last = step_ > 0 ? (step_ - 1) / er_interval_ : -1;
        if (nrec < 0 || rec_first < 0 || rec_first + nrec - 1 > last || rec_first <= last - er_ring_ ||
            (nrec && !out))
            throw Error(AXG_E_ARG, "ElementOpGroup::dumpToFile || records not in the device ring.");
        AXG_CUDA(cudaStreamSynchronize(stream_));
        const size_t per = (size_t)nwave_ * (size_t)er_words_;
        std::vector<C> h(per);
        for (int r = 0; r < nrec; r++) {
            const int slot = (rec_first + r) % er_ring_;
            AXG_CUDA(cudaMemcpy(h.data(), er_out_.p + (size_t)slot * per, per * sizeof(C), cudaMemcpyDeviceToHost));
            double *o = out + (size_t)r * per * 2;
            for (size_t i = 0; i < per; i++) { o[2 * i] = (double)h[i].x; o[2 * i + 1] = (double)h[i].y; }
        }
    }
    void synchronize() override { AXG_CUDA(cudaStreamSynchronize(stream_)); }
    int64_t launches() const override { return launches_; }
    void set_timing(bool on) override {
        timing_ = on;
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
        time_ms_ = 0; time_n_ = 0;
    }
    void stiffness_time(double *ms, int64_t *n) override {
        AXG_CUDA(cudaStreamSynchronize(stream_));
        *ms = time_ms_;
        *n = time_n_;
    }
    void stiffness_cost(double *bytes, double *flops) const override {
        double b = 0, f = 0;
        for (auto &bk : sb_) { b += bk->bytes; f += bk->flops; }
        for (auto &bk : fb_) { b += bk->bytes; f += bk->flops; }
        // points: read u once, write f once, per wavefield
        b += nwave_ * ((double)sp_.total * 3 * 2 * sizeof(C) + (double)fp_.total * 2 * sizeof(C));
        *bytes = b;
        *flops = f;
    }
    double point_cost() const override {
        double b = 0;
        for (const PointDev *P : {&sp_, &fp_}) {
            double per = 0;
            per += 2 * sizeof(C);                          // stiff read + zero write
            per += 2 * sizeof(C);                          // accel read + write
            per += 4 * sizeof(CD);                         // d, v read + write
            if (COMP) per += 4 * sizeof(cx_t<float>);      // compensation terms
            if (P->displ_elem.p) per += sizeof(C);         // element copy of d
            b += per * (double)P->total * P->ndim * nwave_;
        }
        return b;
    }
    void set_stream(void *s) override {
        stream_ = s ? (cudaStream_t)s : own_stream_;
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    }
    void set_team_override(int cls, int team) override {
        if (cls < 0 || cls >= kNrClasses) throw Error(AXG_E_ARG, "Engine::set_team_override || bad class");
        team_override_[cls] = team;
    }
    int bucket_count() const override { return (int)(sb_.size() + fb_.size()); }

    // ------------------------------------------------------------ adjoint ---
    void forward_checkpointed(int nsteps, int interval) override {
        need();
        if (!std::is_same<T, double>::value || !std::is_same<D, double>::value)
            throw Error(AXG_E_UNSUPPORTED, "axg_forward_checkpointed || needs an FP64 handle.");
        check_adjoint_model();
        if (nsteps <= 0 || interval <= 0) throw Error(AXG_E_ARG, "axg_forward_checkpointed || bad sizes.");
        ensure_capacity(step_ + nsteps);
        const size_t nf = (size_t)sp_.total * 3;
        const int nck = (nsteps + interval - 1) / interval;
        ck_displ_.alloc(nf * nck); ck_veloc_.alloc(nf * nck); ck_accel_.alloc(nf * nck);
        if (state_wave_ > 0) ck_state_.alloc((size_t)state_wave_ * nck);
        ck_n_ = nsteps; ck_interval_ = interval; ck_step0_ = step_;
        for (int c = 0; c < nck; c++) {
            copy_fields_out(c);
            run(std::min(interval, nsteps - c * interval), true);
        }
        AXG_CUDA(cudaStreamSynchronize(stream_));
    }

    void adjoint_run(const double *seis_adj, double *grad_mod, double *grad_mass, double *grad_u0,
                     double *grad_v0) override {
        need();
        if (ck_n_ <= 0) throw Error(AXG_E_STATE, "axg_adjoint_run || no checkpointed forward run.");
        if (st_n_ > 0 && !seis_adj) throw Error(AXG_E_ARG, "axg_adjoint_run || seismogram cotangents missing.");
        build_adjoint_arrays();
        if (adj_slices_ && !adj_iso_only_)
            throw Error(AXG_E_UNSUPPORTED, "axg_adjoint_run || per-slice sensitivities need isotropic, non-attenuating elements.");
        const size_t nf = (size_t)sp_.total * 3;
        const int nck = (ck_n_ + ck_interval_ - 1) / ck_interval_;
        const int end_step = ck_step0_ + ck_n_;
        // state after the forward run, restored at the end
        DBuf<C> fin_d, fin_v, fin_a;
        fin_d.alloc(nf); fin_v.alloc(nf); fin_a.alloc(nf);
        AXG_CUDA(cudaMemcpyAsync(fin_d.p, sp_.displ.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(fin_v.p, sp_.veloc.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(fin_a.p, sp_.accel.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        DBuf<AT> fin_s;
        if (state_wave_ > 0) {
            fin_s.alloc((size_t)state_wave_);
            AXG_CUDA(cudaMemcpyAsync(fin_s.p, state_.p, (size_t)state_wave_ * sizeof(AT), cudaMemcpyDeviceToDevice,
                                     stream_));
        }
        if (adj_astate_n_ > 0) adj_astate_.zero(stream_);
        DBuf<C> ub, vb, ab, g, seg_u, seg_a, gw, kt;
        ub.alloc(nf); vb.alloc(nf); ab.alloc(nf); g.alloc(nf);
        ub.zero(stream_); vb.zero(stream_); ab.zero(stream_);
        if (adj_3d_) {   // W^-1 g and the forward kernels' -K W^-1 g
            gw.alloc(nf); kt.alloc(nf);
            kt.zero(stream_);
        }
        seg_u.alloc(nf * ck_interval_); seg_a.alloc(nf * ck_interval_);
        adj_grad_.zero(stream_);
        adj_gmass_.zero(stream_);
        if (adj_slices_) {
            build_adjoint_slices();
            adj_grad3_.zero(stream_);
            adj_gmass3_.zero(stream_);
        }
        // every seismogram cotangent of the run on the device at once (no host round trip per step)
        DBuf<double> r;
        if (st_n_) {
            const size_t nrec = (size_t)(end_step + st_interval_ - 1) / st_interval_;
            r.alloc(nrec * st_n_ * 3);
            AXG_CUDA(cudaMemcpyAsync(r.p, seis_adj, nrec * st_n_ * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                     stream_));
        }
        const int threads = 256;
        for (int c = nck - 1; c >= 0; c--) {
            const int len = std::min(ck_interval_, ck_n_ - c * ck_interval_);
            copy_fields_in(c);
            step_ = ck_step0_ + c * ck_interval_;
            set_step(step_);
            // recompute the segment, keeping u_n and a_n (the forward step's graph, which reads
            // the step from the device counter set above)
            if (!cfg_.plain && !graph_exec_) capture();
            for (int i = 0; i < len; i++) {
                AXG_CUDA(cudaMemcpyAsync(seg_u.p + nf * i, sp_.displ.p, nf * sizeof(C),
                                         cudaMemcpyDeviceToDevice, stream_));
                if (cfg_.plain) {
                    launch_step();
                } else {
                    AXG_CUDA(cudaGraphLaunch(graph_exec_, stream_));
                    launches_ += kernels_per_step_;
                }
                AXG_CUDA(cudaMemcpyAsync(seg_a.p + nf * i, sp_.accel.p, nf * sizeof(C),
                                         cudaMemcpyDeviceToDevice, stream_));
            }
            for (int i = len - 1; i >= 0; i--) {
                const int n = step_ + i;
                AdjPointArgs<T> pa;
                pa.nmodes = sp_.total; pa.mode_pt = sp_.mode_pt.p; pa.off = sp_.off.p; pa.nr = sp_.nr.p;
                pa.flags = sp_.flags.p; pa.inv_mass1 = sp_.inv1.p; pa.ubar = ub.p; pa.vbar = vb.p;
                pa.abar_out = ab.p; pa.a_n = seg_a.p + nf * i; pa.g = g.p; pa.grad_mass = adj_gmass_.p;
                pa.h = (T)cfg_.dt;
                if (adj_slices_) {
                    const int sblocks = (int)std::min<int64_t>((adj_mass3_pairs_ + threads - 1) / threads,
                                                               (int64_t)prop_.multiProcessorCount * 8);
                    adjoint_mass_slices_kernel<T><<<std::max(sblocks, 1), threads, 0, stream_>>>(
                        sp_.n, sp_.off.p, sp_.nr.p, adj_gmass3_off_.p, sp_.inv1.p, ub.p, vb.p, ab.p,
                        seg_a.p + nf * i, pa.h, adj_tw_.p, adj_tw_off_.p, adj_gmass3_.p);
                    post_launch();
                }
                adjoint_point_kernel<T><<<(unsigned)((nf + ADJ_POINT_BLOCK - 1) / ADJ_POINT_BLOCK), ADJ_POINT_BLOCK, 0,
                                          stream_>>>(pa);
                post_launch();
                AdjointArgs<T> aa;
                aa.n_elem = model_.se.count; aa.nr = e_nr_.p; aa.pts = e_pts_.p; aa.axial = e_axial_.p;
                aa.geom = adj_geom_.p; aa.mod = adj_mod_.p; aa.mod_off = adj_mod_off_.p;
                aa.pt_off = sp_.off.p; aa.pt_nu = sp_.nu.p; aa.u = seg_u.p + nf * i; aa.g = g.p;
                // -K g goes straight into ubar: the point kernel above has read ubar of step n+1,
                // and ubar_n = ubar + (-K g) + R^T r_n is a sum. With 3-D elements -K^T g =
                // -W K W^-1 g comes from the forward kernels and the adjoint kernel adds only
                // the sensitivities.
                if (adj_3d_) {
                    const int wblocks = (int)((nf + 255) / 256);
                    adjoint_weight_kernel<T><<<wblocks, 256, 0, stream_>>>((int)nf, sp_.mode_pt.p, sp_.off.p,
                                                                          sp_.nr.p, g.p, gw.p, ub.p, kt.p, 0);
                    post_launch();
                    for (auto &bp : sb_) {
                        SolidBucket &b = *bp;
                        SolidArgs<T, AT> sa;
                        sa.n_elem = b.n; sa.nr = b.nr.p; sa.pts = b.pts.p; sa.axial = b.axial.p;
                        sa.geom = b.geom.p; sa.trig = b.trig.p; sa.mod = b.mod.p; sa.mod_off = b.mod_off.p;
                        sa.attmod = b.attmod.p; sa.att_off = b.att_off.p; sa.state = state_.p;
                        sa.state_off = b.state_off.p; sa.pt_off = sp_.off.p; sa.pt_nu = sp_.nu.p;
                        sa.displ = gw.p;
                        sa.stiff = kt.p; sa.tw = tw_.p; sa.tw_off = tw_off_.p;
                        sa.nsls = cfg_.nsls;
                        for (int l = 0; l < 8; l++) {
                            sa.alpha[l] = (AT)cfg_.att_alpha[l]; sa.beta[l] = (AT)cfg_.att_beta[l];
                            sa.gamma[l] = (AT)cfg_.att_gamma[l];
                        }
                        sa.gmat = gmat_.p;
                        sa.nwave = 1;
                        sa.fstride = nf;
                        sa.sstride = (size_t)state_wave_;
                        launch_solid_args(b, sa);
                    }
                    adjoint_weight_kernel<T><<<wblocks, 256, 0, stream_>>>((int)nf, sp_.mode_pt.p, sp_.off.p,
                                                                          sp_.nr.p, g.p, gw.p, ub.p, kt.p, 1);
                    post_launch();
                }
                aa.out = adj_3d_ ? nullptr : ub.p; aa.ifact = adj_ifact_.p; aa.grad = adj_grad_.p; aa.gmat = gmat_.p;
                aa.grad3 = adj_slices_ ? adj_grad3_.p : nullptr;
                aa.grad3_off = adj_grad3_off_.p;
                aa.tw = adj_tw_.p;
                aa.tw_off = adj_tw_off_.p;
                aa.rheo = adj_rheo_.p; aa.rtz = adj_rtz_.p; aa.trig = adj_trig_.p; aa.grad_off = adj_grad_off_.p;
                aa.att = adj_att_.p; aa.attmod = adj_attmod_.p; aa.attmod_off = adj_attmod_off_.p;
                aa.astate = adj_astate_.p; aa.astate_off = adj_astate_off_.p; aa.nsls = cfg_.nsls;
                for (int l = 0; l < 8; l++) {
                    aa.alpha[l] = l < cfg_.nsls ? (T)cfg_.att_alpha[l] : (T)0;
                    aa.beta[l] = l < cfg_.nsls ? (T)cfg_.att_beta[l] : (T)0;
                    aa.gamma[l] = l < cfg_.nsls ? (T)cfg_.att_gamma[l] : (T)0;
                }
                const int nu_max = adj_nr_max_ / 2 + 1;
                const size_t smem = (size_t)nu_max * (75 + 75 + 150 + (adj_slices_ ? 300 : 0)) * sizeof(C);
                const int grid = std::min(model_.se.count, prop_.multiProcessorCount * 8);
                if (adj_slices_) adjoint_stiffness_kernel<T, true><<<grid, 128, smem, stream_>>>(aa, nu_max);
                else if (adj_generic_) adjoint_stiffness_kernel<T, false, true><<<grid, 128, smem, stream_>>>(aa, nu_max);
                else adjoint_stiffness_kernel<T, false><<<grid, 128, smem, stream_>>>(aa, nu_max);
                post_launch();
                if (st_n_ && n % st_interval_ == 0) {
                    const int rec = n / st_interval_;
                    adjoint_station_kernel<T><<<(st_n_ * 3 + 127) / 128, 128, 0, stream_>>>(
                        st_n_, st_el_.p, st_w_.p, st_phi_.p, e_nr_.p, e_pts_.p, sp_.off.p, sp_.nu.p,
                        r.p + (size_t)rec * st_n_ * 3, ub.p);
                    post_launch();
                }
            }
        }
        AXG_CUDA(cudaStreamSynchronize(stream_));
        auto d2h_cx = [&](const C *src, double *dst) {
            std::vector<C> hbuf(nf);
            AXG_CUDA(cudaMemcpy(hbuf.data(), src, nf * sizeof(C), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < nf; i++) { dst[2 * i] = (double)hbuf[i].x; dst[2 * i + 1] = (double)hbuf[i].y; }
        };
        if (grad_u0) d2h_cx(ub.p, grad_u0);
        if (grad_v0) d2h_cx(vb.p, grad_v0);
        if (grad_mod) {
            std::vector<T> hg((size_t)adj_grad_n_);
            AXG_CUDA(cudaMemcpy(hg.data(), adj_grad_.p, hg.size() * sizeof(T), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < hg.size(); i++) grad_mod[i] = (double)hg[i];
        }
        if (grad_mass) {
            std::vector<T> hm(sp_.n);
            AXG_CUDA(cudaMemcpy(hm.data(), adj_gmass_.p, hm.size() * sizeof(T), cudaMemcpyDeviceToHost));
            for (int i = 0; i < sp_.n; i++) grad_mass[i] = (double)hm[i];
        }
        // back to the state after the forward run
        AXG_CUDA(cudaMemcpyAsync(sp_.displ.p, fin_d.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(sp_.veloc.p, fin_v.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(sp_.accel.p, fin_a.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        if (state_wave_ > 0)
            AXG_CUDA(cudaMemcpyAsync(state_.p, fin_s.p, (size_t)state_wave_ * sizeof(AT), cudaMemcpyDeviceToDevice,
                                     stream_));
        sp_.stiff.zero(stream_);
        step_ = end_step;
        set_step(step_);
    }

    // The stiffness evaluation of launch_stiffness for one caller-owned wavefield (solid x / f,
    // fluid x / f on the device, in C), with the SLS memory variables in `scratch` cleared
    // first: the result is that of a handle at rest. Nothing is allocated.
    void stiffness_noalloc(const void *sx, void *sf, const void *fx, void *ff, void *scratch,
                           size_t cap) override {
        need();
        const char *who = "axg_compute_stiffness_noalloc || ";
        auto aligned = [](const void *p) { return ((uintptr_t)p % alignof(C)) == 0; };
        if (!sb_.empty() && (!sx || !sf))
            throw Error(AXG_E_ARG, std::string(who) + "solid field pointers missing.");
        if (!fb_.empty() && (!fx || !ff))
            throw Error(AXG_E_ARG, std::string(who) + "fluid field pointers missing.");
        if ((sx && !aligned(sx)) || (sf && !aligned(sf)) || (fx && !aligned(fx)) || (ff && !aligned(ff)))
            throw Error(AXG_E_ARG, std::string(who) + "field pointers must be aligned to a complex value.");
        const size_t need_bytes = (size_t)state_wave_ * sizeof(AT);
        if (need_bytes > cap)
            throw Error(AXG_E_ARG, std::string(who) + "the model's SLS state (" + std::to_string(need_bytes) +
                                       " bytes) exceeds the fixed scratch of " + std::to_string(cap) + " bytes.");
        if (need_bytes) AXG_CUDA(cudaMemsetAsync(scratch, 0, need_bytes, stream_));
        for (auto &bp : sb_) {
            SolidBucket &b = *bp;
            SolidArgs<T, AT> a;
            a.n_elem = b.n; a.nr = b.nr.p; a.pts = b.pts.p; a.axial = b.axial.p;
            a.geom = b.geom.p; a.trig = b.trig.p; a.mod = b.mod.p; a.mod_off = b.mod_off.p;
            a.attmod = b.attmod.p; a.att_off = b.att_off.p; a.state = reinterpret_cast<AT *>(scratch);
            a.state_off = b.state_off.p; a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p;
            a.displ = reinterpret_cast<const C *>(sx); a.stiff = reinterpret_cast<C *>(sf);
            a.tw = tw_.p; a.tw_off = tw_off_.p;
            a.nsls = cfg_.nsls;
            for (int l = 0; l < 8; l++) {
                a.alpha[l] = (AT)cfg_.att_alpha[l]; a.beta[l] = (AT)cfg_.att_beta[l];
                a.gamma[l] = (AT)cfg_.att_gamma[l];
            }
            a.gmat = gmat_.p;
            a.nwave = 1;
            a.fstride = 0;
            a.sstride = 0;
            launch_solid_args(b, a);
        }
        for (auto &bp : fb_) {
            FluidBucket &b = *bp;
            FluidArgs<T> a;
            a.n_elem = b.n; a.nr = b.nr.p; a.pts = b.pts.p; a.axial = b.axial.p; a.geom = b.geom.p;
            a.K = b.K.p; a.K_off = b.K_off.p; a.pt_off = fp_.off.p; a.pt_nu = fp_.nu.p;
            a.displ = reinterpret_cast<const C *>(fx); a.stiff = reinterpret_cast<C *>(ff);
            a.tw = tw_.p; a.tw_off = tw_off_.p;
            a.gmat = gmat_.p;
            a.nwave = 1;
            a.fstride = 0;
            a.x = b.xpool.p; a.x_off = b.xoff.p; a.x3d = b.x3d.p; a.trig = b.trig.p;
            int blocks = (b.n + b.tpc - 1) / b.tpc;
            b.kernel<<<blocks, b.team * b.tpc, b.tpc * b.team_bytes, stream_>>>(a, b.nr_max, b.tpc,
                                                                              b.team_bytes);
            post_launch();
        }
    }
    int device() const override { return cfg_.device; }

    void gather_stiffness(int solid, int64_t n, const int64_t *slots, void *buf) override {
        need();
        PointDev &P = solid ? sp_ : fp_;
        check_slots("axg_gather_stiffness || ", P, n, slots, buf);
        if (n == 0) return;
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)prop_.multiProcessorCount * 8);
        gather_slots_kernel<C><<<blocks, 256, 0, stream_>>>(P.stiff.p, slots, n, reinterpret_cast<C *>(buf));
        post_launch();
    }
    void scatter_add_stiffness(int solid, int64_t n, const int64_t *slots, const void *buf) override {
        need();
        PointDev &P = solid ? sp_ : fp_;
        check_slots("axg_scatter_add_stiffness || ", P, n, slots, buf);
        if (n == 0) return;
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)prop_.multiProcessorCount * 8);
        scatter_add_slots_kernel<C><<<blocks, 256, 0, stream_>>>(P.stiff.p, slots, n, reinterpret_cast<const C *>(buf));
        post_launch();
    }

private:
    void check_slots(const char *who, const PointDev &P, int64_t n, const int64_t *slots, const void *buf) const {
        if (n < 0) throw Error(AXG_E_ARG, std::string(who) + "negative count.");
        if (n > 0 && (!slots || !buf)) throw Error(AXG_E_ARG, std::string(who) + "slot or buffer pointer missing.");
        if (n > (int64_t)P.total * P.ndim)
            throw Error(AXG_E_ARG, std::string(who) + "more slots than the field holds.");
        if (nwave_ != 1) throw Error(AXG_E_UNSUPPORTED, std::string(who) + "one wavefield per handle.");
        if ((reinterpret_cast<uintptr_t>(buf) % alignof(C)) != 0)
            throw Error(AXG_E_ARG, std::string(who) + "buffer must be aligned to a complex value.");
    }
    void check_adjoint_model() const {
        const HostSolidElements &h = model_.se;
        if (fp_.n > 0) throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || fluid elements are not differentiated.");
        if (nwave_ != 1) throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || one wavefield per handle.");
        if (model_.prt.count) throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || PRT elements are not differentiated.");
        bool any3d = false, wide = false;
        for (int e = 0; e < h.count; e++) {
            const bool e3d = h.is3d.size() && h.is3d[e];
            const bool att = h.att.size() && h.att[e] != AXG_ATT_NONE;
            any3d |= e3d;
            wide |= att || h.rheo[e] != RHEO_ISO;
            if (e3d) {
                // 3-D (per-slice) moduli: isotropic and elastic, and no Nyquist mode that the
                // element and a point of it treat differently (where elements of different
                // even nr share a point the reference's operator is not self-adjoint in any
                // one weighted product)
                if (h.rheo[e] != RHEO_ISO || att)
                    throw Error(AXG_E_UNSUPPORTED,
                                "axg_adjoint || 3-D elements must be isotropic and non-attenuating.");
                for (int q = 0; q < 25; q++) {
                    const int np_ = sp_.h_nr[h.pts[(size_t)e * 25 + q]];
                    if (((h.nr[e] % 2) == 0 || (np_ % 2) == 0) && np_ != h.nr[e])
                        throw Error(AXG_E_UNSUPPORTED,
                                    "axg_adjoint || a 3-D element of even nr needs the same nr at its points.");
                }
            }
            if (h.rheo[e] != RHEO_ISO && h.rtz.size() && h.rtz[e] && h.theta.size() < (size_t)(e + 1) * 25)
                throw Error(AXG_E_ARG, "axg_adjoint || RTZ element without theta.");
        }
        if (any3d && wide)
            throw Error(AXG_E_UNSUPPORTED,
                        "axg_adjoint || 3-D elements do not mix with TI, 21-Cij or attenuating ones.");
        for (int p = 0; p < sp_.n; p++)
            if (model_.sp.mass_nr.size() && model_.sp.mass_nr[p] > 1)
                throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || 3-D masses are not differentiated.");
    }
    void copy_fields_out(int c) {
        const size_t nf = (size_t)sp_.total * 3;
        AXG_CUDA(cudaMemcpyAsync(ck_displ_.p + nf * c, sp_.displ.p, nf * sizeof(CD), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(ck_veloc_.p + nf * c, sp_.veloc.p, nf * sizeof(CD), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(ck_accel_.p + nf * c, sp_.accel.p, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        if (state_wave_ > 0)   // the SLS memory variables of the step
            AXG_CUDA(cudaMemcpyAsync(ck_state_.p + (size_t)state_wave_ * c, state_.p, (size_t)state_wave_ * sizeof(AT),
                                     cudaMemcpyDeviceToDevice, stream_));
    }
    void copy_fields_in(int c) {
        const size_t nf = (size_t)sp_.total * 3;
        AXG_CUDA(cudaMemcpyAsync(sp_.displ.p, ck_displ_.p + nf * c, nf * sizeof(CD), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(sp_.veloc.p, ck_veloc_.p + nf * c, nf * sizeof(CD), cudaMemcpyDeviceToDevice, stream_));
        AXG_CUDA(cudaMemcpyAsync(sp_.accel.p, ck_accel_.p + nf * c, nf * sizeof(C), cudaMemcpyDeviceToDevice, stream_));
        if (state_wave_ > 0)
            AXG_CUDA(cudaMemcpyAsync(state_.p, ck_state_.p + (size_t)state_wave_ * c, (size_t)state_wave_ * sizeof(AT),
                                     cudaMemcpyDeviceToDevice, stream_));
        sp_.stiff.zero(stream_);
    }
    // per-slice sensitivity buffers: [2][nr_e][25] per element, [nr_p] per point, and the
    // twiddles of every nr they use
    void build_adjoint_slices() {
        if (adj_slices_built_) return;
        const HostSolidElements &h = model_.se;
        std::vector<int64_t> goff(h.count), moff(sp_.n + 1);
        int64_t o = 0;
        std::vector<int> nrs;
        for (int e = 0; e < h.count; e++) { goff[e] = o; o += (int64_t)2 * h.nr[e] * 25; nrs.push_back(h.nr[e]); }
        adj_grad3_.alloc(std::max<int64_t>(o, 1));
        adj_grad3_n_ = o;
        o = 0;
        for (int p = 0; p < sp_.n; p++) { moff[p] = o; o += sp_.h_nr[p]; nrs.push_back(sp_.h_nr[p]); }
        moff[sp_.n] = o;
        adj_mass3_pairs_ = o;
        adj_gmass3_.alloc(std::max<int64_t>(o, 1));
        adj_grad3_off_.upload(goff);
        adj_gmass3_off_.upload(moff);
        int nrm = 1;
        for (int n : nrs) nrm = std::max(nrm, n);
        std::vector<int> toff;
        std::vector<T> tw = twiddle_pool<T>(nrs, nrm, toff);
        adj_tw_.upload(tw);
        adj_tw_off_.upload(toff);
        const int nu_max = adj_nr_max_ / 2 + 1;
        const size_t smem = (size_t)nu_max * 600 * sizeof(C);
        if (smem > 200 * 1024) throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || nr too large for per-slice sensitivities.");
        raise_smem_limit((const void *)adjoint_stiffness_kernel<T, true>, smem);
        adj_slices_built_ = true;
    }

public:
    void set_adjoint_slices(bool on) override { need(); adj_slices_ = on; }
    void get_adjoint_slices(double *g3, double *m3) override {
        need();
        if (!adj_slices_built_)
            throw Error(AXG_E_STATE, "axg_get_adjoint_slices || no adjoint run with per-slice sensitivities.");
        AXG_CUDA(cudaStreamSynchronize(stream_));
        if (g3) {
            std::vector<T> hb((size_t)adj_grad3_n_);
            if (!hb.empty()) AXG_CUDA(cudaMemcpy(hb.data(), adj_grad3_.p, hb.size() * sizeof(T), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < hb.size(); i++) g3[i] = (double)hb[i];
        }
        if (m3) {
            std::vector<T> hb((size_t)adj_mass3_pairs_);
            if (!hb.empty()) AXG_CUDA(cudaMemcpy(hb.data(), adj_gmass3_.p, hb.size() * sizeof(T), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < hb.size(); i++) m3[i] = (double)hb[i];
        }
    }

private:
    void build_adjoint_arrays() {
        if (adj_built_) return;
        const HostSolidElements &h = model_.se;
        std::vector<T> geom((size_t)h.count * 250), ifact((size_t)h.count * 25), mod, trig;
        int64_t gsize = 0;
        std::vector<int64_t> moff(h.count), goff(h.count);
        std::vector<int> rheo(h.count), att(h.count, ATT_NONE);
        std::vector<uint8_t> rtz(h.count, 0);
        std::vector<T> attmod;
        std::vector<int64_t> aoff(h.count, -1), soff(h.count, -1);
        int64_t astate_n = 0;
        adj_nr_max_ = 1;
        adj_generic_ = false;
        adj_iso_only_ = true;
        adj_3d_ = false;
        for (int e = 0; e < h.count; e++) {
            adj_nr_max_ = std::max(adj_nr_max_, h.nr[e]);
            for (int c = 0; c < 5; c++)
                for (int q = 0; q < 25; q++) {
                    geom[(size_t)e * 250 + c * 25 + q] = (T)h.geom[(size_t)e * 150 + c * 25 + q];
                    geom[(size_t)e * 250 + 125 + c * 25 + q] =
                        (T)(h.geom[(size_t)e * 150 + c * 25 + q] * h.geom[(size_t)e * 150 + 125 + q]);
                }
            for (int q = 0; q < 25; q++) ifact[(size_t)e * 25 + q] = (T)h.geom[(size_t)e * 150 + 125 + q];
            // phi-constant moduli [nmod][1][25]; isotropic-only models keep [n][2][25]
            const int nm = nmod_of(h.rheo[e]);
            moff[e] = (int64_t)mod.size();
            goff[e] = gsize;
            if (h.is3d.size() && h.is3d[e]) {
                // 3-D element (isotropic): -K^T g comes from the forward kernels; the pool keeps
                // slice 0 of lambda, mu, which only feeds the skipped quadrature
                adj_3d_ = true;
                for (int c = 0; c < 2; c++)
                    for (int q = 0; q < 25; q++)
                        mod.push_back((T)h.moduli[h.mat_off[e] + (size_t)c * h.nr[e] * 25 + q]);
            } else {
                for (int i = 0; i < nm * 25; i++) mod.push_back((T)h.moduli[h.mat_off[e] + i]);
            }
            gsize += nm * 25;
            rheo[e] = h.rheo[e];
            if (h.att.size() && h.att[e] != AXG_ATT_NONE) {
                // dlambda, dmu [2][npa] and the adjoint SLS state [nsls + 1][6][nu][npa]; the
                // gradient gains two rows (dlambda, dmu at the element points; with CG4 at its
                // four points)
                const int npa = h.att[e] == AXG_ATT_CG4 ? 4 : 25;
                att[e] = h.att[e] == AXG_ATT_CG4 ? ATT_CG4 : ATT_FULL;
                aoff[e] = (int64_t)attmod.size();
                for (int i = 0; i < 2 * npa; i++) attmod.push_back((T)h.att_moduli[h.att_off[e] + i]);
                soff[e] = astate_n;
                astate_n += (int64_t)(cfg_.nsls + 1) * 6 * (h.nr[e] / 2 + 1) * npa;
                gsize += 50;
                adj_generic_ = true;
                adj_iso_only_ = false;
            }
            if (h.rheo[e] != RHEO_ISO) {
                adj_generic_ = true;
                adj_iso_only_ = false;
                // RTZ frames matter to TI / 21-Cij elements only (the isotropic stress is frame-free)
                if (h.rtz.size() && h.rtz[e]) {
                    rtz[e] = 1;
                    trig.resize((size_t)h.count * 100, (T)0);
                    for (int q = 0; q < 25; q++) {
                        const double t = h.theta[(size_t)e * 25 + q];
                        trig[(size_t)e * 100 + q] = (T)std::sin(t);
                        trig[(size_t)e * 100 + 25 + q] = (T)std::cos(t);
                        trig[(size_t)e * 100 + 50 + q] = (T)std::sin(2. * t);
                        trig[(size_t)e * 100 + 75 + q] = (T)std::cos(2. * t);
                    }
                }
            }
        }
        if (trig.empty()) trig.push_back((T)0);
        adj_geom_.upload(geom); adj_ifact_.upload(ifact); adj_mod_.upload(mod); adj_mod_off_.upload(moff);
        adj_grad_n_ = gsize;
        adj_grad_off_.upload(goff);
        if (attmod.empty()) attmod.push_back((T)0);
        adj_att_.upload(att);
        adj_attmod_.upload(attmod);
        adj_attmod_off_.upload(aoff);
        adj_astate_off_.upload(soff);
        adj_astate_n_ = astate_n;
        adj_astate_.alloc(std::max<int64_t>(astate_n, 1));
        adj_rheo_.upload(rheo);
        adj_rtz_.upload(rtz);
        adj_trig_.upload(trig);
        adj_grad_.alloc(std::max<int64_t>(adj_grad_n_, 1));
        adj_gmass_.alloc(sp_.n);
        if (!e_nr_.p) {
            e_nr_.upload(h.nr); e_pts_.upload(h.pts);
            std::vector<uint8_t> ax(h.axial.begin(), h.axial.end());
            e_axial_.upload(ax);
        }
        int nu_max = adj_nr_max_ / 2 + 1;
        size_t smem = (size_t)nu_max * 300 * sizeof(C);
        if (smem > 200 * 1024) throw Error(AXG_E_UNSUPPORTED, "axg_adjoint || nr too large.");
        raise_smem_limit((const void *)adjoint_stiffness_kernel<T, false>, smem);
        raise_smem_limit((const void *)adjoint_stiffness_kernel<T, true>, smem);
        raise_smem_limit((const void *)adjoint_stiffness_kernel<T, false, true>, smem);
        adj_built_ = true;
    }

    void need() const {
        if (!finalized_) throw Error(AXG_E_STATE, "Engine::step || axg_finalize not called.");
    }
    void set_step(int tstep) {
        tstep_host_ = tstep;
        AXG_CUDA(cudaMemcpyAsync(step_dev_.p, &tstep_host_, sizeof(int), cudaMemcpyHostToDevice, stream_));
        AXG_CUDA(cudaStreamSynchronize(stream_));
    }
    void check_finite() {
        int flag = 0;
        AXG_CUDA(cudaMemcpyAsync(&flag, nonfinite_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        AXG_CUDA(cudaStreamSynchronize(stream_));
        if (flag) throw Error(AXG_E_UNSTABLE, "Domain::checkStability || Non-finite displacement.");
    }

    // -------------------------------------------------------- points ---
    // MassOceanLoad1D constructor (MassOceanLoad1D.hpp): coefficients in double, cast
    void build_ocean(const HostModel &m) {
        build_ocean3d(m);
        ocean_n_ = m.ocean.count;
        if (!ocean_n_) return;
        std::vector<T> c((size_t)4 * ocean_n_);
        for (int i = 0; i < ocean_n_; i++) {
            const int p = m.ocean.pt[i];
            const int64_t mo = m.sp.mass_off.size() ? m.sp.mass_off[p] : p;
            const double mass = m.sp.mass[mo], mv = mass + m.ocean.mass_ocean[i];
            const double ct = std::cos(m.ocean.theta[i]), st = std::sin(m.ocean.theta[i]);
            c[4 * i] = (T)(1. / mass * ct * ct + 1. / mv * st * st);
            c[4 * i + 1] = (T)(1. / mass * st * st + 1. / mv * ct * ct);
            c[4 * i + 2] = (T)((1. / mv - 1. / mass) * ct * st);
            c[4 * i + 3] = (T)(1 / mass);
            sp_.h_flags[p] |= PT_OCEAN;
        }
        ocean_pt_.upload(m.ocean.pt);
        ocean_c_.upload(c);
        sp_.flags.upload(sp_.h_flags);
    }

    // MassOceanLoad3D constructor (MassOceanLoad3D.cpp): 1/m and k = sqrt(m0 / (m (m + m0))) n
    // per slice, in double, cast; these points leave the Mass3D list (their kernel does 1/M)
    void build_ocean3d(const HostModel &m) {
        ocean3_n_ = m.ocean3.count;
        if (!ocean3_n_) return;
        std::vector<T> c;
        std::vector<int64_t> coff;
        for (int i = 0; i < ocean3_n_; i++) {
            const int p = m.ocean3.pt[i], nr = m.sp.nr[p];
            const int mnr = m.sp.mass_nr.size() ? m.sp.mass_nr[p] : 1;
            const int64_t mo = m.sp.mass_off.size() ? m.sp.mass_off[p] : p;
            coff.push_back((int64_t)c.size());
            for (int k = 0; k < nr; k++) {
                const double mass = m.sp.mass[mo + (mnr > 1 ? k : 0)];
                const int64_t q = m.ocean3.off[i] + k;
                const double m0 = m.ocean3.mass_ocean[q];
                const double sk = std::sqrt(m0 / (mass * (mass + m0)));
                c.push_back((T)(1.0 / mass));
                for (int d = 0; d < 3; d++) c.push_back((T)(sk * m.ocean3.normal[q * 3 + d]));
            }
            sp_.h_flags[p] = (uint8_t)((sp_.h_flags[p] & ~PT_MASS3D) | PT_OCEAN);
        }
        ocean3_pt_.upload(m.ocean3.pt);
        ocean3_coff_.upload(coff);
        ocean3_c_.upload(c);
        sp_.flags.upload(sp_.h_flags);
        std::vector<int> pt3d;
        for (int p = 0; p < sp_.n; p++)
            if (sp_.h_flags[p] & PT_MASS3D) pt3d.push_back(p);
        sp_.n3d = (int)pt3d.size();
        sp_.pt3d.upload(pt3d);
    }

    void build_points(const HostPoints &h, PointDev &P, bool solid) {
        P.n = h.count;
        P.ndim = solid ? 3 : 1;
        P.h_off.resize(P.n); P.h_nu.resize(P.n); P.h_nr.resize(P.n);
        std::vector<int> mode_pt, pt3d;
        std::vector<uint8_t> flags(P.n, 0);
        std::vector<T> inv1(P.n, (T)0), inv3;
        std::vector<int64_t> im_off(P.n, 0);
        int o = 0;
        for (int p = 0; p < P.n; p++) {
            int nr = h.nr[p];
            if (nr < 1) throw Error(AXG_E_ARG, "Point::Point || nr must be >= 1.");
            P.h_nr[p] = nr; P.h_nu[p] = nr / 2 + 1; P.h_off[p] = o;
            for (int a = 0; a < P.h_nu[p]; a++) mode_pt.push_back(p);
            o += P.h_nu[p];
            P.nr_max = std::max(P.nr_max, nr);
            int mnr = h.mass_nr.size() ? h.mass_nr[p] : 1;
            int64_t mo = h.mass_off.size() ? h.mass_off[p] : p;
            if (mnr == 1) {
                inv1[p] = (T)(1.0 / h.mass[mo]);        // Mass1D: (Real)(1 / mass)
            } else {
                if (mnr != nr) throw Error(AXG_E_ARG, "Mass3D::checkCompatibility || Incompatible sizes.");
                flags[p] |= PT_MASS3D;
                pt3d.push_back(p);
                im_off[p] = (int64_t)inv3.size();
                for (int k = 0; k < mnr; k++) inv3.push_back((T)(1.0 / h.mass[mo + k]));
            }
            if (h.axial.size() && h.axial[p]) flags[p] |= PT_AXIAL;
            if (h.surface.size() && h.surface[p]) flags[p] |= PT_SURFACE;
        }
        P.total = o;
        P.n3d = (int)pt3d.size();
        P.off.upload(P.h_off); P.nu.upload(P.h_nu); P.nr.upload(P.h_nr);
        P.mode_pt.upload(mode_pt); P.pt3d.upload(pt3d);
        P.flags.upload(flags); P.inv1.upload(inv1);
        P.h_flags = flags;
        if (inv3.empty()) inv3.push_back((T)0);
        P.inv3.upload(inv3); P.im_off.upload(im_off);
        size_t nf = (size_t)P.total * P.ndim * nwave_;
        P.stiff.alloc(nf); P.stiff.zero(stream_);
        P.accel.alloc(nf); P.accel.zero(stream_);
        P.displ.alloc(nf); P.displ.zero(stream_);
        P.veloc.alloc(nf); P.veloc.zero(stream_);
        if (sizeof(D) != sizeof(T)) { P.displ_elem.alloc(nf); P.displ_elem.zero(stream_); }
        if (COMP) { P.cd.alloc(nf); P.cd.zero(stream_); P.cv.alloc(nf); P.cv.zero(stream_); }
    }
    // displacement as seen by the elements
    const C *elem_displ(const PointDev &P) const {
        if constexpr (sizeof(D) != sizeof(T)) return P.displ_elem.p;
        else return reinterpret_cast<const C *>(P.displ.p);
    }

    // ------------------------------------------------------- solid buckets ---
    using SolidKernel = void (*)(const SolidArgs<T, AT>, int, int, int, int, size_t);
    // NS: the register-resident SLS recursions are built for 3 and 5 SLS (3-D slices and
    // 1-D Fourier slots); other counts take the generic path
    template <int RHEO, int ATT, bool IS3D, bool RTZ>
    static SolidKernel pick4(int nsls, bool fft) {
#ifndef AXG_GENERIC_SLS_ONLY
        if constexpr (ATT != ATT_NONE) {
            if constexpr (IS3D) {
                if (fft && nsls == 3) return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 3, true>;
                if (fft && nsls == 5) return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 5, true>;
            }
            if (nsls == 3) return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 3>;
            if (nsls == 5) return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 5>;
        }
#endif
        if constexpr (IS3D && ATT == ATT_NONE) {
            if (fft) return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 0, true>;
        }
        return solid_stiffness_kernel<T, AT, RHEO, ATT, IS3D, RTZ, 0>;
    }
    template <int RHEO, int ATT, bool IS3D>
    static SolidKernel pick3(bool rtz, int nsls, bool fft) {
        if constexpr (RHEO == RHEO_ISO) return pick4<RHEO, ATT, IS3D, false>(nsls, fft);
        else return rtz ? pick4<RHEO, ATT, IS3D, true>(nsls, fft) : pick4<RHEO, ATT, IS3D, false>(nsls, fft);
    }
    template <int RHEO, int ATT>
    static SolidKernel pick2(bool is3d, bool rtz, int nsls, bool fft) {
        return is3d ? pick3<RHEO, ATT, true>(rtz, nsls, fft) : pick3<RHEO, ATT, false>(rtz, nsls, fft);
    }
    template <int RHEO>
    static SolidKernel pick1(int att, bool is3d, bool rtz, int nsls, bool fft) {
        switch (att) {
            case ATT_NONE: return pick2<RHEO, ATT_NONE>(is3d, rtz, nsls, fft);
            case ATT_FULL: return pick2<RHEO, ATT_FULL>(is3d, rtz, nsls, fft);
            default: return pick2<RHEO, ATT_CG4>(is3d, rtz, nsls, fft);
        }
    }
    static SolidKernel pick_solid(int rheo, int att, bool is3d, bool rtz, int nsls, bool fft) {
        switch (rheo) {
            case RHEO_ISO: return pick1<RHEO_ISO>(att, is3d, rtz, nsls, fft);
            case RHEO_TISO: return pick1<RHEO_TISO>(att, is3d, rtz, nsls, fft);
            default: return pick1<RHEO_ANISO>(att, is3d, rtz, nsls, fft);
        }
    }

    using PrtKernel = void (*)(const PrtArgs<T, AT>, int, int, int, size_t);
    template <int RHEO, int ATT>
    static PrtKernel pick_prt2(bool is3d, bool rtz) {
        if (is3d) return rtz ? solid_prt_kernel<T, AT, RHEO, ATT, true, true> : solid_prt_kernel<T, AT, RHEO, ATT, true, false>;
        return rtz ? solid_prt_kernel<T, AT, RHEO, ATT, false, true> : solid_prt_kernel<T, AT, RHEO, ATT, false, false>;
    }
    template <int RHEO>
    static PrtKernel pick_prt1(int att, bool is3d, bool rtz) {
        switch (att) {
            case ATT_NONE: return pick_prt2<RHEO, ATT_NONE>(is3d, rtz);
            case ATT_FULL: return pick_prt2<RHEO, ATT_FULL>(is3d, rtz);
            default: return pick_prt2<RHEO, ATT_CG4>(is3d, rtz);
        }
    }
    static PrtKernel pick_prt(int rheo, int att, bool is3d, bool rtz) {
        switch (rheo) {
            case RHEO_ISO: return pick_prt1<RHEO_ISO>(att, is3d, rtz);
            case RHEO_TISO: return pick_prt1<RHEO_TISO>(att, is3d, rtz);
            default: return pick_prt1<RHEO_ANISO>(att, is3d, rtz);
        }
    }

    int nmod_of(int rheo) const { return rheo == RHEO_ISO ? 2 : rheo == RHEO_TISO ? 5 : 21; }

    // Colour of every element for deterministic assembly (axg_config.deterministic): greedy, in
    // element order, the smallest colour none of the element's points has seen yet; all zero
    // otherwise. Within one colour no two elements share a point, so each launch adds at most
    // one contribution to any point stiffness, and the launches run one after another: the sums
    // come out in the same order on every run.
    std::vector<int> element_colours(const std::vector<int> &pts, int count, int npoints) const {
        std::vector<int> colour(count, 0);
        if (!cfg_.deterministic) return colour;
        std::vector<uint64_t> seen(std::max(npoints, 1), 0);
        for (int e = 0; e < count; e++) {
            uint64_t used = 0;
            for (int q = 0; q < 25; q++) {
                const int p = pts[(size_t)e * 25 + q];
                if (p >= 0 && p < npoints) used |= seen[p];
            }
            if (~used == 0) throw Error(AXG_E_UNSUPPORTED, "Engine::finalize || more than 64 element colours.");
            int c = 0;
            while (used & (uint64_t(1) << c)) c++;
            colour[e] = c;
            for (int q = 0; q < 25; q++) {
                const int p = pts[(size_t)e * 25 + q];
                if (p >= 0 && p < npoints) seen[p] |= uint64_t(1) << c;
            }
        }
        return colour;
    }

    void build_solid_buckets(const HostSolidElements &h) {
        // group elements by (rheology, attenuation, 1-D/3-D, RTZ, nr class, PRT)
        const HostPrt &hp = model_.prt;
        std::vector<int> prt_of(h.count, -1);
        for (int i = 0; i < hp.count; i++) prt_of[hp.elem[i]] = i;
        // deterministic assembly: elements coloured so that no two of one colour share a point,
        // one bucket per colour, the buckets launched in turn
        const std::vector<int> colour = element_colours(h.pts, h.count, sp_.n);
        std::map<std::tuple<int, int, int, int, int, int, int, int>, std::vector<int>> groups;
        for (int e = 0; e < h.count; e++) {
            int att = h.att.size() ? h.att[e] : ATT_NONE;
            int is3d = h.is3d.size() ? h.is3d[e] : 0;
            int rtz = h.rtz.size() ? h.rtz[e] : 0;
            const int prt = prt_of[e] >= 0 ? 1 : 0;
            // isotropic rheology is frame invariant; with PRT the RTZ frame carries the factors
            if (h.rheo[e] == RHEO_ISO && !prt) rtz = 0;
            if (att != ATT_NONE && cfg_.nsls <= 0)
                throw Error(AXG_E_ARG, "Attenuation::checkCompatibility || nsls must be > 0.");
            const int part = h.part.size() == (size_t)h.count ? h.part[e] : 0;
            groups[{h.rheo[e], att, is3d, rtz, cfg_.plain ? 0 : nr_class(h.nr[e]), prt, colour[e], part}].push_back(e);
        }
        int64_t state_total = 0;
        std::vector<std::vector<int64_t>> state_offs;
        for (auto &kv : groups) {
            auto b = std::make_unique<SolidBucket>();
            std::tie(b->rheo, b->att, b->is3d, b->rtz, b->cls, b->prt, std::ignore, b->part) = kv.first;
            std::vector<T> xpool;
            std::vector<int64_t> xoff;
            std::vector<uint8_t> x3d;
            const std::vector<int> &ids = kv.second;
            b->n = (int)ids.size();
            b->nr_max = 1;
            std::vector<int> nr(b->n), pts((size_t)b->n * 25);
            std::vector<uint8_t> ax(b->n);
            std::vector<T> geom((size_t)b->n * 250), trig, mod, attm;
            std::vector<int64_t> moff(b->n), aoff(b->n, 0), soff(b->n, 0);
            if (b->rtz) trig.resize((size_t)b->n * 100);
            int nm = nmod_of(b->rheo);
            int npa = b->att == ATT_CG4 ? 4 : 25;
            double bytes = 0, flops = 0;
            for (int k = 0; k < b->n; k++) {
                int e = ids[k];
                int enr = h.nr[e], enu = enr / 2 + 1, ns = b->is3d ? enr : 1;
                nr[k] = enr;
                b->nr_max = std::max(b->nr_max, enr);
                ax[k] = h.axial[e];
                for (int q = 0; q < 25; q++) {
                    int p = h.pts[(size_t)e * 25 + q];
                    if (p < 0 || p >= sp_.n) throw Error(AXG_E_ARG, "SolidElement::SolidElement || point index out of range.");
                    pts[(size_t)k * 25 + q] = p;
                }
                const double *g = &h.geom[(size_t)e * 150];
                for (int c = 0; c < 5; c++)
                    for (int q = 0; q < 25; q++) {
                        // plain operators cast to Real; _IF products formed in double
                        // (GradientQuadrature.hpp:122-137)
                        geom[(size_t)k * 250 + c * 25 + q] = (T)g[c * 25 + q];
                        geom[(size_t)k * 250 + 125 + c * 25 + q] = (T)(g[c * 25 + q] * g[125 + q]);
                    }
                if (b->rtz)
                    for (int q = 0; q < 25; q++) {
                        double t = h.theta[(size_t)e * 25 + q];
                        trig[(size_t)k * 100 + q] = (T)std::sin(t);
                        trig[(size_t)k * 100 + 25 + q] = (T)std::cos(t);
                        trig[(size_t)k * 100 + 50 + q] = (T)std::sin(2. * t);
                        trig[(size_t)k * 100 + 75 + q] = (T)std::cos(2. * t);
                    }
                moff[k] = (int64_t)mod.size();
                const double *mm = &h.moduli[h.mat_off[e]];
                for (size_t i = 0; i < (size_t)nm * ns * 25; i++) mod.push_back((T)mm[i]);
                if (b->att != ATT_NONE) {
                    aoff[k] = (int64_t)attm.size();
                    const double *am = &h.att_moduli[h.att_off[e]];
                    for (size_t i = 0; i < (size_t)2 * ns * npa; i++) attm.push_back((T)am[i]);
                    int64_t slots = b->is3d ? (int64_t)enr * npa : (int64_t)enu * npa * 2;
                    soff[k] = state_total;
                    state_total += (int64_t)(cfg_.nsls + 1) * 6 * slots;
                }
                // algorithmic bytes and flops of this element: every operand read once, the SLS state
                // read and written once, point modes counted with the points (stiffness roofline)
                double s = sizeof(T), sa = sizeof(AT);
                bytes += 6 * 25 * s + 25 * 4 + 8;                        // geometry, point ids, nr
                bytes += (double)nm * ns * 25 * s;                        // moduli
                if (b->att != ATT_NONE) {
                    bytes += 2.0 * ns * npa * s;                          // dlambda, dmu
                    double slots = b->is3d ? (double)enr * npa : (double)enu * npa * 2;
                    bytes += 2.0 * (cfg_.nsls + 1) * 6 * slots * sa * nwave_;   // state read + write
                }
                if (b->rtz) bytes += 25 * s;                              // theta
                if (b->prt) {
                    // PRT factors X0..X3 and their |J|-scaled copies (PRT.hpp constructor: the
                    // products formed in double, then cast)
                    const int i = prt_of[e];
                    const int xns = hp.x3d[i] ? enr : 1;
                    const double *x = &hp.x[hp.off[i]];
                    const size_t xs = (size_t)xns * 25;
                    xoff.push_back((int64_t)xpool.size());
                    x3d.push_back(hp.x3d[i]);
                    for (int c = 0; c < 4; c++)
                        for (size_t j = 0; j < xs; j++) xpool.push_back((T)x[c * xs + j]);
                    for (int c = 0; c < 4; c++)
                        for (size_t j = 0; j < xs; j++) xpool.push_back((T)(x[c * xs + j] * x[4 * xs + j]));
                    bytes += 8.0 * xs * s;
                }
                flops += nwave_ * (double)enu * 25 * (2 * 3 * 10 * 4 + 60);   // gradient
                flops += nwave_ * (double)enu * 25 * (2 * 3 * 10 * 4 + 60);   // quadrature
                double pw = nm == 2 ? 16 : nm == 5 ? 22 : 72;             // stress per point
                if (b->is3d) {
                    flops += nwave_ * 2.0 * 150 * enr * enu * 4;          // two direct DFTs
                    flops += nwave_ * (double)enr * 25 * pw;
                    if (b->att != ATT_NONE) flops += nwave_ * (double)enr * npa * (cfg_.nsls * 6 * 4 + 14);
                } else {
                    flops += nwave_ * (double)enu * 25 * pw * 2;
                    if (b->att != ATT_NONE) flops += nwave_ * (double)enu * npa * 2 * (cfg_.nsls * 6 * 4 + 14);
                }
            }
            b->bytes = bytes;
            b->flops = flops;
            b->nr.upload(nr); b->pts.upload(pts); b->axial.upload(ax);
            b->geom.upload(geom);
            if (trig.empty()) trig.push_back((T)0);
            b->trig.upload(trig);
            if (mod.empty()) mod.push_back((T)0);
            if (attm.empty()) attm.push_back((T)0);
            b->mod.upload(mod); b->attmod.upload(attm);
            b->mod_off.upload(moff); b->att_off.upload(aoff);
            state_offs.push_back(soff);
            if (b->prt) {
                b->xpool.upload(xpool); b->xoff.upload(xoff); b->x3d.upload(x3d);
                b->pkernel = pick_prt(b->rheo, b->att, b->is3d, b->rtz);
            } else {
                // the slice FFTs: batched 3-D buckets of the register-resident slice path that
                // hold an nr of at least AXG_FFT_MIN_NR (the plain method keeps the direct sums)
                const bool reg_path = b->att == ATT_NONE || cfg_.nsls == 3 || cfg_.nsls == 5;
                b->fft = (!cfg_.plain && b->is3d && reg_path && AXG_FFT_MIN_NR > 0 && b->nr_max >= AXG_FFT_MIN_NR) ? 1 : 0;
                b->kernel = pick_solid(b->rheo, b->att, b->is3d, b->rtz, cfg_.nsls, b->fft != 0);
            }
            configure_bucket(*b);
            sb_.push_back(std::move(b));
        }
        state_wave_ = state_total;
        state_.alloc(std::max<int64_t>(state_total * nwave_, 1));
        state_.zero(stream_);
        for (size_t i = 0; i < sb_.size(); i++) sb_[i]->state_off.upload(state_offs[i]);
    }

#ifndef AXG_QC_FOR_TWO_CTAS
#define AXG_QC_FOR_TWO_CTAS 1
#endif
    void configure_bucket(SolidBucket &b, int team_req = 0) {
        int team = team_req ? team_req
                            : (cfg_.plain ? 256 : (team_override_[b.cls] ? team_override_[b.cls] : default_team(b.cls)));
        // shared memory per team (the PRT kernel holds 9 gradient components instead of 6)
        const int nu_max = b.nr_max / 2 + 1;
        auto bytes_of = [&](int q, int m) {
            return b.prt ? prt_layout<T>(b.nr_max, q).total : team_layout<T>(b.nr_max, q, m).total;
        };
        const void *kfn = b.prt ? (const void *)b.pkernel : (const void *)b.kernel;
        // split the 25 points of the slice phase if needed
        const size_t budget = 200 * 1024;
        int qc = 25, mt = nu_max;
        size_t total = bytes_of(qc, mt);
        while (total > budget && qc > 1) { qc = (qc + 1) / 2; total = bytes_of(qc, mt); }
        if (total > budget && !b.prt) {
            // large nr: the gather / gradient and the quadrature run over tiles of mt modes;
            // the largest point chunk for which a tile of at least 8 modes fits (any tile
            // with one-point chunks as the last resort)
            for (qc = 25;; qc = (qc + 1) / 2) {
                mt = nu_max;
                while (mt > 1 && bytes_of(qc, mt) > budget) mt = (mt + 1) / 2;
                total = bytes_of(qc, mt);
                if ((total <= budget && mt >= std::min(8, nu_max)) || qc == 1) break;
            }
        }
        if (total > budget)
            throw Error(AXG_E_UNSUPPORTED, "SolidElement::expandWorkspace || nr too large for shared memory.");
#if AXG_QC_FOR_TWO_CTAS
        // a one-element CTA too large for two per SM: smaller point chunks of the slice phase
        // often let a second CTA in
        // (kept only when it does: smaller chunks alone idle threads in the slice passes)
        if (team >= 128 && b.is3d && mt == nu_max) {
            // the shared memory of AXG_SOLID_MIN_BLOCKS CTAs per SM (228 KB per SM, 1 KB of it
            // reserved per CTA)
            const size_t two_per_sm = AXG_SOLID_MIN_BLOCKS >= 3 ? (size_t)(228 / AXG_SOLID_MIN_BLOCKS - 1) * 1024
                                                                : (size_t)110 * 1024;
            int qn = qc;
            size_t tn = total;
            while (qn > 5 && tn > two_per_sm) {
                const size_t th = bytes_of((qn + 1) / 2, mt);
                if (th >= tn) break;
                qn = (qn + 1) / 2;
                tn = th;
            }
            if (tn <= two_per_sm) {
                qc = qn;
                total = tn;
            } else if (!cfg_.plain && !b.prt) {
                // large nr: point chunks alone cannot get there while region B holds a whole
                // element's modes; mode tiles of at least 8 modes as well, the largest point
                // chunk (of at least 2 points) first
                for (int qm = qc; qm >= 2; qm = (qm + 1) / 2) {
                    int mm = nu_max;
                    while (mm > 8 && bytes_of(qm, mm) > two_per_sm) mm = (mm + 1) / 2;
                    if (bytes_of(qm, mm) <= two_per_sm) {
                        qc = qm;
                        mt = mm;
                        total = bytes_of(qm, mm);
                        break;
                    }
                    if (qm == 2) break;
                }
            }
        }
#endif
        b.qc = qc;
        b.mt = mt;
        b.team_bytes = total;
        b.team = team;
        int tpc = std::max(1, 256 / team);
        while (tpc > 1 && (size_t)tpc * total > budget) tpc--;
        if (team > 32) tpc = std::min(tpc, 15);
        b.tpc = tpc;
        raise_smem_limit(kfn, tpc * total);
        // one CTA per group of tpc elements: measured faster on B200 than a persistent grid
        // (the hardware scheduler refills an SM as soon as any CTA ends, which hides the
        // tail of uneven nr better than a fixed walk). AXG_PERSISTENT_GRID restores the
        // persistent walk with next-element L2 prefetch.
        b.grid = (b.n + tpc - 1) / tpc;
        b.ahead = 0;
#if AXG_PREFETCH_AHEAD > 0
        if (!cfg_.plain && !b.prt) {
            int per_sm = 0;
            AXG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, team * tpc, tpc * total));
            b.ahead = AXG_PREFETCH_AHEAD * std::max(per_sm, 1) * prop_.multiProcessorCount * tpc;
        }
#endif
#ifdef AXG_PERSISTENT_GRID
        int per_sm = 0;
        AXG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, team * tpc, tpc * total));
        if (!cfg_.plain && !b.prt)
            b.grid = std::max(1, std::min(b.grid, std::max(1, per_sm) * prop_.multiProcessorCount));
#endif
    }

    // The project's autotuner: for every solid bucket, time each feasible team size
    // (threads per element) on the bucket's own elements and keep the fastest. The
    // fields are zero at this point, so the trial launches change no result; the
    // attenuation state and the stiffness are cleared afterwards all the same.
    void autotune() {
        cudaEvent_t t0, t1;
        AXG_CUDA(cudaEventCreate(&t0));
        AXG_CUDA(cudaEventCreate(&t1));
        for (auto &bp : sb_) {
            SolidBucket &b = *bp;
            float best = 1e30f;
            int best_team = b.team;
            for (int team : {32, 64, 128, 256}) {
                b.team = team;
                configure_bucket(b, team);
                float ms = 0;
                for (int rep = 0; rep < 3; rep++) {
                    AXG_CUDA(cudaEventRecord(t0, stream_));
                    launch_solid_bucket(b);
                    AXG_CUDA(cudaEventRecord(t1, stream_));
                    AXG_CUDA(cudaEventSynchronize(t1));
                    float x = 0;
                    AXG_CUDA(cudaEventElapsedTime(&x, t0, t1));
                    if (rep > 0) ms += x;   // the first launch warms caches
                }
                if (ms < best) { best = ms; best_team = team; }
            }
            configure_bucket(b, best_team);
            tuned_.push_back({b.cls, best_team, best / 2});
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        state_.zero(stream_);
        sp_.stiff.zero(stream_);
        AXG_CUDA(cudaStreamSynchronize(stream_));
    }

    // several buckets, and several handles on one device, can share one kernel instantiation,
    // and its dynamic shared memory limit is an attribute of the function on that device, not of
    // a handle: the limit only ever rises, to the largest any handle has asked for
    void raise_smem_limit(const void *kernel, size_t bytes) {
        static std::mutex mu;
        static std::map<std::pair<int, const void *>, size_t> limits;
        std::lock_guard<std::mutex> lock(mu);
        size_t &cur = limits[{cfg_.device, kernel}];
        if (bytes <= cur) return;
        cur = bytes;
        AXG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    }

    // ------------------------------------------------------- fluid buckets ---
    using FluidKernel = void (*)(const FluidArgs<T>, int, int, size_t);
    void build_fluid_buckets(const HostFluidElements &h) {
        // group by (1-D/3-D, nr class, PRT mode: 0 none, 1 PRT, 2 PRT in the RTZ frame)
        const HostPrt &hp = model_.prt_f;
        std::vector<int> prt_of(h.count, -1);
        for (int i = 0; i < hp.count; i++) prt_of[hp.elem[i]] = i;
        const std::vector<int> colour = element_colours(h.pts, h.count, fp_.n);
        std::map<std::tuple<int, int, int, int, int>, std::vector<int>> groups;
        for (int e = 0; e < h.count; e++) {
            const int mode = prt_of[e] < 0 ? 0 : (hp.theta.empty() ? 1 : 2);
            const int part = h.part.size() == (size_t)h.count ? h.part[e] : 0;
            groups[{h.is3d.size() ? h.is3d[e] : 0, cfg_.plain ? 0 : nr_class(h.nr[e]), mode, colour[e], part}]
                .push_back(e);
        }
        for (auto &kv : groups) {
            auto b = std::make_unique<FluidBucket>();
            std::tie(b->is3d, b->cls, b->prt, std::ignore, b->part) = kv.first;
            std::vector<T> xpool, trig;
            std::vector<int64_t> xoff;
            std::vector<uint8_t> x3d;
            const std::vector<int> &ids = kv.second;
            b->n = (int)ids.size();
            b->nr_max = 1;
            std::vector<int> nr(b->n), pts((size_t)b->n * 25);
            std::vector<uint8_t> ax(b->n);
            std::vector<T> geom((size_t)b->n * 250), K;
            std::vector<int64_t> koff(b->n);
            double bytes = 0, flops = 0;
            for (int k = 0; k < b->n; k++) {
                int e = ids[k];
                int enr = h.nr[e], enu = enr / 2 + 1, ns = b->is3d ? enr : 1;
                nr[k] = enr;
                b->nr_max = std::max(b->nr_max, enr);
                ax[k] = h.axial[e];
                for (int q = 0; q < 25; q++) {
                    int p = h.pts[(size_t)e * 25 + q];
                    if (p < 0 || p >= fp_.n) throw Error(AXG_E_ARG, "FluidElement::FluidElement || point index out of range.");
                    pts[(size_t)k * 25 + q] = p;
                }
                const double *g = &h.geom[(size_t)e * 150];
                for (int c = 0; c < 5; c++)
                    for (int q = 0; q < 25; q++) {
                        geom[(size_t)k * 250 + c * 25 + q] = (T)g[c * 25 + q];
                        geom[(size_t)k * 250 + 125 + c * 25 + q] = (T)(g[c * 25 + q] * g[125 + q]);
                    }
                koff[k] = (int64_t)K.size();
                const double *mm = &h.moduli[h.mat_off[e]];
                for (int i = 0; i < ns * 25; i++) K.push_back((T)mm[i]);
                double s = sizeof(T);
                bytes += 6 * 25 * s + 25 * 4 + 8 + (double)ns * 25 * s;
                if (b->prt) {
                    const int i = prt_of[e];
                    const int xns = hp.x3d[i] ? enr : 1;
                    const size_t xs = (size_t)xns * 25;
                    const double *x = &hp.x[hp.off[i]];
                    xoff.push_back((int64_t)xpool.size());
                    x3d.push_back(hp.x3d[i]);
                    for (int c = 0; c < 4; c++)
                        for (size_t j = 0; j < xs; j++) xpool.push_back((T)x[c * xs + j]);
                    for (int c = 0; c < 4; c++)
                        for (size_t j = 0; j < xs; j++) xpool.push_back((T)(x[c * xs + j] * x[4 * xs + j]));
                    bytes += 8.0 * xs * s;
                    if (b->prt == 2) {
                        // CoordTransformSpherical constructor: sin / cos of theta, cast
                        for (int q = 0; q < 25; q++) trig.push_back((T)std::sin(hp.theta[(size_t)i * 25 + q]));
                        for (int q = 0; q < 25; q++) trig.push_back((T)std::cos(hp.theta[(size_t)i * 25 + q]));
                    }
                } else {
                    xoff.push_back(0);
                    x3d.push_back(0);
                }
                flops += (double)enu * 25 * 2 * (10 * 4 + 20);
                if (b->is3d) flops += 2.0 * 75 * enr * enu * 4;
            }
            b->bytes = bytes;
            b->flops = flops;
            b->nr.upload(nr); b->pts.upload(pts); b->axial.upload(ax);
            b->geom.upload(geom);
            if (K.empty()) K.push_back((T)0);
            b->K.upload(K); b->K_off.upload(koff);
            if (xpool.empty()) xpool.push_back((T)0);
            if (trig.empty()) trig.push_back((T)0);
            b->xpool.upload(xpool); b->xoff.upload(xoff); b->x3d.upload(x3d); b->trig.upload(trig);
            if (b->is3d)
                b->kernel = b->prt == 0 ? (FluidKernel)fluid_stiffness_kernel<T, true, 0>
                          : b->prt == 1 ? (FluidKernel)fluid_stiffness_kernel<T, true, 1>
                                        : (FluidKernel)fluid_stiffness_kernel<T, true, 2>;
            else
                b->kernel = b->prt == 0 ? (FluidKernel)fluid_stiffness_kernel<T, false, 0>
                          : b->prt == 1 ? (FluidKernel)fluid_stiffness_kernel<T, false, 1>
                                        : (FluidKernel)fluid_stiffness_kernel<T, false, 2>;
            int team = cfg_.plain ? 256 : (team_override_[b->cls] ? team_override_[b->cls] : default_team(b->cls));
            TeamLayout L = fluid_layout<T>(b->nr_max);
            if (L.total > 200 * 1024)
                throw Error(AXG_E_UNSUPPORTED, "FluidElement || nr too large for shared memory.");
            b->team = team;
            b->team_bytes = L.total;
            int tpc = std::max(1, 256 / team);
            while (tpc > 1 && (size_t)tpc * L.total > 200 * 1024) tpc--;
            if (team > 32) tpc = std::min(tpc, 15);
            b->tpc = tpc;
            raise_smem_limit((const void *)b->kernel, tpc * L.total);
            fb_.push_back(std::move(b));
        }
    }

    // ------------------------------------------------- coupling / sources ---
    void build_coupling(const HostCoupling &h) {
        cp_n_ = h.count;
        if (!cp_n_) return;
        std::vector<T> nsu(cp_n_), nzu(cp_n_), nsa(cp_n_), nza(cp_n_);
        for (int i = 0; i < cp_n_; i++) {
            // SolidFluidCoupling1D: normals cast to Real, assembled normals / fluid mass
            nsu[i] = (T)h.nsu[i]; nzu[i] = (T)h.nzu[i];
            nsa[i] = (T)(h.nsa[i] / h.mf[i]); nza[i] = (T)(h.nza[i] / h.mf[i]);
            if (sp_.h_nu[h.sp[i]] != fp_.h_nu[h.fp[i]])
                throw Error(AXG_E_ARG, "SolidFluidCoupling::SolidFluidCoupling || coupled points differ in nr.");
        }
        cp_sp_.upload(h.sp); cp_fp_.upload(h.fp);
        cp_nsu_.upload(nsu); cp_nzu_.upload(nzu); cp_nsa_.upload(nsa); cp_nza_.upload(nza);
    }

    void build_abc(const HostModel &m) {
        // ClaytonSolid1D / ClaytonFluid1D constructors: coefficients in double, cast to Real
        auto solid = [&](const HostClayton &h) {
            std::vector<T> c((size_t)4 * h.count);
            for (int i = 0; i < h.count; i++) {
                const double ct = std::cos(h.theta[i]), st = std::sin(h.theta[i]);
                const double rsa = h.rvs[i] * h.area[i], rpa = h.rvp[i] * h.area[i];
                c[4 * i] = (T)(rsa * ct * ct + rpa * st * st);
                c[4 * i + 1] = (T)(rsa * st * st + rpa * ct * ct);
                c[4 * i + 2] = (T)((rpa - rsa) * ct * st);
                c[4 * i + 3] = (T)rsa;
            }
            return c;
        };
        // group conditions per point, keeping the given order within a point
        auto group = [](const std::vector<int> &pt, int ncoef, const std::vector<T> &c, DBuf<int> &upt,
                        DBuf<int> &first, DBuf<T> &cdev) {
            std::vector<int> idx(pt.size());
            for (size_t i = 0; i < idx.size(); i++) idx[i] = (int)i;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return pt[x] < pt[y]; });
            std::vector<int> u, f;
            std::vector<T> cs;
            for (size_t k = 0; k < idx.size(); k++) {
                if (k == 0 || pt[idx[k]] != pt[idx[k - 1]]) { u.push_back(pt[idx[k]]); f.push_back((int)k); }
                for (int j = 0; j < ncoef; j++) cs.push_back(c[(size_t)idx[k] * ncoef + j]);
            }
            f.push_back((int)idx.size());
            upt.upload(u); first.upload(f); cdev.upload(cs);
            return (int)u.size();
        };
        cls_n_ = m.cl_s.count ? group(m.cl_s.pt, 4, solid(m.cl_s), cls_pt_, cls_first_, cls_c_) : 0;
        clf_n_ = 0;
        if (m.cl_f.count) {
            std::vector<T> c(m.cl_f.count);
            for (int i = 0; i < m.cl_f.count; i++) c[i] = (T)(m.cl_f.area[i] / m.cl_f.rvp[i]);
            clf_n_ = group(m.cl_f.pt, 1, c, clf_pt_, clf_first_, clf_c_);
        }
        auto sponge = [&](const HostSponge &h, int np, DBuf<T> &out) {
            if (!h.count) return;
            std::vector<T> g(np, (T)0);
            for (int i = 0; i < h.count; i++) g[h.pt[i]] = (T)h.gamma[i];
            out.upload(g);
        };
        sponge(m.sg_s, sp_.n, sg_s_);
        sponge(m.sg_f, fp_.n, sg_f_);
        // 3-D Clayton (ClaytonSolid3D / ClaytonFluid3D constructors: in double, cast), grouped
        // per point in the given order, per-slice coefficients of each condition in a pool
        auto clay3 = [&](const HostClayton3D &h, const HostPoints &hp, bool solid, Abc3D &out) {
            out.n = 0;
            if (!h.count) return;
            std::vector<int> idx(h.count);
            for (int i = 0; i < h.count; i++) idx[i] = i;
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return h.pt[x] < h.pt[y]; });
            std::vector<int> u, first;
            std::vector<int64_t> coff;
            std::vector<T> c;
            for (int k = 0; k < h.count; k++) {
                const int i = idx[k], p = h.pt[i], nr = hp.nr[p];
                if (k == 0 || p != h.pt[idx[k - 1]]) { u.push_back(p); first.push_back(k); }
                coff.push_back((int64_t)c.size());
                for (int j = 0; j < nr; j++) {
                    const int64_t q = h.off[i] + j;
                    if (solid) {
                        const double rsa = h.rvs[q] * h.area[q];
                        const double sk = std::sqrt((h.rvp[q] - h.rvs[q]) * h.area[q]);
                        c.push_back((T)rsa);
                        for (int d = 0; d < 3; d++) c.push_back((T)(sk * h.normal[q * 3 + d]));
                    } else {
                        c.push_back((T)(h.area[q] / h.rvp[q]));
                    }
                }
            }
            first.push_back(h.count);
            out.n = (int)u.size();
            out.pt.upload(u); out.first.upload(first); out.coff.upload(coff); out.c.upload(c);
        };
        clay3(m.cl3_s, m.sp, true, cl3_s_);
        clay3(m.cl3_f, m.fp, false, cl3_f_);
        auto sponge3 = [&](const HostSponge3D &h, const HostPoints &hp, Abc3D &out) {
            out.n = h.count;
            if (!h.count) return;
            std::vector<int64_t> goff;
            std::vector<T> g;
            for (int i = 0; i < h.count; i++) {
                goff.push_back((int64_t)g.size());
                for (int j = 0; j < hp.nr[h.pt[i]]; j++) g.push_back((T)h.gamma[h.off[i] + j]);
            }
            out.pt.upload(h.pt); out.coff.upload(goff); out.c.upload(g);
        };
        sponge3(m.sg3_s, m.sp, sg3_s_);
        sponge3(m.sg3_f, m.fp, sg3_f_);
    }

    void launch_clayton() {
        for (int solid = 1; solid >= 0; solid--) {
            PointDev &P = solid ? sp_ : fp_;
            const int n = solid ? cls_n_ : clf_n_;
            if (n) {
                ClaytonArgs<T, D> a;
                a.n = n; a.ndim = P.ndim; a.pt = solid ? cls_pt_.p : clf_pt_.p; a.off = P.off.p; a.nu = P.nu.p;
                a.first = solid ? cls_first_.p : clf_first_.p;
                a.c = solid ? cls_c_.p : clf_c_.p; a.veloc = P.veloc.p; a.stiff = P.stiff.p;
                a.nwave = nwave_; a.fstride = (size_t)P.total * P.ndim;
                clayton_kernel<T, D><<<(n * 32 + 255) / 256, 256, 0, stream_>>>(a);
                post_launch();
            }
            Abc3D &c3 = solid ? cl3_s_ : cl3_f_;
            if (c3.n) {
                Clayton3DArgs<T, D> a;
                a.n = c3.n; a.ndim = P.ndim; a.pt = c3.pt.p; a.first = c3.first.p; a.coff = c3.coff.p;
                a.c = c3.c.p; a.nr = P.nr.p; a.off = P.off.p; a.tw = tw_.p; a.tw_off = tw_off_.p;
                a.veloc = P.veloc.p; a.stiff = P.stiff.p; a.nr_max = P.nr_max; a.nwave = nwave_;
                a.fstride = (size_t)P.total * P.ndim;
                const int wpb = 4;
                clayton3d_kernel<T, D><<<(c3.n * nwave_ + wpb - 1) / wpb, 32 * wpb,
                                         (size_t)wpb * 6 * P.nr_max * sizeof(T), stream_>>>(a);
                post_launch();
            }
        }
    }

    static_assert(AXG_SCAN_CAP == AXG_SCAN_MAX_PEAKS, "scanning capacity must match the header");
    void build_scanning(const HostModel &m) {
        if (!m.scan.enabled) return;
        if (nwave_ != 1) throw Error(AXG_E_UNSUPPORTED, "WavefieldScanning || one wavefield per handle.");
        auto one = [&](bool all, const std::vector<int> &pts, const PointDev &P, ScanDev &S) {
            S.h_pt.clear();
            if (all) for (int p = 0; p < P.n; p++) S.h_pt.push_back(p);
            else S.h_pt = pts;
            S.n = (int)S.h_pt.size();
            if (!S.n) return;
            const size_t mm = (size_t)S.n * P.ndim;
            S.pt.upload(S.h_pt);
            S.cnt.alloc(mm); S.cnt.zero(stream_);
            S.nu1.alloc(mm * AXG_SCAN_CAP); S.nu1.zero(stream_);
            S.h2p.alloc(mm); S.h2p.zero(stream_);
            S.h2pp.alloc(mm); S.h2pp.zero(stream_);
            S.key.alloc(mm * AXG_SCAN_CAP); S.key.zero(stream_);
        };
        one(m.scan.all_solid, m.scan.solid_pts, sp_, scan_s_);
        one(m.scan.all_fluid, m.scan.fluid_pts, fp_, scan_f_);
    }

    // Domain::doScanning (Domain.cpp:466-490) at the device's current step
    void launch_scan() {
        const HostScanning &h = model_.scan;
        if (!h.enabled) return;
        for (int solid = 1; solid >= 0; solid--) {
            ScanDev &S = solid ? scan_s_ : scan_f_;
            PointDev &P = solid ? sp_ : fp_;
            if (!S.n) continue;
            ScanArgs<T, D> a;
            a.n = S.n; a.ndim = P.ndim; a.pt = S.pt.p; a.off = P.off.p; a.nr = P.nr.p; a.displ = P.displ.p;
            // WavefieldScanning stores squared tolerances in double; doScanning takes Real
            a.tol_fourier_h2 = (T)(h.tol_fourier_h1 * h.tol_fourier_h1);
            a.rel_tol_h2 = (T)(h.rel_tol_h1 * h.rel_tol_h1);
            a.abs_tol_h2 = (T)(h.abs_tol_h1 * h.abs_tol_h1);
            a.max_peaks = std::min(h.max_peaks, AXG_SCAN_CAP);
            a.interval = h.interval;
            a.step = step_dev_.p;
            a.h2p = S.h2p.p; a.h2pp = S.h2pp.p; a.cnt = S.cnt.p; a.key = S.key.p; a.nu1 = S.nu1.p;
            const int m = S.n * P.ndim;
            scan_kernel<T, D><<<(m + 255) / 256, 256, 0, stream_>>>(a);
            post_launch();
        }
    }

    void scanning_nr(int32_t *solid_nr, int32_t *fluid_nr) override {
        need();
        for (int solid = 1; solid >= 0; solid--) {
            int32_t *out = solid ? solid_nr : fluid_nr;
            if (!out) continue;
            PointDev &P = solid ? sp_ : fp_;
            ScanDev &S = solid ? scan_s_ : scan_f_;
            for (int p = 0; p < P.n; p++) out[p] = -1;
            if (!S.n) continue;
            const size_t mm = (size_t)S.n * P.ndim;
            std::vector<int> cnt(mm), nu1(mm * AXG_SCAN_CAP);
            AXG_CUDA(cudaStreamSynchronize(stream_));
            AXG_CUDA(cudaMemcpy(cnt.data(), S.cnt.p, mm * sizeof(int), cudaMemcpyDeviceToHost));
            AXG_CUDA(cudaMemcpy(nu1.data(), S.nu1.p, mm * AXG_SCAN_CAP * sizeof(int), cudaMemcpyDeviceToHost));
            for (int i = 0; i < S.n; i++) {
                const int p = S.h_pt[i];
                int best = 1;
                for (int c = 0; c < P.ndim; c++) {
                    const size_t t = (size_t)i * P.ndim + c;
                    int r = 1;   // reportScanningNr: 1 without candidates
                    if (cnt[t] > 0) {
                        int nu = 0;
                        for (int k = 0; k < cnt[t]; k++) nu = std::max(nu, nu1[(size_t)k * mm + t]);
                        r = std::min(nu * 2 + 1, P.h_nr[p]);
                    }
                    best = std::max(best, r);
                }
                out[p] = best;
            }
        }
    }

    void launch_sponge3d(PointDev &P, Abc3D &g) {
        Sponge3DArgs<T, D> a;
        a.n = g.n; a.ndim = P.ndim; a.pt = g.pt.p; a.goff = g.coff.p; a.gamma = g.c.p; a.nr = P.nr.p;
        a.off = P.off.p; a.tw = tw_.p; a.tw_off = tw_off_.p; a.veloc = P.veloc.p; a.displ = P.displ.p;
        a.stiff = P.stiff.p; a.nr_max = P.nr_max; a.nwave = nwave_; a.fstride = (size_t)P.total * P.ndim;
        const int wpb = 4;
        sponge3d_kernel<T, D><<<(g.n * nwave_ + wpb - 1) / wpb, 32 * wpb, (size_t)wpb * 3 * P.nr_max * sizeof(T),
                                stream_>>>(a);
        post_launch();
    }

    void build_pressure_sources(const HostSources &ps) {
        ps_n_ = ps.count;
        if (!ps_n_) return;
        for (int i = 0; i < ps.count; i++)
            if (ps.elem[i] < 0 || ps.elem[i] >= model_.fe.count)
                throw Error(AXG_E_ARG, "FluidPressure::FluidPressure || element index out of range.");
        ps_el_.upload(ps.elem); ps_nu_.upload(ps.nu); ps_wave_.upload(ps.wave);
        std::vector<int64_t> off(ps.pat_off.begin(), ps.pat_off.end());
        ps_po_.upload(off);
        std::vector<C> p(std::max<size_t>(ps.pattern.size() / 2, 1), mk<T>(0, 0));
        for (size_t i = 0; i < ps.pattern.size() / 2; i++) p[i] = mk<T>((T)ps.pattern[2 * i], (T)ps.pattern[2 * i + 1]);
        ps_pat_.upload(p);
        fe_pts_.upload(model_.fe.pts);
    }

    void build_sources(const HostSources &ms, const HostSources &fs) {
        auto conv = [](const HostSources &h, DBuf<int> &el, DBuf<int> &nu, DBuf<int64_t> &po,
                       DBuf<C> &pat) {
            el.upload(h.elem); nu.upload(h.nu);
            std::vector<int64_t> off(h.count);
            for (int i = 0; i < h.count; i++) off[i] = h.pat_off[i];
            po.upload(off);
            std::vector<C> p(h.pattern.size() / 2);
            for (size_t i = 0; i < p.size(); i++) p[i] = mk<T>((T)h.pattern[2 * i], (T)h.pattern[2 * i + 1]);
            if (p.empty()) p.push_back(mk<T>(0, 0));
            pat.upload(p);
        };
        ms_n_ = ms.count;
        fs_n_ = fs.count;
        if (ms_n_) { conv(ms, ms_el_, ms_nu_, ms_po_, ms_pat_); ms_wave_.upload(ms.wave); }
        if (fs_n_) { conv(fs, fs_el_, fs_nu_, fs_po_, fs_pat_); fs_wave_.upload(fs.wave); }
        for (int i = 0; i < ms.count; i++)
            if (ms.elem[i] < 0 || ms.elem[i] >= model_.se.count)
                throw Error(AXG_E_ARG, "SolidMoment::SolidMoment || element index out of range.");
        // element lookup tables in original order for the source kernels
        if (ms_n_ || fs_n_ || model_.st.count) upload_elem_tables(ms_n_ || model_.st.gradient);
    }

    // solid-element tables in the model's order for the source, station and element-record
    // kernels: nr, points, axial flags and, when asked, the geometry [e][250] (the first
    // five 25-rows of the element's geometry, then the same scaled by the last row)
    void upload_elem_tables(bool geom) {
        const HostSolidElements &h = model_.se;
        if (!e_nr_.n && h.count) {
            e_nr_.upload(h.nr); e_pts_.upload(h.pts);
            std::vector<uint8_t> ax(h.axial.begin(), h.axial.end());
            e_axial_.upload(ax);
        }
        if (geom && !e_geom_.n && h.count) {
            std::vector<T> g((size_t)h.count * 250);
            for (int e = 0; e < h.count; e++)
                for (int c = 0; c < 5; c++)
                    for (int q = 0; q < 25; q++) {
                        g[(size_t)e * 250 + c * 25 + q] = (T)h.geom[(size_t)e * 150 + c * 25 + q];
                        g[(size_t)e * 250 + 125 + c * 25 + q] =
                            (T)(h.geom[(size_t)e * 150 + c * 25 + q] * h.geom[(size_t)e * 150 + 125 + q]);
                    }
            e_geom_.upload(g);
        }
    }

    void build_stations(const HostStations &h) {
        st_n_ = h.count;
        st_interval_ = std::max(1, h.interval);
        if (!st_n_) return;
        st_el_.upload(h.elem);
        std::vector<T> w(h.w.size()), phi(h.phi.size());
        for (size_t i = 0; i < w.size(); i++) w[i] = (T)h.w[i];
        for (size_t i = 0; i < phi.size(); i++) phi[i] = (T)h.phi[i];
        st_w_.upload(w); st_phi_.upload(phi);
    }

    // STF table and seismogram buffer large enough for steps [0, nsteps)
    void ensure_capacity(int nsteps) {
        bool changed = false;
        if ((ms_n_ || fs_n_ || ps_n_) && nsteps > stf_valid_) {
            int cap = std::max(nsteps, 2 * stf_cap_);
            fill_stf(cap, nsteps);
            changed = true;
        }
        if (st_n_) {
            int need_rec = (nsteps + st_interval_ - 1) / st_interval_;
            if (need_rec > seis_cap_) {
                int cap = std::max(need_rec, 2 * seis_cap_);
                DBuf<double> nb;
                nb.alloc((size_t)cap * nwave_ * st_n_ * 3);
                nb.zero(stream_);
                if (seis_cap_)
                    AXG_CUDA(cudaMemcpyAsync(nb.p, seis_.p, (size_t)seis_cap_ * nwave_ * st_n_ * 3 * sizeof(double),
                                             cudaMemcpyDeviceToDevice, stream_));
                AXG_CUDA(cudaStreamSynchronize(stream_));
                std::swap(seis_.p, nb.p); std::swap(seis_.n, nb.n);
                if (model_.st.gradient) {
                    DBuf<double> ng;
                    ng.alloc((size_t)cap * nwave_ * st_n_ * 9);
                    ng.zero(stream_);
                    if (seis_cap_)
                        AXG_CUDA(cudaMemcpyAsync(ng.p, seis_grad_.p,
                                                 (size_t)seis_cap_ * nwave_ * st_n_ * 9 * sizeof(double),
                                                 cudaMemcpyDeviceToDevice, stream_));
                    AXG_CUDA(cudaStreamSynchronize(stream_));
                    std::swap(seis_grad_.p, ng.p); std::swap(seis_grad_.n, ng.n);
                }
                seis_cap_ = cap;
                changed = true;
            }
        }
        if (changed && graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    }
    static T src_stf(const HostSources &h, int i, double t) {
        auto it = h.table.find(i);
        return it == h.table.end() ? (T)stf_value(h.stf[i], t) : stf_table_value<T>(it->second, t);
    }
    static double stf_value(const axg_stf &s, double time) {
        // GaussianSTF::getValue (GaussianSTF.hpp:35-58)
        const double invSqrtPi = 1. / std::sqrt(M_PI);
        const double f = s.decay_factor / s.half_duration;
        double t = time - s.time_shift, ft = f * t;
        switch (s.derivative_order) {
            case -1: return std::erf(ft) * 0.5 + 0.5;
            case 0: return invSqrtPi * f * std::exp(-ft * ft);
            case 1: return invSqrtPi * std::pow(f, 3) * std::exp(-ft * ft) * (-2. * t);
            case 2: return invSqrtPi * std::pow(f, 3) * std::exp(-ft * ft) * (4. * ft * ft - 2.);
        }
        throw Error(AXG_E_ARG, "GaussianSTF::getValue || Unsupported derivative order.");
    }
    // Steps [0, need) must evaluate: a table source without padding throws there as
    // StreamSTF::getValue does when the run asks for a time out of its range. The steps
    // [need, cap) are evaluated ahead only as far as every source is defined; the table is
    // valid up to the first step that is not (slots after it stay zero and are never read,
    // ensure_capacity refills before a run needs them).
    void fill_stf(int cap, int need) {
        // t accumulated as NewmarkTimeScheme::solve does (t += mDt)
        std::vector<T> ms((size_t)cap * std::max(ms_n_, 1), (T)0), fs((size_t)cap * std::max(fs_n_, 1), (T)0),
            ps((size_t)cap * std::max(ps_n_, 1), (T)0);
        double t = cfg_.t0;
        int valid = cap;
        for (int k = 0; k < cap; k++) {
            try {
                for (int i = 0; i < ms_n_; i++) ms[(size_t)k * ms_n_ + i] = src_stf(model_.ms, i, t);
                for (int i = 0; i < fs_n_; i++) fs[(size_t)k * fs_n_ + i] = src_stf(model_.fs, i, t);
                for (int i = 0; i < ps_n_; i++) ps[(size_t)k * ps_n_ + i] = src_stf(model_.ps, i, t);
            } catch (const Error &) {
                if (k < need) throw;
                for (int i = 0; i < ms_n_; i++) ms[(size_t)k * ms_n_ + i] = (T)0;
                for (int i = 0; i < fs_n_; i++) fs[(size_t)k * fs_n_ + i] = (T)0;
                for (int i = 0; i < ps_n_; i++) ps[(size_t)k * ps_n_ + i] = (T)0;
                valid = k;
                break;
            }
            t += cfg_.dt;
        }
        ms_stf_.upload(ms);
        fs_stf_.upload(fs);
        ps_stf_.upload(ps);
        stf_cap_ = cap;
        stf_valid_ = valid;
    }

    // ------------------------------------------------------------ launches ---
    void launch_sources() {
        if ((ms_n_ || fs_n_) && stf_cap_ <= 0)
            throw Error(AXG_E_STATE, "Domain::applySources || source-time table not allocated.");
        if (ms_n_) {
            MomentArgs<T> a;
            a.nsrc = ms_n_; a.elem = ms_el_.p; a.nu = ms_nu_.p; a.pat_off = ms_po_.p;
            a.pattern = ms_pat_.p; a.stf = ms_stf_.p; a.stf_steps = stf_cap_; a.step = step_dev_.p;
            a.e_nr = e_nr_.p; a.e_pts = e_pts_.p; a.e_axial = e_axial_.p; a.e_geom = e_geom_.p;
            a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p; a.stiff = sp_.stiff.p; a.gmat = gmat_.p;
            a.wave = ms_wave_.p; a.fstride = (size_t)sp_.total * 3;
            moment_source_kernel<T><<<ms_n_, 128, 0, stream_>>>(a);
            post_launch();
        }
        if (fs_n_) {
            ForceArgs<T> a;
            a.nsrc = fs_n_; a.elem = fs_el_.p; a.nu = fs_nu_.p; a.pat_off = fs_po_.p;
            a.pattern = fs_pat_.p; a.stf = fs_stf_.p; a.stf_steps = stf_cap_; a.step = step_dev_.p;
            a.e_pts = e_pts_.p; a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p; a.stiff = sp_.stiff.p;
            a.wave = fs_wave_.p; a.fstride = (size_t)sp_.total * 3;
            force_source_kernel<T><<<fs_n_, 128, 0, stream_>>>(a);
            post_launch();
        }
    }

    void launch_pressure_sources() {
        if (stf_cap_ <= 0)
            throw Error(AXG_E_STATE, "Domain::applySources || source-time table not allocated.");
        ForceArgs<T> a;
        a.nsrc = ps_n_; a.elem = ps_el_.p; a.nu = ps_nu_.p; a.pat_off = ps_po_.p;
        a.pattern = ps_pat_.p; a.stf = ps_stf_.p; a.stf_steps = stf_cap_; a.step = step_dev_.p;
        a.e_pts = fe_pts_.p; a.pt_off = fp_.off.p; a.pt_nu = fp_.nu.p; a.stiff = fp_.stiff.p;
        a.wave = ps_wave_.p; a.fstride = (size_t)fp_.total;
        pressure_source_kernel<T><<<ps_n_, 128, 0, stream_>>>(a);
        post_launch();
    }

    // every bucket (part < 0) or the buckets of one element part
    void launch_stiffness(int part = -1) {
        if (timing_) AXG_CUDA(cudaEventRecord(ev0_, stream_));
        for (auto &bp : sb_)
            if (part < 0 || bp->part == part) launch_solid_bucket(*bp);
        if (timing_) AXG_CUDA(cudaEventRecord(ev1_, stream_));
        launch_fluid(part);
    }

    void launch_solid_bucket(SolidBucket &b) {
        {
            SolidArgs<T, AT> a;
            a.n_elem = b.n; a.nr = b.nr.p; a.pts = b.pts.p; a.axial = b.axial.p;
            a.geom = b.geom.p; a.trig = b.trig.p; a.mod = b.mod.p; a.mod_off = b.mod_off.p;
            a.attmod = b.attmod.p; a.att_off = b.att_off.p; a.state = state_.p;
            a.state_off = b.state_off.p; a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p;
            a.displ = elem_displ(sp_); a.stiff = sp_.stiff.p; a.tw = tw_.p; a.tw_off = tw_off_.p;
            a.nsls = cfg_.nsls;
            for (int l = 0; l < 8; l++) {
                a.alpha[l] = (AT)cfg_.att_alpha[l]; a.beta[l] = (AT)cfg_.att_beta[l];
                a.gamma[l] = (AT)cfg_.att_gamma[l];
            }
            a.gmat = gmat_.p;
            a.nwave = nwave_;
            a.fstride = (size_t)sp_.total * 3;
            a.sstride = (size_t)state_wave_;
            launch_solid_args(b, a);
        }
    }

    // one solid bucket's kernel with the given arguments (the PRT kernel takes the bucket's
    // factors on top)
    void launch_solid_args(SolidBucket &b, const SolidArgs<T, AT> &a) {
        if (b.prt) {
            PrtArgs<T, AT> pa;
            pa.s = a; pa.x = b.xpool.p; pa.x_off = b.xoff.p; pa.x3d = b.x3d.p;
            b.pkernel<<<b.grid, b.team * b.tpc, b.tpc * b.team_bytes, stream_>>>(pa, b.nr_max, b.qc, b.tpc,
                                                                               b.team_bytes);
        } else {
            SolidArgs<T, AT> af = a;
            af.fft_min_nr = b.fft ? AXG_FFT_MIN_NR : 0;
            af.prefetch_ahead = b.ahead;
            b.kernel<<<b.grid, b.team * b.tpc, b.tpc * b.team_bytes, stream_>>>(af, b.nr_max, b.qc, b.mt, b.tpc,
                                                                              b.team_bytes);
        }
        post_launch();
    }

    void launch_fluid(int part = -1) {
        for (auto &bp : fb_) {
            FluidBucket &b = *bp;
            if (part >= 0 && b.part != part) continue;
            FluidArgs<T> a;
            a.n_elem = b.n; a.nr = b.nr.p; a.pts = b.pts.p; a.axial = b.axial.p; a.geom = b.geom.p;
            a.K = b.K.p; a.K_off = b.K_off.p; a.pt_off = fp_.off.p; a.pt_nu = fp_.nu.p;
            a.displ = elem_displ(fp_); a.stiff = fp_.stiff.p; a.tw = tw_.p; a.tw_off = tw_off_.p;
            a.gmat = gmat_.p;
            a.nwave = nwave_;
            a.fstride = (size_t)fp_.total;
            a.x = b.xpool.p; a.x_off = b.xoff.p; a.x3d = b.x3d.p; a.trig = b.trig.p;
            int blocks = (b.n + b.tpc - 1) / b.tpc;
            b.kernel<<<blocks, b.team * b.tpc, b.tpc * b.team_bytes, stream_>>>(a, b.nr_max, b.tpc,
                                                                              b.team_bytes);
            post_launch();
        }
    }

    void build_coupling3d(const HostModel &m) {
        const HostCoupling3D &h = m.sf3;
        cp3_n_ = h.count;
        if (!cp3_n_) return;
        int nrm = 1;
        for (int i = 0; i < h.count; i++) {
            if (h.sp[i] < 0 || h.sp[i] >= m.sp.count || h.fp[i] < 0 || h.fp[i] >= m.fp.count ||
                m.sp.nr[h.sp[i]] != m.fp.nr[h.fp[i]] || h.off[i] < 0 ||
                h.off[i] + m.sp.nr[h.sp[i]] > (int64_t)(h.nu3.size() / 3))
                throw Error(AXG_E_ARG, "SolidFluidCoupling3D::checkCompatibility || Incompatible sizes.");
            nrm = std::max(nrm, m.sp.nr[h.sp[i]]);
        }
        cp3_nr_max_ = nrm;
        cp3_sp_.upload(h.sp); cp3_fp_.upload(h.fp); cp3_off_.upload(h.off);
        std::vector<T> a(h.nu3.begin(), h.nu3.end()), b(h.na3.begin(), h.na3.end());
        cp3_nu_.upload(a); cp3_na_.upload(b);
    }

    void launch_coupling() {
        if (cp3_n_) {
            Coupling3DArgs<T> a;
            a.n = cp3_n_; a.sp = cp3_sp_.p; a.fp = cp3_fp_.p; a.coff = cp3_off_.p; a.nu3 = cp3_nu_.p;
            a.na3 = cp3_na_.p; a.s_off = sp_.off.p; a.s_nr = sp_.nr.p; a.f_off = fp_.off.p;
            a.tw = tw_.p; a.tw_off = tw_off_.p; a.s_displ = elem_displ(sp_); a.s_stiff = sp_.stiff.p;
            a.f_stiff = fp_.stiff.p; a.nr_max = cp3_nr_max_; a.nwave = nwave_;
            a.s_stride = (size_t)sp_.total * 3; a.f_stride = (size_t)fp_.total;
            const int wpb = 4;
            solid_fluid3d_kernel<T><<<(cp3_n_ * nwave_ + wpb - 1) / wpb, 32 * wpb,
                                      (size_t)wpb * 4 * cp3_nr_max_ * sizeof(T), stream_>>>(a);
            post_launch();
        }
        if (!cp_n_) return;
        CouplingArgs<T> a;
        a.n = cp_n_; a.sp = cp_sp_.p; a.fp = cp_fp_.p;
        a.nsu = cp_nsu_.p; a.nzu = cp_nzu_.p; a.nsa_m = cp_nsa_.p; a.nza_m = cp_nza_.p;
        a.s_off = sp_.off.p; a.f_off = fp_.off.p; a.f_nu = fp_.nu.p;
        a.s_displ = elem_displ(sp_); a.s_stiff = sp_.stiff.p; a.f_stiff = fp_.stiff.p;
        a.nwave = nwave_; a.s_stride = (size_t)sp_.total * 3; a.f_stride = (size_t)fp_.total;
        int threads = 256, blocks = (cp_n_ * 32 + threads - 1) / threads;
        solid_fluid_kernel<T><<<blocks, threads, 0, stream_>>>(a);
        post_launch();
    }

    void launch_stations() {
        if (!st_n_) return;
        StationArgs<T> a;
        a.nst = st_n_; a.elem = st_el_.p; a.w = st_w_.p; a.phi = st_phi_.p;
        a.e_nr = e_nr_.p; a.e_pts = e_pts_.p; a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p;
        a.displ = elem_displ(sp_); a.out = seis_.p; a.interval = st_interval_;
        a.max_rec = seis_cap_; a.step = step_dev_.p;
        a.nwave = nwave_; a.fstride = (size_t)sp_.total * 3;
        const int threads = 128;                          // four stations per block
        const int blocks = (int)(((size_t)st_n_ * nwave_ * 32 + threads - 1) / threads);
        station_kernel<T><<<blocks, threads, 0, stream_>>>(a);
        post_launch();
        if (model_.st.gradient) {
            StationGradArgs<T> g;
            g.nst = st_n_; g.elem = st_el_.p; g.w = st_w_.p; g.phi = st_phi_.p;
            g.e_nr = e_nr_.p; g.e_pts = e_pts_.p; g.e_axial = e_axial_.p; g.e_geom = e_geom_.p;
            g.gmat = gmat_.p; g.pt_off = sp_.off.p; g.pt_nu = sp_.nu.p; g.displ = elem_displ(sp_);
            g.out = seis_grad_.p; g.interval = st_interval_; g.max_rec = seis_cap_; g.step = step_dev_.p;
            g.nwave = nwave_; g.fstride = (size_t)sp_.total * 3;
            station_grad_kernel<T><<<blocks, threads, 0, stream_>>>(g);
            post_launch();
        }
    }

    void launch_element_record() {
        if (!er_n_) return;
        ElemRecordArgs<T> a;
        a.n = er_n_; a.elem = er_elem_.p; a.gll = er_gll_.p; a.kind = er_kind_.p; a.off = er_off_.p;
        a.words = er_words_; a.e_nr = e_nr_.p; a.e_pts = e_pts_.p; a.e_axial = e_axial_.p;
        a.e_geom = e_geom_.p; a.gmat = gmat_.p; a.pt_off = sp_.off.p; a.pt_nu = sp_.nu.p;
        a.displ = elem_displ(sp_); a.out = er_out_.p; a.interval = er_interval_; a.ring = er_ring_;
        a.step = step_dev_.p; a.nwave = nwave_; a.fstride = (size_t)sp_.total * 3;
        const int threads = 256;                          // eight entries per block
        const int blocks = (int)(((size_t)er_n_ * nwave_ * 32 + threads - 1) / threads);
        element_record_kernel<T><<<blocks, threads, 0, stream_>>>(a);
        post_launch();
    }

    void launch_points(int mask) {
        for (int solid = 1; solid >= 0; solid--) {
            PointDev &P = solid ? sp_ : fp_;
            if (!P.n) continue;
            if (P.n3d && (mask & 3)) {
                Mass3DArgs<T> a;
                a.n = P.n3d; a.pt = P.pt3d.p; a.nr = P.nr.p; a.off = P.off.p; a.flags = P.flags.p;
                a.inv_mass = P.inv3.p; a.im_off = P.im_off.p; a.tw = tw_.p; a.tw_off = tw_off_.p;
                a.stiff = P.stiff.p; a.ndim = P.ndim; a.solid = solid; a.nr_max = P.nr_max;
                a.nwave = nwave_; a.fstride = (size_t)P.total * P.ndim;
                a.mask = mask;
                int wpb = 4;
                mass3d_kernel<T><<<(P.n3d * nwave_ + wpb - 1) / wpb, 32 * wpb, wpb * P.nr_max * sizeof(T), stream_>>>(a);
                post_launch();
            }
            if (solid && ocean3_n_ && (mask & 3)) {
                Ocean3DArgs<T> o;
                o.n = ocean3_n_; o.pt = ocean3_pt_.p; o.coff = ocean3_coff_.p; o.c = ocean3_c_.p;
                o.nr = P.nr.p; o.off = P.off.p; o.flags = P.flags.p; o.tw = tw_.p; o.tw_off = tw_off_.p;
                o.stiff = P.stiff.p; o.nr_max = P.nr_max; o.nwave = nwave_;
                o.fstride = (size_t)P.total * P.ndim; o.mask = mask;
                const int wpb = 4;
                ocean3d_kernel<T><<<(ocean3_n_ * nwave_ + wpb - 1) / wpb, 32 * wpb,
                                    (size_t)wpb * 3 * P.nr_max * sizeof(T), stream_>>>(o);
                post_launch();
            }
            if (solid && ocean_n_ && (mask & 3)) {
                OceanArgs<T> o;
                o.n = ocean_n_; o.pt = ocean_pt_.p; o.c = ocean_c_.p; o.nr = P.nr.p; o.off = P.off.p;
                o.flags = P.flags.p; o.stiff = P.stiff.p; o.nwave = nwave_;
                o.fstride = (size_t)P.total * P.ndim; o.mask = mask;
                ocean_mass_kernel<T><<<(ocean_n_ * nwave_ * 32 + 255) / 256, 256, 0, stream_>>>(o);
                post_launch();
            }
            PointArgs<T, D> a;
            a.nmodes = P.total; a.ndim = P.ndim; a.solid = solid; a.mode_pt = P.mode_pt.p;
            a.off = P.off.p; a.nr = P.nr.p; a.flags = P.flags.p; a.inv_mass1 = P.inv1.p;
            a.stiff = P.stiff.p; a.accel = P.accel.p; a.displ = P.displ.p; a.veloc = P.veloc.p;
            a.cd = P.cd.p; a.cv = P.cv.p; a.displ_elem = P.displ_elem.p;
            if constexpr (sizeof(D) == sizeof(T)) {
                // NewmarkTimeScheme::update statics, formed in double then cast to Real
                a.dt = (D)cfg_.dt; a.half_dt = (D)(.5 * cfg_.dt); a.half_dt_dt = (D)(.5 * cfg_.dt * cfg_.dt);
            } else {
                a.dt = cfg_.dt; a.half_dt = .5 * cfg_.dt; a.half_dt_dt = .5 * cfg_.dt * cfg_.dt;
            }
            a.nonfinite = nonfinite_.p;
            a.mask = mask;
            a.nwave = nwave_;
            a.sponge = solid ? sg_s_.p : sg_f_.p;
            int threads = POINT_BLOCK, blocks = (int)(((int64_t)P.total * nwave_ * P.ndim + threads - 1) / threads);
            Abc3D &g3 = solid ? sg3_s_ : sg3_f_;
            const bool press = !solid && ps_n_ && (mask & 2);
            if ((g3.n || press) && (mask & 2)) {
                // a 3-D sponge and fluid pressure sources act on the acceleration between
                // 1/M and the update
                a.mask = mask & 3;
                point_update_kernel<T, D, COMP><<<blocks, threads, 0, stream_>>>(a);
                post_launch();
                if (g3.n) launch_sponge3d(P, g3);
                if (press) launch_pressure_sources();
                if (!(mask & 4)) continue;
                a.mask = 4;
            }
            point_update_kernel<T, D, COMP><<<blocks, threads, 0, stream_>>>(a);
            post_launch();
        }
    }

    void launch_step() {
        launch_sources();
        launch_stiffness();
        launch_clayton();
        launch_coupling();
        launch_stations();
        launch_element_record();
        launch_scan();
        launch_points(7);
        advance_step_kernel<T><<<1, 1, 0, stream_>>>(step_dev_.p);
        post_launch();
    }

    void post_launch() {
        launches_++;
        cudaError_t e = cudaPeekAtLastError();
        if (e != cudaSuccess)
            throw Error(AXG_E_CUDA, std::string("Engine::launch || ") + cudaGetErrorString(e));
    }

    void capture() {
        cudaGraph_t g;
        int64_t before = launches_;
        AXG_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            launch_step();
        } catch (...) {
            cudaStreamEndCapture(stream_, &g);
            throw;
        }
        AXG_CUDA(cudaStreamEndCapture(stream_, &g));
        kernels_per_step_ = launches_ - before;
        launches_ = before;
        AXG_CUDA(cudaGraphInstantiate(&graph_exec_, g, 0));
        cudaGraphDestroy(g);
    }

    // ---------------------------------------------------------------- data ---
    axg_config cfg_;
    HostModel model_;
    cudaDeviceProp prop_;
    cudaStream_t own_stream_ = nullptr, stream_ = nullptr;
    bool finalized_ = false;
    int step_ = 0, tstep_host_ = 0;
    int64_t launches_ = 0, kernels_per_step_ = 0;
    bool timing_ = false;
    double time_ms_ = 0;
    int64_t time_n_ = 0;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    int team_override_[kNrClasses];
    struct Tuned { int cls, team; float ms; };
    std::vector<Tuned> tuned_;
    // differentiation
    DBuf<CD> ck_displ_, ck_veloc_;
    DBuf<C> ck_accel_;
    int ck_n_ = 0, ck_interval_ = 0, ck_step0_ = 0;
    bool adj_built_ = false;
    int adj_nr_max_ = 1;
    bool adj_slices_ = false, adj_slices_built_ = false;
    int64_t adj_grad3_n_ = 0, adj_mass3_pairs_ = 0;
    DBuf<T> adj_grad3_, adj_gmass3_, adj_tw_;
    DBuf<int64_t> adj_grad3_off_, adj_gmass3_off_;
    DBuf<int> adj_tw_off_;
    DBuf<T> adj_geom_, adj_ifact_, adj_mod_, adj_grad_, adj_gmass_;
    DBuf<int64_t> adj_mod_off_, adj_grad_off_;
    DBuf<int> adj_rheo_;
    DBuf<uint8_t> adj_rtz_;
    DBuf<T> adj_trig_;
    int64_t adj_grad_n_ = 0, adj_astate_n_ = 0;
    DBuf<int> adj_att_;
    DBuf<T> adj_attmod_;
    DBuf<int64_t> adj_attmod_off_, adj_astate_off_;
    DBuf<C> adj_astate_;
    DBuf<AT> ck_state_;
    bool adj_generic_ = false, adj_iso_only_ = true, adj_3d_ = false;

    DBuf<T> gmat_, tw_;
    DBuf<int> tw_off_;
    PointDev sp_, fp_;
    std::vector<std::unique_ptr<SolidBucket>> sb_;
    std::vector<std::unique_ptr<FluidBucket>> fb_;
    DBuf<AT> state_;
    int cp_n_ = 0;
    DBuf<int> cp_sp_, cp_fp_;
    DBuf<T> cp_nsu_, cp_nzu_, cp_nsa_, cp_nza_;
    int ms_n_ = 0, fs_n_ = 0, stf_cap_ = 0, stf_valid_ = 0;
    DBuf<int> ms_el_, ms_nu_, fs_el_, fs_nu_, ms_wave_, fs_wave_;
    int nwave_ = 1;
    int64_t state_wave_ = 0;
    int cls_n_ = 0, clf_n_ = 0;
    Abc3D cl3_s_, cl3_f_, sg3_s_, sg3_f_;
    struct ScanDev {
        int n = 0;
        std::vector<int> h_pt;
        DBuf<int> pt, cnt, nu1;
        DBuf<T> h2p, h2pp, key;
    };
    ScanDev scan_s_, scan_f_;
    int ocean_n_ = 0, ocean3_n_ = 0;
    DBuf<int> ocean3_pt_;
    DBuf<int64_t> ocean3_coff_;
    DBuf<T> ocean3_c_;
    DBuf<int> ocean_pt_;
    DBuf<T> ocean_c_;
    DBuf<int> cls_pt_, clf_pt_, cls_first_, clf_first_;
    DBuf<T> cls_c_, clf_c_, sg_s_, sg_f_;
    DBuf<int64_t> ms_po_, fs_po_;
    DBuf<C> ms_pat_, fs_pat_;
    DBuf<T> ms_stf_, fs_stf_;
    DBuf<int> e_nr_, e_pts_;
    int ps_n_ = 0;
    int cp3_n_ = 0, cp3_nr_max_ = 1;
    DBuf<int> cp3_sp_, cp3_fp_;
    DBuf<int64_t> cp3_off_;
    DBuf<T> cp3_nu_, cp3_na_;
    DBuf<int> ps_el_, ps_nu_, ps_wave_, fe_pts_;
    DBuf<int64_t> ps_po_;
    DBuf<C> ps_pat_;
    DBuf<T> ps_stf_;
    DBuf<uint8_t> e_axial_;
    DBuf<T> e_geom_;
    int st_n_ = 0, st_interval_ = 1, seis_cap_ = 0;
    DBuf<int> st_el_;
    DBuf<T> st_w_, st_phi_;
    DBuf<double> seis_, seis_grad_;
    int er_n_ = 0, er_interval_ = 1, er_ring_ = 1;
    int64_t er_words_ = 0;
    DBuf<int> er_elem_, er_gll_, er_kind_;
    DBuf<int64_t> er_off_;
    DBuf<C> er_out_;
    DBuf<int> step_dev_, nonfinite_;
};

}  // namespace axg
