// capi.cpp -- the extern "C" boundary (include/axg.h). Copies the caller's
// arrays into the host model, validates them, and forwards to the engine. No
// exception crosses this boundary: every failure becomes an AXG_E_* code with a
// "Class::method || message" text available from axg_last_error().
#include "engine.hpp"

#include <cstring>
#include <string>

struct axg_solver {
    axg_config cfg;
    axg::HostModel model;
    std::unique_ptr<axg::EngineBase> eng;
    std::string err;
    bool finalized = false;
};

namespace {

thread_local std::string g_create_error;

template <class F>
int guarded(axg_solver *h, F &&f) {
    if (!h) return AXG_E_ARG;
    try {
        f();
        return AXG_OK;
    } catch (const axg::Error &e) {
        h->err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        h->err = e.what();
        return AXG_E_ARG;
    }
}

template <class X>
std::vector<X> copy(const X *p, size_t n) {
    return p ? std::vector<X>(p, p + n) : std::vector<X>();
}

void need_open(const axg_solver *h) {
    if (h->finalized) throw axg::Error(AXG_E_STATE, "axg_set || model already finalized.");
}

void points_from(axg::HostPoints &hp, int count, const int32_t *nr, const int32_t *mnr,
                 const int64_t *moff, const double *mass, const uint8_t *axial,
                 const uint8_t *surface, int ndim, const char *who) {
    if (count < 0 || (count && (!nr || !mass)))
        throw axg::Error(AXG_E_ARG, std::string(who) + " || missing nr or mass.");
    hp.count = count;
    hp.ndim = ndim;
    hp.nr = copy(nr, count);
    hp.mass_nr = copy(mnr, count);
    hp.mass_off = copy(moff, count);
    size_t nmass = 0;
    for (int p = 0; p < count; p++) {
        int m = mnr ? mnr[p] : 1;
        if (nr[p] < 1) throw axg::Error(AXG_E_ARG, std::string(who) + " || nr must be >= 1.");
        if (m != 1 && m != nr[p]) throw axg::Error(AXG_E_ARG, std::string(who) + " || mass_nr must be 1 or nr.");
        size_t end = (size_t)(moff ? moff[p] : p) + m;
        nmass = std::max(nmass, end);
        if (!moff && m != 1) throw axg::Error(AXG_E_ARG, std::string(who) + " || mass_offset required for 3-D mass.");
    }
    hp.mass = copy(mass, nmass);
    for (double v : hp.mass)
        if (!(v > 0)) throw axg::Error(AXG_E_ARG, std::string(who) + " || mass must be positive.");
    hp.axial = copy(axial, count);
    hp.surface = copy(surface, count);
}

int nmod(int rheo) { return rheo == AXG_ISO ? 2 : rheo == AXG_TISO ? 5 : 21; }

}  // namespace

extern "C" {

const char *axg_version(void) { return "axg 0.1 (sm_100a, nPol=4)"; }

int axg_create(const axg_config *cfg, axg_solver **out) {
    if (!cfg || !out) return AXG_E_ARG;
    *out = nullptr;
    if (cfg->precision < AXG_FP64 || cfg->precision > AXG_MIXED) return AXG_E_ARG;
    if (!(cfg->dt > 0) || cfg->nsls < 0 || cfg->nsls > AXG_MAX_SLS || cfg->nwave < 0) return AXG_E_ARG;
    axg_solver *h = new axg_solver();
    h->cfg = *cfg;
    try {
        switch (cfg->precision) {
            case AXG_FP32: h->eng = axg::make_engine_fp32(*cfg); break;
            case AXG_FP64: h->eng = axg::make_engine_fp64(*cfg); break;
            default: h->eng = axg::make_engine_mixed(*cfg); break;
        }
    } catch (const axg::Error &e) {
        g_create_error = e.what();
        delete h;
        return e.code;
    }
    *out = h;
    return AXG_OK;
}

int axg_destroy(axg_solver *h) {
    delete h;
    return AXG_OK;
}

const char *axg_last_error(const axg_solver *h) {
    return h ? h->err.c_str() : g_create_error.c_str();
}

int axg_set_solid_points(axg_solver *h, const axg_solid_points *p) {
    return guarded(h, [&] {
        need_open(h);
        if (!p) throw axg::Error(AXG_E_ARG, "SolidPoint || null description.");
        points_from(h->model.sp, p->count, p->nr, p->mass_nr, p->mass_offset, p->mass, p->axial,
                    nullptr, 3, "SolidPoint::SolidPoint");
    });
}

int axg_set_fluid_points(axg_solver *h, const axg_fluid_points *p) {
    return guarded(h, [&] {
        need_open(h);
        if (!p) throw axg::Error(AXG_E_ARG, "FluidPoint || null description.");
        points_from(h->model.fp, p->count, p->nr, p->mass_nr, p->mass_offset, p->mass, p->axial,
                    p->surface, 1, "FluidPoint::FluidPoint");
    });
}

int axg_set_solid_elements(axg_solver *h, const axg_solid_elements *e) {
    return guarded(h, [&] {
        need_open(h);
        const char *who = "SolidElement::SolidElement";
        if (!e || e->count < 0) throw axg::Error(AXG_E_ARG, std::string(who) + " || null description.");
        int n = e->count;
        if (n && (!e->nr || !e->points || !e->axial || !e->geometry || !e->rheology ||
                  !e->mat_offset || !e->moduli))
            throw axg::Error(AXG_E_ARG, std::string(who) + " || missing array.");
        axg::HostSolidElements &s = h->model.se;
        s.count = n;
        s.nr = copy(e->nr, n);
        s.pts = copy(e->points, (size_t)n * 25);
        s.axial = copy(e->axial, n);
        s.geom = copy(e->geometry, (size_t)n * 150);
        s.rtz = copy(e->rtz, n);
        s.rheo = copy(e->rheology, n);
        s.is3d = copy(e->is3d, n);
        s.att = copy(e->attenuation, n);
        s.mat_off = copy(e->mat_offset, n);
        s.att_off = copy(e->att_offset, n);
        bool any_rtz = false;
        size_t nm_end = 0, na_end = 0;
        for (int i = 0; i < n; i++) {
            if (s.nr[i] < 1) throw axg::Error(AXG_E_ARG, std::string(who) + " || nr must be >= 1.");
            if (s.rheo[i] < AXG_ISO || s.rheo[i] > AXG_ANISO)
                throw axg::Error(AXG_E_ARG, std::string(who) + " || unknown rheology.");
            int ns = (s.is3d.size() && s.is3d[i]) ? s.nr[i] : 1;
            nm_end = std::max(nm_end, (size_t)s.mat_off[i] + (size_t)nmod(s.rheo[i]) * ns * 25);
            int att = s.att.size() ? s.att[i] : AXG_ATT_NONE;
            if (att < AXG_ATT_NONE || att > AXG_ATT_CG4)
                throw axg::Error(AXG_E_ARG, std::string(who) + " || unknown attenuation.");
            if (att != AXG_ATT_NONE) {
                if (!e->att_offset || !e->att_moduli)
                    throw axg::Error(AXG_E_ARG, std::string(who) + " || attenuation arrays missing.");
                int npa = att == AXG_ATT_CG4 ? 4 : 25;
                na_end = std::max(na_end, (size_t)s.att_off[i] + (size_t)2 * ns * npa);
            }
            if (s.rtz.size() && s.rtz[i]) any_rtz = true;
            // the element's nr is the maximum over its points (Element::pointSet)
        }
        if (any_rtz && !e->theta) throw axg::Error(AXG_E_ARG, std::string(who) + " || theta required for RTZ.");
        s.theta = copy(e->theta, any_rtz ? (size_t)n * 25 : 0);
        s.moduli = copy(e->moduli, nm_end);
        s.att_moduli = copy(e->att_moduli, na_end);
    });
}

int axg_set_fluid_elements(axg_solver *h, const axg_fluid_elements *e) {
    return guarded(h, [&] {
        need_open(h);
        const char *who = "FluidElement::FluidElement";
        if (!e || e->count < 0) throw axg::Error(AXG_E_ARG, std::string(who) + " || null description.");
        int n = e->count;
        if (n && (!e->nr || !e->points || !e->axial || !e->geometry || !e->mat_offset || !e->moduli))
            throw axg::Error(AXG_E_ARG, std::string(who) + " || missing array.");
        axg::HostFluidElements &s = h->model.fe;
        s.count = n;
        s.nr = copy(e->nr, n);
        s.pts = copy(e->points, (size_t)n * 25);
        s.axial = copy(e->axial, n);
        s.geom = copy(e->geometry, (size_t)n * 150);
        s.is3d = copy(e->is3d, n);
        s.mat_off = copy(e->mat_offset, n);
        size_t end = 0;
        for (int i = 0; i < n; i++) {
            if (s.nr[i] < 1) throw axg::Error(AXG_E_ARG, std::string(who) + " || nr must be >= 1.");
            int ns = (s.is3d.size() && s.is3d[i]) ? s.nr[i] : 1;
            end = std::max(end, (size_t)s.mat_off[i] + (size_t)ns * 25);
        }
        s.moduli = copy(e->moduli, end);
    });
}

int axg_set_solid_fluid(axg_solver *h, const axg_solid_fluid *c) {
    return guarded(h, [&] {
        need_open(h);
        if (!c || c->count < 0) throw axg::Error(AXG_E_ARG, "SolidFluidCoupling || null description.");
        axg::HostCoupling &s = h->model.sf;
        int n = c->count;
        s.count = n;
        s.sp = copy(c->solid_point, n); s.fp = copy(c->fluid_point, n);
        s.nsu = copy(c->ns_unassembled, n); s.nzu = copy(c->nz_unassembled, n);
        s.nsa = copy(c->ns_assembled, n); s.nza = copy(c->nz_assembled, n);
        s.mf = copy(c->mass_fluid, n);
        if (n && (s.sp.empty() || s.fp.empty() || s.nsu.empty() || s.nzu.empty() || s.nsa.empty() ||
                  s.nza.empty() || s.mf.empty()))
            throw axg::Error(AXG_E_ARG, "SolidFluidCoupling || missing array.");
    });
}

static void sources_from(axg::HostSources &s, int n, const int32_t *el, const int32_t *nu,
                         const int64_t *po, const double *pat, const axg_stf *stf, const int32_t *wave,
                         int nwave, int ndim, const char *who) {
    if (n < 0 || (n && (!el || !nu || !po || !pat || !stf)))
        throw axg::Error(AXG_E_ARG, std::string(who) + " || missing array.");
    s.count = n;
    s.elem = copy(el, n);
    s.nu = copy(nu, n);
    s.pat_off = copy(po, n);
    s.stf = copy(stf, n);
    s.wave = wave ? copy(wave, n) : std::vector<int>(n, 0);
    for (int i = 0; i < n; i++)
        if (s.wave[i] < 0 || s.wave[i] >= nwave)
            throw axg::Error(AXG_E_ARG, std::string(who) + " || wavefield index out of range.");
    size_t end = 0;
    for (int i = 0; i < n; i++) {
        if (nu[i] < 1) throw axg::Error(AXG_E_ARG, std::string(who) + " || pattern needs >= 1 mode.");
        if (stf[i].derivative_order < -1 || stf[i].derivative_order > 2)
            throw axg::Error(AXG_E_ARG, "GaussianSTF::getValue || Unsupported derivative order.");
        end = std::max(end, (size_t)po[i] + (size_t)nu[i] * ndim * 25);
    }
    s.pattern = copy(pat, 2 * end);
}

int axg_set_moment_sources(axg_solver *h, const axg_moment_sources *s) {
    return guarded(h, [&] {
        need_open(h);
        if (!s) throw axg::Error(AXG_E_ARG, "SolidMoment || null description.");
        sources_from(h->model.ms, s->count, s->element, s->nu, s->pattern_offset, s->pattern, s->stf,
                     s->wavefield, std::max(1, h->cfg.nwave), 6, "SolidMoment::SolidMoment");
    });
}

int axg_set_force_sources(axg_solver *h, const axg_force_sources *s) {
    return guarded(h, [&] {
        need_open(h);
        if (!s) throw axg::Error(AXG_E_ARG, "SolidForce || null description.");
        sources_from(h->model.fs, s->count, s->element, s->nu, s->pattern_offset, s->pattern, s->stf,
                     s->wavefield, std::max(1, h->cfg.nwave), 3, "SolidForce::SolidForce");
    });
}

int axg_set_pressure_sources(axg_solver *h, const axg_pressure_sources *s) {
    return guarded(h, [&] {
        need_open(h);
        if (!s) throw axg::Error(AXG_E_ARG, "FluidPressure || null description.");
        sources_from(h->model.ps, s->count, s->element, s->nu, s->pattern_offset, s->pattern, s->stf,
                     s->wavefield, std::max(1, h->cfg.nwave), 1, "FluidPressure::FluidPressure");
    });
}

int axg_set_stf_table(axg_solver *h, int32_t kind, int32_t index, int32_t n, const double *times,
                      const double *values, int32_t padding, double left, double right, int32_t pad_first) {
    return guarded(h, [&] {
        need_open(h);
        if (kind < 0 || kind > 2 || !times || !values)
            throw axg::Error(AXG_E_ARG, "STF::buildInparam || bad STF table arguments.");
        axg::HostSources &src = kind == 0 ? h->model.ms : kind == 1 ? h->model.fs : h->model.ps;
        if (index < 0 || index >= src.count)
            throw axg::Error(AXG_E_ARG, "STF::buildInparam || source index out of range.");
        if (n < 2)
            throw axg::Error(AXG_E_ARG, "StreamSTF::StreamSTF || Insufficient time points, at least 2.");
        for (int i = 1; i < n; i++)
            if (!(times[i] > times[i - 1]))
                throw axg::Error(AXG_E_ARG, "StreamSTF::StreamSTF || Time points are not ascendingly sorted.");
        axg::HostStfTable tb;
        tb.t.assign(times, times + n);
        tb.v.assign(values, values + n);
        tb.padding = padding != 0;
        tb.left = left; tb.right = right;
        tb.pad_first = pad_first != 0;
        src.table[index] = tb;
    });
}

int axg_set_stations(axg_solver *h, const axg_stations *s, int32_t record_interval) {
    return guarded(h, [&] {
        need_open(h);
        if (!s || s->count < 0 || (s->count && (!s->element || !s->weights || !s->phi)))
            throw axg::Error(AXG_E_ARG, "StationSolid || missing array.");
        axg::HostStations &st = h->model.st;
        st.count = s->count;
        st.interval = record_interval > 0 ? record_interval : 1;
        st.elem = copy(s->element, s->count);
        st.w = copy(s->weights, (size_t)s->count * 25);
        st.phi = copy(s->phi, s->count);
    });
}

int axg_set_station_gradient(axg_solver *h, int32_t enable) {
    return guarded(h, [&] {
        need_open(h);
        h->model.st.gradient = enable ? 1 : 0;
    });
}

int axg_set_clayton(axg_solver *h, int32_t solid, const axg_clayton *c) {
    return guarded(h, [&] {
        need_open(h);
        if (!c || c->count < 0 || (c->count && (!c->point || !c->rho_vp || !c->area ||
                                                 (solid && (!c->rho_vs || !c->theta)))))
            throw axg::Error(AXG_E_ARG, "ClaytonSolid1D || missing array.");
        axg::HostClayton &x = solid ? h->model.cl_s : h->model.cl_f;
        x.count = c->count;
        x.pt = copy(c->point, c->count);
        x.rvp = copy(c->rho_vp, c->count);
        x.rvs = solid ? copy(c->rho_vs, c->count) : std::vector<double>(c->count, 0.);
        x.area = copy(c->area, c->count);
        x.theta = solid ? copy(c->theta, c->count) : std::vector<double>(c->count, 0.);
        for (int i = 0; i < c->count; i++)
            if (!solid && !(x.rvp[i] > 0)) throw axg::Error(AXG_E_ARG, "ClaytonFluid1D || rho vp must be positive.");
    });
}

int axg_set_sponge(axg_solver *h, int32_t solid, int32_t count, const int32_t *point, const double *gamma) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || (count && (!point || !gamma))) throw axg::Error(AXG_E_ARG, "Sponge || missing array.");
        axg::HostSponge &x = solid ? h->model.sg_s : h->model.sg_f;
        x.count = count;
        x.pt = copy(point, count);
        x.gamma = copy(gamma, count);
    });
}

int axg_set_clayton3d(axg_solver *h, int32_t solid, const axg_clayton3d *c) {
    return guarded(h, [&] {
        need_open(h);
        if (!c || c->count < 0 || c->nvalues < 0 ||
            (c->count && (!c->point || !c->offset || !c->rho_vp || !c->area ||
                          (solid && (!c->rho_vs || !c->normal)))))
            throw axg::Error(AXG_E_ARG, "ClaytonSolid3D || missing array.");
        axg::HostClayton3D &x = solid ? h->model.cl3_s : h->model.cl3_f;
        x.count = c->count;
        x.pt = copy(c->point, c->count);
        x.off = copy(c->offset, c->count);
        x.rvp = copy(c->rho_vp, c->nvalues);
        x.rvs = solid ? copy(c->rho_vs, c->nvalues) : std::vector<double>();
        x.area = copy(c->area, c->nvalues);
        x.normal = solid ? copy(c->normal, (size_t)c->nvalues * 3) : std::vector<double>();
    });
}

int axg_set_sponge3d(axg_solver *h, int32_t solid, int32_t count, const int32_t *point, const int64_t *offset,
                     int64_t nvalues, const double *gamma) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || nvalues < 0 || (count && (!point || !offset || !gamma)))
            throw axg::Error(AXG_E_ARG, "Sponge || missing array.");
        axg::HostSponge3D &x = solid ? h->model.sg3_s : h->model.sg3_f;
        x.count = count;
        x.pt = copy(point, count);
        x.off = copy(offset, count);
        x.gamma = copy(gamma, nvalues);
    });
}

int axg_set_prt(axg_solver *h, int32_t count, const int32_t *element, const int64_t *offset,
                const uint8_t *is3d_prt, int64_t nvalues, const double *x) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || nvalues < 0 || (count && (!element || !offset || !is3d_prt || !x)))
            throw axg::Error(AXG_E_ARG, "PRT || missing array.");
        axg::HostPrt &p = h->model.prt;
        p.count = count;
        p.elem = copy(element, count);
        p.off = copy(offset, count);
        p.x3d = copy(is3d_prt, count);
        p.x = copy(x, nvalues);
    });
}

int axg_set_prt_fluid(axg_solver *h, int32_t count, const int32_t *element, const int64_t *offset,
                      const uint8_t *is3d_prt, int64_t nvalues, const double *x, const double *theta) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || nvalues < 0 || (count && (!element || !offset || !is3d_prt || !x)))
            throw axg::Error(AXG_E_ARG, "PRT || missing array.");
        axg::HostPrt &p = h->model.prt_f;
        p.count = count;
        p.elem = copy(element, count);
        p.off = copy(offset, count);
        p.x3d = copy(is3d_prt, count);
        p.x = copy(x, nvalues);
        p.theta = theta ? copy(theta, (size_t)count * 25) : std::vector<double>();
    });
}

int axg_set_scanning(axg_solver *h, const axg_scanning *sc) {
    return guarded(h, [&] {
        need_open(h);
        if (!sc) throw axg::Error(AXG_E_ARG, "WavefieldScanning || missing parameters.");
        if (sc->interval < 1 || sc->max_num_peaks < 1 || !(sc->tol_fourier_h1 > 0) || !(sc->rel_tol_h1 >= 0) ||
            !(sc->abs_tol_h1 >= 0))
            throw axg::Error(AXG_E_ARG, "WavefieldScanning || invalid parameters.");
        if ((sc->n_solid > 0 && !sc->solid_points) || (sc->n_fluid > 0 && !sc->fluid_points))
            throw axg::Error(AXG_E_ARG, "WavefieldScanning || missing point list.");
        axg::HostScanning &x = h->model.scan;
        x.enabled = true;
        x.tol_fourier_h1 = sc->tol_fourier_h1; x.rel_tol_h1 = sc->rel_tol_h1; x.abs_tol_h1 = sc->abs_tol_h1;
        x.max_peaks = sc->max_num_peaks; x.interval = sc->interval;
        x.all_solid = sc->n_solid < 0; x.all_fluid = sc->n_fluid < 0;
        x.solid_pts = sc->n_solid > 0 ? copy(sc->solid_points, sc->n_solid) : std::vector<int>();
        x.fluid_pts = sc->n_fluid > 0 ? copy(sc->fluid_points, sc->n_fluid) : std::vector<int>();
    });
}

int axg_scanning_nr(axg_solver *h, int32_t *solid_nr, int32_t *fluid_nr) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_scanning_nr || axg_finalize not called.");
        h->eng->scanning_nr(solid_nr, fluid_nr);
    });
}

int axg_set_solid_fluid3d(axg_solver *h, int32_t count, const int32_t *solid_point, const int32_t *fluid_point,
                          const int64_t *offset, int64_t nvalues, const double *normal_u, const double *normal_a,
                          const double *mass_fluid) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || nvalues < 0 ||
            (count && (!solid_point || !fluid_point || !offset || !normal_u || !normal_a || !mass_fluid)))
            throw axg::Error(AXG_E_ARG, "SolidFluidCoupling3D || missing array.");
        axg::HostCoupling3D &x = h->model.sf3;
        x.count = count;
        x.sp = copy(solid_point, count);
        x.fp = copy(fluid_point, count);
        x.off = copy(offset, count);
        x.nu3.resize((size_t)nvalues * 3);
        x.na3.resize((size_t)nvalues * 3);
        for (int64_t k = 0; k < nvalues; k++)
            for (int c = 0; c < 3; c++) {
                x.nu3[(size_t)k * 3 + c] = normal_u[(size_t)k * 3 + c];
                x.na3[(size_t)k * 3 + c] = normal_a[(size_t)k * 3 + c] / mass_fluid[k];
            }
    });
}

int axg_set_ocean_load(axg_solver *h, int32_t count, const int32_t *point, const double *mass_ocean,
                       const double *theta) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || (count && (!point || !mass_ocean || !theta)))
            throw axg::Error(AXG_E_ARG, "MassOceanLoad1D || missing array.");
        axg::HostOcean &x = h->model.ocean;
        x.count = count;
        x.pt = copy(point, count);
        x.mass_ocean = copy(mass_ocean, count);
        x.theta = copy(theta, count);
    });
}

int axg_set_ocean_load3d(axg_solver *h, int32_t count, const int32_t *point, const int64_t *offset,
                         int64_t nvalues, const double *mass_ocean, const double *normal) {
    return guarded(h, [&] {
        need_open(h);
        if (count < 0 || nvalues < 0 || (count && (!point || !offset || !mass_ocean || !normal)))
            throw axg::Error(AXG_E_ARG, "MassOceanLoad3D || missing array.");
        axg::HostOcean3D &x = h->model.ocean3;
        x.count = count;
        x.pt = copy(point, count);
        x.off = copy(offset, count);
        x.mass_ocean = copy(mass_ocean, nvalues);
        x.normal = copy(normal, (size_t)nvalues * 3);
    });
}

int axg_finalize(axg_solver *h) {
    return guarded(h, [&] {
        need_open(h);
        axg::HostModel &m = h->model;
        for (int e = 0; e < m.se.count; e++)
            for (int q = 0; q < 25; q++) {
                int p = m.se.pts[(size_t)e * 25 + q];
                if (p < 0 || p >= m.sp.count)
                    throw axg::Error(AXG_E_ARG, "SolidElement::SolidElement || point index out of range.");
                if (m.sp.nr[p] > m.se.nr[e])
                    throw axg::Error(AXG_E_ARG, "Element::pointSet || element nr below a point's nr.");
            }
        for (int e = 0; e < m.fe.count; e++)
            for (int q = 0; q < 25; q++) {
                int p = m.fe.pts[(size_t)e * 25 + q];
                if (p < 0 || p >= m.fp.count)
                    throw axg::Error(AXG_E_ARG, "FluidElement::FluidElement || point index out of range.");
                if (m.fp.nr[p] > m.fe.nr[e])
                    throw axg::Error(AXG_E_ARG, "Element::pointSet || element nr below a point's nr.");
            }
        for (int i = 0; i < m.sf.count; i++)
            if (m.sf.sp[i] < 0 || m.sf.sp[i] >= m.sp.count || m.sf.fp[i] < 0 || m.sf.fp[i] >= m.fp.count)
                throw axg::Error(AXG_E_ARG, "SolidFluidCoupling || point index out of range.");
        for (const axg::HostSources *s : {&m.ms, &m.fs})
            for (int i = 0; i < s->count; i++)
                if (s->elem[i] < 0 || s->elem[i] >= m.se.count)
                    throw axg::Error(AXG_E_ARG, "SolidSource || element index out of range.");
        for (int i = 0; i < m.st.count; i++)
            if (m.st.elem[i] < 0 || m.st.elem[i] >= m.se.count)
                throw axg::Error(AXG_E_ARG, "StationSolid || element index out of range.");
        for (int i = 0; i < m.cl_s.count; i++)
            if (m.cl_s.pt[i] < 0 || m.cl_s.pt[i] >= m.sp.count)
                throw axg::Error(AXG_E_ARG, "ClaytonSolid1D || point index out of range.");
        for (int i = 0; i < m.cl_f.count; i++)
            if (m.cl_f.pt[i] < 0 || m.cl_f.pt[i] >= m.fp.count)
                throw axg::Error(AXG_E_ARG, "ClaytonFluid1D || point index out of range.");
        {
            // MassOceanLoad1D replaces a solid point's Mass1D: once per point, 1-D masses only
            std::vector<char> seen(m.sp.count, 0);
            for (int i = 0; i < m.ocean.count; i++) {
                const int p = m.ocean.pt[i];
                if (p < 0 || p >= m.sp.count)
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad1D || point index out of range.");
                if (seen[p]) throw axg::Error(AXG_E_ARG, "MassOceanLoad1D || point listed twice.");
                seen[p] = 1;
                if (m.sp.mass_nr.size() && m.sp.mass_nr[p] > 1)
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad1D || a Mass3D point needs a 3-D ocean load.");
                if (!(m.ocean.mass_ocean[i] >= 0))
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad1D || negative ocean mass.");
            }
            for (int i = 0; i < m.ocean3.count; i++) {
                const int p = m.ocean3.pt[i];
                if (p < 0 || p >= m.sp.count)
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad3D || point index out of range.");
                if (seen[p]) throw axg::Error(AXG_E_ARG, "MassOceanLoad3D || point listed twice.");
                seen[p] = 1;
                const int nr = m.sp.nr[p];
                if (m.sp.mass_nr.size() && m.sp.mass_nr[p] > 1 && m.sp.mass_nr[p] != nr)
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad3D::checkCompatibility || Incompatible sizes.");
                if (m.ocean3.off[i] < 0 || m.ocean3.off[i] + nr > (int64_t)m.ocean3.mass_ocean.size())
                    throw axg::Error(AXG_E_ARG, "MassOceanLoad3D::checkCompatibility || Incompatible sizes.");
                for (int k = 0; k < nr; k++)
                    if (!(m.ocean3.mass_ocean[m.ocean3.off[i] + k] >= 0))
                        throw axg::Error(AXG_E_ARG, "MassOceanLoad3D || negative ocean mass.");
            }
        }
        // 3-D conditions: nr values of the point from each offset
        for (int solid = 1; solid >= 0; solid--) {
            const axg::HostPoints &P = solid ? m.sp : m.fp;
            const axg::HostClayton3D &c = solid ? m.cl3_s : m.cl3_f;
            for (int i = 0; i < c.count; i++) {
                const int p = c.pt[i];
                if (p < 0 || p >= P.count)
                    throw axg::Error(AXG_E_ARG, "ClaytonSolid3D || point index out of range.");
                if (c.off[i] < 0 || c.off[i] + P.nr[p] > (int64_t)c.rvp.size())
                    throw axg::Error(AXG_E_ARG, "ClaytonSolid3D::checkCompatibility || Incompatible sizes.");
                for (int k = 0; k < P.nr[p]; k++)
                    if (!(c.rvp[c.off[i] + k] > 0))
                        throw axg::Error(AXG_E_ARG, "ClaytonFluid3D || rho vp must be positive.");
            }
            const axg::HostSponge3D &g = solid ? m.sg3_s : m.sg3_f;
            const axg::HostSponge &g1 = solid ? m.sg_s : m.sg_f;
            std::vector<char> seen(P.count, 0);
            for (int i = 0; i < g1.count; i++)
                if (g1.pt[i] >= 0 && g1.pt[i] < P.count) seen[g1.pt[i]] = 1;
            for (int i = 0; i < g.count; i++) {
                const int p = g.pt[i];
                if (p < 0 || p >= P.count) throw axg::Error(AXG_E_ARG, "Sponge || point index out of range.");
                if (seen[p]) throw axg::Error(AXG_E_ARG, "Sponge || point listed twice.");
                seen[p] = 1;
                if (g.off[i] < 0 || g.off[i] + P.nr[p] > (int64_t)g.gamma.size())
                    throw axg::Error(AXG_E_ARG, "Sponge::Sponge || Incompatible sizes.");
            }
        }
        for (int solid = 1; solid >= 0; solid--) {
            const std::vector<int> &pts = solid ? m.scan.solid_pts : m.scan.fluid_pts;
            const int np = solid ? m.sp.count : m.fp.count;
            std::vector<char> seen(np, 0);
            for (int p : pts) {
                if (p < 0 || p >= np) throw axg::Error(AXG_E_ARG, "WavefieldScanning || point index out of range.");
                if (seen[p]) throw axg::Error(AXG_E_ARG, "WavefieldScanning || point listed twice.");
                seen[p] = 1;
            }
        }
        for (int solid = 1; solid >= 0; solid--) {
            // PRT: one per element, sizes, 3-D factors on 3-D elements only
            const axg::HostPrt &pr = solid ? m.prt : m.prt_f;
            const int ne = solid ? m.se.count : m.fe.count;
            std::vector<char> seen(ne, 0);
            for (int i = 0; i < pr.count; i++) {
                const int e = pr.elem[i];
                if (e < 0 || e >= ne) throw axg::Error(AXG_E_ARG, "PRT || element index out of range.");
                if (seen[e]) throw axg::Error(AXG_E_ARG, "PRT || element listed twice.");
                seen[e] = 1;
                const std::vector<uint8_t> &is3d = solid ? m.se.is3d : m.fe.is3d;
                const bool e3d = is3d.size() && is3d[e];
                if (pr.x3d[i] && !e3d)
                    throw axg::Error(AXG_E_ARG, "PRT::checkCompatibility || 3-D PRT on a 1-D element.");
                const int64_t ns = pr.x3d[i] ? (solid ? m.se.nr[e] : m.fe.nr[e]) : 1;
                if (pr.off[i] < 0 || pr.off[i] + 5 * ns * 25 > (int64_t)pr.x.size())
                    throw axg::Error(AXG_E_ARG, "PRT::checkCompatibility || Incompatible sizes.");
            }
        }
        // one Sponge per point (GLLPoint::release averages the boundaries' gammas first)
        for (const auto &sg : {std::make_pair(&m.sg_s, m.sp.count), std::make_pair(&m.sg_f, m.fp.count)}) {
            std::vector<char> seen(sg.second, 0);
            for (int i = 0; i < sg.first->count; i++) {
                const int p = sg.first->pt[i];
                if (p < 0 || p >= sg.second) throw axg::Error(AXG_E_ARG, "Sponge || point index out of range.");
                if (seen[p]) throw axg::Error(AXG_E_ARG, "Sponge || point listed twice.");
                seen[p] = 1;
            }
        }
        h->eng->finalize(m);
        h->finalized = true;
    });
}

int axg_apply_sources(axg_solver *h, int32_t tstep) {
    return guarded(h, [&] { h->eng->apply_sources(tstep); });
}
int axg_compute_stiffness(axg_solver *h) {
    return guarded(h, [&] { h->eng->compute_stiffness(); });
}
int axg_compute_stiffness_part(axg_solver *h, int32_t part) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_compute_stiffness_part || axg_finalize not called.");
        h->eng->compute_stiffness_part(part);
    });
}
int axg_set_element_parts(axg_solver *h, const uint8_t *solid_part, const uint8_t *fluid_part) {
    return guarded(h, [&] {
        need_open(h);
        auto take = [](std::vector<uint8_t> &dst, const uint8_t *src, int count) {
            dst.clear();
            if (!src) return;
            for (int e = 0; e < count; e++)
                if (src[e] > 1) throw axg::Error(AXG_E_ARG, "axg_set_element_parts || a part is 0 or 1.");
            dst.assign(src, src + count);
        };
        take(h->model.se.part, solid_part, h->model.se.count);
        take(h->model.fe.part, fluid_part, h->model.fe.count);
    });
}
// no device allocation: the SLS memory of the evaluation lives in the library's fixed
// device array (noalloc.cu), looked up on this handle's device at the first call there
int axg_compute_stiffness_noalloc(axg_solver *h, const void *solid_x, void *solid_f, const void *fluid_x,
                                  void *fluid_f) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_compute_stiffness_noalloc || axg_finalize not called.");
        void *scratch = axg::noalloc_scratch(h->eng->device());
        h->eng->stiffness_noalloc(solid_x, solid_f, fluid_x, fluid_f, scratch, AXG_NOALLOC_SCRATCH_BYTES);
    });
}
int axg_gather_stiffness(axg_solver *h, int32_t solid, int64_t n, const int64_t *slots, void *buf) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_gather_stiffness || axg_finalize not called.");
        h->eng->gather_stiffness(solid, n, slots, buf);
    });
}
int axg_scatter_add_stiffness(axg_solver *h, int32_t solid, int64_t n, const int64_t *slots, const void *buf) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_scatter_add_stiffness || axg_finalize not called.");
        h->eng->scatter_add_stiffness(solid, n, slots, buf);
    });
}
int axg_apply_bc_before_assembly(axg_solver *h) {
    return guarded(h, [&] { h->eng->bc_before(); });
}
int axg_apply_bc_after_assembly(axg_solver *h) {
    return guarded(h, [&] { h->eng->point_stage(1); });
}
int axg_stiff_to_accel(axg_solver *h) {
    return guarded(h, [&] { h->eng->point_stage(2); });
}
int axg_newmark_update(axg_solver *h) {
    return guarded(h, [&] { h->eng->point_stage(4); });
}
int axg_record_stations(axg_solver *h, int32_t tstep) {
    return guarded(h, [&] { h->eng->record(tstep); });
}
int axg_run(axg_solver *h, int32_t nsteps, int32_t use_graph) {
    return guarded(h, [&] {
        if (nsteps < 0) throw axg::Error(AXG_E_ARG, "NewmarkTimeScheme::solve || nsteps < 0.");
        h->eng->run(nsteps, use_graph != 0);
    });
}
int axg_current_step(const axg_solver *h, int32_t *tstep) {
    if (!h || !tstep) return AXG_E_ARG;
    *tstep = h->eng->step();
    return AXG_OK;
}

int axg_get_field(axg_solver *h, int32_t solid, int32_t which, double *host_out) {
    return guarded(h, [&] {
        if (!host_out || which < 0 || which > 3) throw axg::Error(AXG_E_ARG, "axg_get_field || bad argument.");
        h->eng->get_field(solid, which, host_out);
    });
}
int axg_set_field(axg_solver *h, int32_t solid, int32_t which, const double *host_in) {
    return guarded(h, [&] {
        if (!host_in || which < 0 || which > 3) throw axg::Error(AXG_E_ARG, "axg_set_field || bad argument.");
        h->eng->set_field(solid, which, host_in);
    });
}
int axg_field_size(const axg_solver *h, int32_t solid, int64_t *n) {
    if (!h || !n) return AXG_E_ARG;
    if (!h->finalized) return AXG_E_STATE;
    *n = h->eng->field_size(solid);
    return AXG_OK;
}
int axg_forward_checkpointed(axg_solver *h, int32_t nsteps, int32_t checkpoint_interval) {
    return guarded(h, [&] { h->eng->forward_checkpointed(nsteps, checkpoint_interval); });
}
int axg_adjoint_run(axg_solver *h, const double *seis_adjoint, double *grad_moduli, double *grad_mass,
                    double *grad_displ0, double *grad_veloc0) {
    return guarded(h, [&] { h->eng->adjoint_run(seis_adjoint, grad_moduli, grad_mass, grad_displ0, grad_veloc0); });
}
int axg_set_adjoint_slices(axg_solver *h, int32_t on) {
    return guarded(h, [&] { h->eng->set_adjoint_slices(on != 0); });
}
int axg_get_adjoint_slices(axg_solver *h, double *grad_moduli_slices, double *grad_mass_slices) {
    return guarded(h, [&] { h->eng->get_adjoint_slices(grad_moduli_slices, grad_mass_slices); });
}
int axg_field_raw_bytes(const axg_solver *h, int32_t solid, int32_t which, int64_t *bytes) {
    if (!h || !bytes || which < 0 || which > 3) return AXG_E_ARG;
    if (!h->finalized) return AXG_E_STATE;
    *bytes = h->eng->field_raw_bytes(solid, which);
    return AXG_OK;
}
int axg_set_field_raw(axg_solver *h, int32_t solid, int32_t which, const void *host, int64_t bytes) {
    return guarded(h, [&] {
        if (!host || which < 0 || which > 3) throw axg::Error(AXG_E_ARG, "axg_set_field_raw || bad argument.");
        h->eng->set_field_raw(solid, which, host, bytes);
    });
}
int axg_get_field_raw(axg_solver *h, int32_t solid, int32_t which, void *host, int64_t bytes) {
    return guarded(h, [&] {
        if (!host || which < 0 || which > 3) throw axg::Error(AXG_E_ARG, "axg_get_field_raw || bad argument.");
        h->eng->get_field_raw(solid, which, host, bytes);
    });
}
int axg_get_seismograms(axg_solver *h, double *host_out, int32_t *nrecords) {
    return guarded(h, [&] {
        int n = h->eng->get_seismograms(host_out);
        if (nrecords) *nrecords = n;
    });
}
int axg_get_station_gradients(axg_solver *h, double *host_out, int32_t *nrecords) {
    return guarded(h, [&] {
        int n = h->eng->get_station_gradients(host_out);
        if (nrecords) *nrecords = n;
    });
}
int axg_set_element_record(axg_solver *h, int32_t n, const int32_t *elem, const int32_t *gll,
                           const int32_t *kind, int32_t interval, int32_t ring) {
    return guarded(h, [&] {
        if (!h->finalized) throw axg::Error(AXG_E_STATE, "axg_set_element_record || axg_finalize not called.");
        h->eng->set_element_record(n, elem, gll, kind, interval, ring);
    });
}
int axg_element_record_words(const axg_solver *h, int64_t *words) {
    if (!h || !words) return AXG_E_ARG;
    if (!h->finalized) return AXG_E_STATE;
    *words = h->eng->element_record_words();
    return AXG_OK;
}
int axg_get_element_records(axg_solver *h, int32_t rec_first, int32_t nrec, double *host_out) {
    return guarded(h, [&] { h->eng->get_element_records(rec_first, nrec, host_out); });
}
int axg_synchronize(axg_solver *h) {
    return guarded(h, [&] { h->eng->synchronize(); });
}
int axg_launch_count(const axg_solver *h, int64_t *n) {
    if (!h || !n) return AXG_E_ARG;
    *n = h->eng->launches();
    return AXG_OK;
}
int axg_set_timing(axg_solver *h, int32_t on) {
    return guarded(h, [&] { h->eng->set_timing(on != 0); });
}
int axg_stiffness_time_ms(axg_solver *h, double *ms, int64_t *launches) {
    return guarded(h, [&] {
        double t = 0;
        int64_t n = 0;
        h->eng->stiffness_time(&t, &n);
        if (ms) *ms = t;
        if (launches) *launches = n;
    });
}
int axg_stiffness_cost(const axg_solver *h, double *bytes, double *flops) {
    if (!h || !bytes || !flops) return AXG_E_ARG;
    if (!h->finalized) return AXG_E_STATE;
    h->eng->stiffness_cost(bytes, flops);
    return AXG_OK;
}
int axg_point_cost(const axg_solver *h, double *bytes) {
    if (!h || !bytes) return AXG_E_ARG;
    if (!h->finalized) return AXG_E_STATE;
    *bytes = h->eng->point_cost();
    return AXG_OK;
}
int axg_set_stream(axg_solver *h, void *stream) {
    return guarded(h, [&] { h->eng->set_stream(stream); });
}
int axg_set_team_size(axg_solver *h, int32_t nr_class, int32_t team) {
    return guarded(h, [&] {
        need_open(h);
        if (team != 32 && team != 64 && team != 128 && team != 256)
            throw axg::Error(AXG_E_ARG, "axg_set_team_size || team must be 32, 64, 128 or 256.");
        h->eng->set_team_override(nr_class, team);
    });
}

}  // extern "C"
