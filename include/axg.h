/*
 * axg.h -- C ABI of the B200 time-step engine for AxiSEM3D (nPol = 4).
 *
 * The engine replaces, for one MPI rank's sub-mesh, the per-time-step work that
 * AxiSEM3D's Domain performs on the CPU:
 *
 *   SolidElement::computeStiff / FluidElement::computeStiff
 *       (SOLVER/src/core/element/SolidElement.cpp:213-222,
 *        SOLVER/src/core/element/FluidElement.cpp:163-172)
 *       called in a loop by Domain::computeStiffness
 *       (SOLVER/src/core/domain/Domain.cpp:298-308)
 *   Domain::applyBC_BeforeAssemblingStiff / applyBC_AfterAssemblingStiff
 *       (Domain.cpp:313-326; SolidFluidCoupling, AxialBoundary, FluidSurfaceBoundary)
 *   Domain::computeStiffToAccel -> SolidPoint/FluidPoint::computeStiffToAccel
 *       (Domain.cpp:335-345, SOLVER/src/core/point/SolidPoint.cpp:28-36,
 *        FluidPoint.cpp:28-54, mass/Mass1D.hpp:25-32, mass/Mass3D.cpp:41-68)
 *   NewmarkTimeScheme::update<Point>
 *       (SOLVER/src/core/time/NewmarkTimeScheme.hpp:47-71)
 *   Domain::applySources -> SolidMoment::apply / SolidForce::apply
 *       (Domain.cpp:285-295, SOLVER/src/core/source/elem_src/solid/SolidMoment.cpp:29-33)
 *   StationSolid::record (displacement channel)
 *       (SOLVER/src/core/output/station-wise/station/StationSolid.cpp:58-91)
 *   the driver loop NewmarkTimeScheme::solve (NewmarkTimeScheme.cpp:41-108)
 *
 * Conventions shared with the reference:
 *   - point index inside an element: ipnt = ipol * 5 + jpol, ipol <-> xi (GLJ on
 *     axial elements, axis at ipol = 0), jpol <-> eta (spectrals.hpp:321-339);
 *   - a point of Fourier order nr stores nu = nr / 2 + 1 complex modes;
 *     an element's nr is the maximum over its 25 points (Element.cpp:28-43);
 *   - Voigt order 0=ss 1=pp 2=zz 3=pz 4=sz 5=sp, engineering shear strain;
 *   - 3-D (azimuthally varying) properties are sampled on slices
 *     phi_k = 2 pi k / nr, k = 0..nr-1.
 *
 * Host-side field layout (axg_get_field / axg_set_field): for each wavefield, for
 * each point in point order, nu_p x ndim complex doubles, row-major in (mode, dim),
 * i.e. the transpose of the reference's column-major eigen::CMatX3
 * (SolidPoint.hpp:126-131).
 *
 * Every function returns AXG_OK (0) or a negative AXG_E_* code; the message is
 * available from axg_last_error(h) in the reference's "Class::method || message"
 * format. No C++ exception crosses this boundary.
 *
 * A handle is not thread-safe: one handle per host thread / CUDA stream, as the
 * reference's element code is non-reentrant (static workspaces,
 * SolidElement.hpp:203-218).
 */
#ifndef AXG_H
#define AXG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AXG_NPED 5
#define AXG_NPEM 25

/* status codes */
#define AXG_OK            0
#define AXG_E_ARG        -1   /* invalid argument or inconsistent sizes   */
#define AXG_E_STATE      -2   /* call out of order (e.g. step before finalize) */
#define AXG_E_CUDA       -3   /* CUDA runtime error                         */
#define AXG_E_UNSTABLE   -4   /* non-finite displacement (Domain::checkStability) */
#define AXG_E_NOMEM      -5   /* device allocation failed                   */
#define AXG_E_UNSUPPORTED -6  /* feature combination not built              */

/* precision of the time loop */
#define AXG_FP64   0  /* everything in double (reference built with -Ddouble=true) */
#define AXG_FP32   1  /* everything in float (reference default build)            */
#define AXG_MIXED  2  /* float stiffness; double Newmark d/v with compensated
                         summation; double attenuation memory variables          */

/* rheology */
#define AXG_ISO    0  /* lambda, mu                                  (Isotropic.hpp)             */
#define AXG_TISO   1  /* A, C, F, L, N                               (TransverselyIsotropic.hpp) */
#define AXG_ANISO  2  /* C11 C12 C13 C14 C15 C16 C22 C23 C24 C25 C26
                         C33 C34 C35 C36 C44 C45 C46 C55 C56 C66   (Anisotropic.hpp)           */

/* attenuation (SLS memory variables) */
#define AXG_ATT_NONE 0
#define AXG_ATT_FULL 1  /* all 25 points          (AttenuationFull.hpp) */
#define AXG_ATT_CG4  2  /* points (1,1) (1,3) (3,1) (3,3)  (AttenuationCG4.hpp) */

/* fields */
#define AXG_FIELD_STIFF 0
#define AXG_FIELD_DISPL 1
#define AXG_FIELD_VELOC 2
#define AXG_FIELD_ACCEL 3

/* mapping of a quad (SOLVER/src/preloop/se_model/quad/mapping) */
#define AXG_MAP_LINEAR    0   /* MappingLinear.hpp    */
#define AXG_MAP_SPHERICAL 1   /* MappingSpherical.hpp */
#define AXG_MAP_SEMI_SPHERICAL 2   /* MappingSemiSpherical.hpp */

#define AXG_MAX_SLS 8

typedef struct axg_config {
    int32_t precision;          /* AXG_FP64 / AXG_FP32 / AXG_MIXED                        */
    int32_t device;             /* CUDA device ordinal                                     */
    double  dt;                 /* time step (NewmarkTimeScheme mDt)                       */
    double  t0;                 /* time of step 0 (TimeScheme mT0)                         */
    int32_t nsls;               /* number of standard linear solids (0 if no attenuation) */
    double  att_alpha[AXG_MAX_SLS]; /* Attenuation::setAlphaBetaGamma statics              */
    double  att_beta[AXG_MAX_SLS];
    double  att_gamma[AXG_MAX_SLS];
    int32_t stability_interval; /* steps between non-finite checks (0 = never)            */
    int32_t deterministic;      /* 1 = bitwise-reproducible assembly: elements coloured so
                                   that no two of a colour share a point, one launch per
                                   colour and bucket (sources in elements that share
                                   points still add in either order); 0 = one launch per
                                   bucket (atomic scatter-add, summation order may vary from
                                   run to run) */
    int32_t compensated;        /* MIXED only: 1 = compensated (Kahan) d/v summation      */
    int32_t plain;              /* 1 = the plain method: one element bucket per material
                                   kind with a fixed 256-thread team (no nr bucketing, no
                                   persistent grid), eager launches instead of CUDA graphs,
                                   no autotuning -- the baseline the batched path is
                                   measured against                                       */
    int32_t autotune;           /* 1 = time the candidate team sizes of every nr bucket at
                                   axg_finalize and keep the fastest                      */
    int32_t nwave;              /* independent wavefields (sources) advanced together on
                                   the same mesh; fields, state and seismograms gain a
                                   leading wavefield dimension (0 or 1 = one)             */
} axg_config;

/* solid GLL points (SolidPoint + Mass1D/Mass3D + AxialBoundary membership) */
typedef struct axg_solid_points {
    int32_t        count;
    const int32_t *nr;          /* [count] Fourier order of each point                      */
    const int32_t *mass_nr;     /* [count] 1 (Mass1D) or nr (Mass3D); NULL = all 1        */
    const int64_t *mass_offset; /* [count] offset into mass; NULL = point index            */
    const double  *mass;        /* integrated mass (not inverted) per point / per slice    */
    const uint8_t *axial;       /* [count] 1 = point on the axis (AxialBoundary); may be NULL */
} axg_solid_points;

/* fluid GLL points (FluidPoint) */
typedef struct axg_fluid_points {
    int32_t        count;
    const int32_t *nr;
    const int32_t *mass_nr;
    const int64_t *mass_offset;
    const double  *mass;        /* integrated 1/kappa (Material::getMass, fluid branch) */
    const uint8_t *axial;       /* AxialBoundary (fluid part) */
    const uint8_t *surface;     /* FluidSurfaceBoundary: stiffness zeroed */
} axg_fluid_points;

/* solid elements: the operands SolidElement holds after Quad::release */
typedef struct axg_solid_elements {
    int32_t        count;
    const int32_t *nr;          /* [count] element nr (max over its points)             */
    const int32_t *points;      /* [count*25] solid point indices                       */
    const uint8_t *axial;       /* [count] GradientQuadrature mAxial                    */
    const double  *geometry;    /* [count*6*25] dsdxii, dsdeta, dzdxii, dzdeta, 1/s,
                                   integral factor (Quad::createGradient, Quad.hpp:155-184) */
    const uint8_t *rtz;         /* [count] rheology in RTZ (spherical meshes); NULL = none */
    const double  *theta;       /* [count*25] polar angle for CoordTransformSpherical    */
    const int32_t *rheology;    /* [count] AXG_ISO / AXG_TISO / AXG_ANISO              */
    const uint8_t *is3d;        /* [count] 1 = properties per slice (nr x 25)           */
    const int64_t *mat_offset;  /* [count] offset (doubles) into moduli                 */
    const double  *moduli;      /* per element [nmod][nslice][25], nslice = nr or 1     */
    const int32_t *attenuation; /* [count] AXG_ATT_*; NULL = none                        */
    const int64_t *att_offset;  /* [count] offset (doubles) into att_moduli              */
    const double  *att_moduli;  /* per element [2][nslice][25 or 4]: dlambda, dmu        */
} axg_solid_elements;

/* fluid elements: FluidElement + Acoustic (K = 1/rho) */
typedef struct axg_fluid_elements {
    int32_t        count;
    const int32_t *nr;
    const int32_t *points;      /* [count*25] fluid point indices */
    const uint8_t *axial;
    const double  *geometry;    /* [count*6*25] as for solids */
    const uint8_t *is3d;
    const int64_t *mat_offset;
    const double  *moduli;      /* per element [nslice][25]: K */
} axg_fluid_elements;

/* solid-fluid coupling pairs (SolidFluidCoupling1D.hpp:26-37) */
typedef struct axg_solid_fluid {
    int32_t        count;
    const int32_t *solid_point;
    const int32_t *fluid_point;
    const double  *ns_unassembled;
    const double  *nz_unassembled;
    const double  *ns_assembled;
    const double  *nz_assembled;
    const double  *mass_fluid;
} axg_solid_fluid;

/* Gaussian-family source-time function (GaussianSTF.hpp:35-58) */
typedef struct axg_stf {
    double  half_duration;
    double  decay_factor;
    double  time_shift;
    int32_t derivative_order;   /* -1 erf, 0 Gaussian, 1, 2 (Ricker) */
} axg_stf;

/* moment-tensor sources (SolidMoment + Mechanism pattern) */
typedef struct axg_moment_sources {
    int32_t        count;
    const int32_t *element;       /* solid element index                        */
    const int32_t *nu;            /* pattern modes (rows of CMatXN6)             */
    const int64_t *pattern_offset;/* offset in complex numbers into pattern      */
    const double  *pattern;       /* per source [nu][6][25] complex (re, im)     */
    const axg_stf *stf;           /* [count] */
    const int32_t *wavefield;     /* [count] wavefield each source drives; NULL = 0 */
} axg_moment_sources;

/* point-force sources (SolidForce + Mechanism pattern) */
typedef struct axg_force_sources {
    int32_t        count;
    const int32_t *element;
    const int32_t *nu;
    const int64_t *pattern_offset;
    const double  *pattern;       /* per source [nu][3][25] complex */
    const axg_stf *stf;
    const int32_t *wavefield;     /* [count]; NULL = 0 */
} axg_force_sources;

/* fluid-pressure sources (FluidPressure, core/source/elem_src/fluid/FluidPressure.cpp, with
   the pattern of Mechanism::release, preloop/source/Mechanism.cpp:59-86): each step the
   fluid points of the element get pattern * STF(t) added to their acceleration after the
   mass term (FluidPoint::computeStiffToAccel, FluidPoint.cpp:42-48), modes below the
   point's nu */
typedef struct axg_pressure_sources {
    int32_t        count;
    const int32_t *element;       /* fluid element index */
    const int32_t *nu;
    const int64_t *pattern_offset;
    const double  *pattern;       /* per source [nu][25] complex */
    const axg_stf *stf;
    const int32_t *wavefield;     /* [count]; NULL = 0 */
} axg_pressure_sources;

/* stations: in-plane Lagrange weights and azimuth (Station.hpp:53-72) */
typedef struct axg_stations {
    int32_t        count;
    const int32_t *element;       /* solid element index  */
    const double  *weights;       /* [count*25]           */
    const double  *phi;           /* [count]              */
} axg_stations;

/* Clayton-Engquist absorbing points with 1-D coefficients (ClaytonSolid1D.hpp,
   ClaytonFluid1D.hpp), applied in Domain::applyBC_BeforeAssemblingStiff */
typedef struct axg_clayton {
    int32_t        count;
    const int32_t *point;         /* solid or fluid point index                       */
    const double  *rho_vp;
    const double  *rho_vs;        /* solid only                                       */
    const double  *area;          /* length of the boundary normal (integration weight) */
    const double  *theta;         /* polar angle of the normal (solid only)            */
} axg_clayton;

/* 3-D Clayton-Engquist conditions (ClaytonSolid3D / ClaytonFluid3D, built in GLLPoint.cpp:148-190
   when the point's properties or normal vary with phi): per condition nr values (nr of its point)
   from offset[i] in every per-slice array */
typedef struct axg_clayton3d {
    int32_t        count;
    const int32_t *point;
    const int64_t *offset;        /* first per-slice value of condition i                 */
    int64_t        nvalues;       /* length of rho_vp / rho_vs / area (normal: 3x)         */
    const double  *rho_vp;
    const double  *rho_vs;        /* solid only                                           */
    const double  *area;          /* length of the boundary normal per slice              */
    const double  *normal;        /* solid only: unit normal (s, phi, z) per slice, [nvalues][3] */
} axg_clayton3d;

/* wavefield scanning (WavefieldScanning.cpp:40-90 parameters; Scanning1D, Point.hpp:106-198):
   every `interval` steps the displacement of each scanned point is checked for energy peaks
   and the number of Fourier modes each peak needs; axg_scanning_nr reports the resulting nr */
typedef struct axg_scanning {
    double         tol_fourier_h1;  /* threshold_Fourier_convergence                      */
    double         rel_tol_h1;      /* relative_amplitude_skipped                          */
    double         abs_tol_h1;      /* absolute_amplitude_skipped                          */
    int32_t        max_num_peaks;   /* peaks kept per component (at most AXG_SCAN_MAX_PEAKS) */
    int32_t        interval;        /* time steps between two scans                        */
    int32_t        n_solid;         /* scanned solid points; -1 = all                      */
    const int32_t *solid_points;
    int32_t        n_fluid;         /* scanned fluid points; -1 = all                      */
    const int32_t *fluid_points;
} axg_scanning;
#define AXG_SCAN_MAX_PEAKS 32

typedef struct axg_solver axg_solver;

/* ---- lifetime ---- */
int  axg_create(const axg_config *cfg, axg_solver **out);
int  axg_destroy(axg_solver *h);
const char *axg_last_error(const axg_solver *h);
const char *axg_version(void);

/* ---- model upload (host copies, nothing borrowed after return) ---- */
int  axg_set_solid_points(axg_solver *h, const axg_solid_points *p);
int  axg_set_fluid_points(axg_solver *h, const axg_fluid_points *p);
int  axg_set_solid_elements(axg_solver *h, const axg_solid_elements *e);
int  axg_set_fluid_elements(axg_solver *h, const axg_fluid_elements *e);
int  axg_set_solid_fluid(axg_solver *h, const axg_solid_fluid *c);
int  axg_set_moment_sources(axg_solver *h, const axg_moment_sources *s);
int  axg_set_force_sources(axg_solver *h, const axg_force_sources *s);
int  axg_set_pressure_sources(axg_solver *h, const axg_pressure_sources *s);
/* StreamSTF / NetCDF_STF (core/source/elem_src/stf/StreamSTF.cpp:63-93, NetCDF_STF.cpp:
   92-140): source `index` of `kind` (0 moment, 1 force, 2 pressure) takes its STF by linear
   interpolation in n (times, values), times ascending; outside them an error (padding 0) or
   left / right (padding 1, FIRST_LAST passes the first and last values); pad_first 1 tests
   the padding before the interpolation as NetCDF_STF does. Call after the sources. */
int  axg_set_stf_table(axg_solver *h, int32_t kind, int32_t index, int32_t n, const double *times,
                       const double *values, int32_t padding, double left, double right, int32_t pad_first);
int  axg_set_stations(axg_solver *h, const axg_stations *s, int32_t record_interval);
/* also record the displacement gradient at the stations (StationSolid::record with the
   G / E / R channels, StationSolid.cpp:58-91; SolidElement::getNablaField, :410-446): the
   nine components d_j u_i of GradientQuadrature::computeGrad9 (index 3 i + j, i and j in
   s, phi, z order; GradientQuadrature.hpp:177-202), interpolated at each station like the
   displacement; strain and curl are linear in it. For elements without particle
   relabelling. Set before axg_finalize. */
int  axg_set_station_gradient(axg_solver *h, int32_t enable);
/* Clayton-Engquist conditions (GLLPoint.cpp:148-190 builds one ClaytonSolid1D /
   ClaytonFluid1D per point and boundary key); a point on two boundaries is listed once per
   boundary, and its conditions are applied in the order listed */
int  axg_set_clayton(axg_solver *h, int32_t solid, const axg_clayton *c);
/* Kosloff sponge (Sponge.hpp, 1-D gamma per point, each point at most once), applied to the acceleration in
   Domain::applyBC_AfterComputingAccel: accel -= 2 gamma veloc + gamma^2 displ */
int  axg_set_sponge(axg_solver *h, int32_t solid, int32_t count, const int32_t *point,
                    const double *gamma);
/* 3-D Clayton conditions: applied after the 1-D ones of axg_set_clayton, in the order
   listed per point (stiff -= R2C(C(C2R(veloc))) per condition) */
int  axg_set_clayton3d(axg_solver *h, int32_t solid, const axg_clayton3d *c);
/* 3-D Kosloff sponge (Sponge.hpp, nr gammas per point, the 3-D constructor): on the
   acceleration in slices, accel -= 2 gamma veloc + gamma^2 displ; gamma[offset[i] ..
   offset[i] + nr - 1] for point[i]; a point carries a 1-D or a 3-D sponge, not both */
int  axg_set_sponge3d(axg_solver *h, int32_t solid, int32_t count, const int32_t *point,
                      const int64_t *offset, int64_t nvalues, const double *gamma);
/* enables wavefield scanning (Domain::doScanning, Domain.cpp:466-490) during axg_run and
   axg_record_stations; before axg_finalize; one wavefield per handle. A max_num_peaks above
   AXG_SCAN_MAX_PEAKS keeps the AXG_SCAN_MAX_PEAKS largest peaks (the reference keeps up to
   max_num_peaks) */
int  axg_set_scanning(axg_solver *h, const axg_scanning *s);
/* Point::reportScanningNr per point (solid: the largest over the three components):
   min(2 nu + 1, nr) of the peaks found, 1 where no peak passed, -1 for unscanned points;
   solid_nr [solid points], fluid_nr [fluid points] (either may be NULL) */
int  axg_scanning_nr(axg_solver *h, int32_t *solid_nr, int32_t *fluid_nr);
/* particle relabelling transformation on solid elements under topography (PRT, PRT/PRT.hpp;
   SolidElement::displToStiff's PRT branch, SolidElement.cpp:113-161): element[i] takes the
   J^-1 components X0..X3 and |J| (PRT constructor arguments) from x[offset[i]...] as
   [5][nslice][25] doubles, nslice = 1 (is3d_prt[i] = 0) or the element's nr (a 3-D PRT, which
   needs a 3-D element, axg_solid_elements.is3d); nvalues = length of x. On a spherical element
   (rtz) the 9-component gradient is taken to the RTZ frame first whatever the rheology. */
int  axg_set_prt(axg_solver *h, int32_t count, const int32_t *element, const int64_t *offset,
                 const uint8_t *is3d_prt, int64_t nvalues, const double *x);
/* the same for fluid elements (FluidElement::displToStiff's PRT branch, FluidElement.cpp:101-148);
   theta [count][25] (the polar angle of each element point, for the RTZ frame of spherical
   meshes) or NULL on cartesian meshes */
int  axg_set_prt_fluid(axg_solver *h, int32_t count, const int32_t *element, const int64_t *offset,
                       const uint8_t *is3d_prt, int64_t nvalues, const double *x, const double *theta);
/* MassOceanLoad1D (point/mass/MassOceanLoad1D.hpp, built in GLLPoint.cpp:66-73) on solid
   surface points under an ocean:
   in computeStiffToAccel the point's own mass acts along the surface and mass + mass_ocean
   across it, the surface normal at polar angle theta; each point at most once, points with
   1-D masses only (a Mass3D point takes axg_set_ocean_load3d) */
/* SolidFluidCoupling3D (core/boundary/solid_fluid/SolidFluidCoupling3D.cpp:40-94; built in
   GLLPoint.cpp:120-145 where the normal or the fluid mass varies with phi): per pair and
   slice of the points' nr (equal on both points), fluid stiff += R2C(n_u . C2R(solid
   displ)), then solid stiff -= R2C(C2R(fluid stiff) n_a / m_fluid); normal_u, normal_a
   [n][3] (s, phi, z) and mass_fluid [n] from offset[i]. A pair given here is not also in
   axg_set_solid_fluid. */
int  axg_set_solid_fluid3d(axg_solver *h, int32_t count, const int32_t *solid_point, const int32_t *fluid_point,
                           const int64_t *offset, int64_t nvalues, const double *normal_u,
                           const double *normal_a, const double *mass_fluid);
int  axg_set_ocean_load(axg_solver *h, int32_t count, const int32_t *point, const double *mass_ocean,
                        const double *theta);
/* MassOceanLoad3D (point/mass/MassOceanLoad3D.cpp, built in GLLPoint.cpp:74-87) where the
   ocean mass or the surface normal varies with phi: per slice, accel = F / m - (F . k) k with
   k = sqrt(m0 / (m (m + m0))) n; m = the point's own masses (1-D or Mass3D), m0 and the unit
   normal (s, phi, z) given per slice: nr values of mass_ocean (3 nr of normal) from offset[i] */
int  axg_set_ocean_load3d(axg_solver *h, int32_t count, const int32_t *point, const int64_t *offset,
                          int64_t nvalues, const double *mass_ocean, const double *normal);
/* builds buckets, uploads to HBM; must precede any time-loop call */
int  axg_finalize(axg_solver *h);

/* ---- the per-step hooks, one Domain method each ---- */
/* Domain::applySources for step tstep (time t0 + tstep*dt accumulated as in solve()) */
int  axg_apply_sources(axg_solver *h, int32_t tstep);
/* Domain::computeStiffness: point stiff -= K u for every element */
int  axg_compute_stiffness(axg_solver *h);
/* Domain::applyBC_BeforeAssemblingStiff (solid-fluid coupling) */
int  axg_apply_bc_before_assembly(axg_solver *h);
/* Domain::applyBC_AfterAssemblingStiff (axial, fluid surface) */
int  axg_apply_bc_after_assembly(axg_solver *h);
/* Domain::computeStiffToAccel (Nyquist, 1/M) */
int  axg_stiff_to_accel(axg_solver *h);
/* NewmarkTimeScheme::update on all points */
int  axg_newmark_update(axg_solver *h);
/* station recording of the displacement at step tstep */
int  axg_record_stations(axg_solver *h, int32_t tstep);
/* nsteps full Newmark steps starting at the handle's step counter
   (NewmarkTimeScheme::solve loop body); use_graph = 1 replays one CUDA graph per step */
int  axg_run(axg_solver *h, int32_t nsteps, int32_t use_graph);
/* step counter of the next step */
int  axg_current_step(const axg_solver *h, int32_t *tstep);

/* ---- differentiation (FP64 handles; phi-constant isotropic, TI or 21-Cij solid
        elements, RTZ frames included, elastic or with FULL / CG4 attenuation, or isotropic
        elastic 3-D elements with per-slice moduli (where an element or a point of it has an
        even nr, both have the same nr); 1-D masses, no fluid; no counterpart in the
        reference, which has no adjoint) ---- */
/* nsteps forward steps from the current state, storing the state every
   checkpoint_interval steps on the device for axg_adjoint_run. A checkpoint holds the point
   displacement, velocity and acceleration and, with attenuation, the SLS memory variables
   ((nsls + 1) x 6 x npa x nu complex values per attenuating element, npa = 25 FULL / 4 CG4),
   so attenuating models may want a longer interval; axg_adjoint_run also takes two segment
   buffers of checkpoint_interval fields each. */
int  axg_forward_checkpointed(axg_solver *h, int32_t nsteps, int32_t checkpoint_interval);
/* time-reversed discrete adjoint of the last axg_forward_checkpointed run, each
   segment recomputed from its checkpoint. seis_adjoint = dJ/d(seismograms),
   [nrecords][nstations][3]. Outputs (host, each may be NULL):
   grad_moduli per element [nmod_e][25] in the order of its moduli (lambda, mu; A, C, F, L,
   N; the 21 Cij), then, for an attenuating element, two rows dJ/d(dlambda, dmu) (CG4: at its
   four points q = 6, 8, 16, 18, zero elsewhere), elements in order, so
   [n_solid_elements][2][25] for an elastic isotropic model;
   grad_mass [n_solid_points]
   dJ/d(point mass), grad_displ0 / grad_veloc0 (sum(nu)*3 complex) dJ/d(initial
   displacement / velocity). The fields end in the state after the forward run. */
int  axg_adjoint_run(axg_solver *h, const double *seis_adjoint, double *grad_moduli,
                     double *grad_mass, double *grad_displ0, double *grad_veloc0);
/* per-slice sensitivities (no counterpart in the reference): with on = 1 the next
   axg_adjoint_run also accumulates the gradient of the misfit with respect to the moduli and
   masses of the 3-D parameterisation, the values at the slices phi_k = 2 pi k / nr that a 3-D
   element or a Mass3D point holds (PhysicalProperty.hpp:99-120): dJ/dlambda and dJ/dmu at
   every (slice, point) of every element, dJ/dM at every slice of every solid point. The
   linearisation point is the handle's model, 1-D or with 3-D isotropic moduli (its masses
   1-D); the sum over slices is the gradient by a phi-constant change (grad_moduli). Elastic isotropic models
   only (axg_adjoint_run returns AXG_E_UNSUPPORTED otherwise). */
int  axg_set_adjoint_slices(axg_solver *h, int32_t on);
/* after such a run: grad_moduli_slices per element [2][nr_e][25] (lambda, mu), elements in
   order; grad_mass_slices per solid point [nr_p]; either may be NULL */
int  axg_get_adjoint_slices(axg_solver *h, double *grad_moduli_slices, double *grad_mass_slices);

/* ---- fields ---- */
/* solid = 1 for solid points, 0 for fluid; host buffer of sum(nu_p)*ndim complex doubles */
int  axg_get_field(axg_solver *h, int32_t solid, int32_t which, double *host_out);
int  axg_set_field(axg_solver *h, int32_t solid, int32_t which, const double *host_in);
/* number of complex values of a field (sum(nu_p) * ndim) */
int  axg_field_size(const axg_solver *h, int32_t solid, int64_t *n);
/* native-precision copies between a (pinned) host buffer and a device field,
   asynchronous on the handle's stream: complex float for FP32 fields, complex
   double for FP64 ones (MIXED: displacement and velocity are double, stiffness
   and acceleration float). bytes must equal axg_field_raw_bytes(). Setting the
   displacement also refreshes the element copy and clears the compensation. */
int  axg_field_raw_bytes(const axg_solver *h, int32_t solid, int32_t which, int64_t *bytes);
int  axg_set_field_raw(axg_solver *h, int32_t solid, int32_t which, const void *host, int64_t bytes);
int  axg_get_field_raw(axg_solver *h, int32_t solid, int32_t which, void *host, int64_t bytes);
/* seismograms recorded so far: [nrecords][nwave][nstations][3] doubles, SPZ components */
int  axg_get_seismograms(axg_solver *h, double *host_out, int32_t *nrecords);
/* station gradients recorded so far: [nrecords][nwave][nstations][9] doubles (after
   axg_set_station_gradient(h, 1)) */
int  axg_get_station_gradients(axg_solver *h, double *host_out, int32_t *nrecords);
/* Element-wise output (ElementOpGroup::record, core/output/element-wise/element/ElementOpGroup.hpp:
   197-215, and ElementOpSolid::record, ElementOpSolid.cpp:48-80, before the RTZ transform and the
   channels, which the host forms): after axg_finalize, entry i names GLL point gll[i] (ipol * 5 +
   jpol) of solid element elem[i] and a kind, 0 = the displacement (3 components), 1 = its gradient
   computeGrad9 (9 components, g[c * 3 + d] = d_d u_c, d = s, phi, z). At every step that is a
   multiple of `interval` the Fourier coefficients of orders 0 .. nr/2 of the element are kept in
   a device ring of `ring` records (record r = step / interval in slot r % ring), so a caller
   that reads them back at least every ring records (buffer_size) never loses one. One record
   per wavefield holds axg_element_record_words complex words: the entries in order, each as
   [order][component]. A new call replaces the previous entries. */
int  axg_set_element_record(axg_solver *h, int32_t n, const int32_t *elem, const int32_t *gll,
                            const int32_t *kind, int32_t interval, int32_t ring);
int  axg_element_record_words(const axg_solver *h, int64_t *words);
/* records rec_first .. rec_first + nrec - 1, which must all be in the ring, into host_out as
   [nrec][nwave][words][re, im] doubles */
int  axg_get_element_records(axg_solver *h, int32_t rec_first, int32_t nrec, double *host_out);
int  axg_synchronize(axg_solver *h);

/* ---- diagnostics ---- */
/* number of kernels launched by this handle since creation */
int  axg_launch_count(const axg_solver *h, int64_t *n);
/* cumulative device time (ms) of the solid stiffness kernels, when timing is on */
int  axg_set_timing(axg_solver *h, int32_t on);
int  axg_stiffness_time_ms(axg_solver *h, double *ms, int64_t *launches);
/* algorithmic HBM bytes and FP32/FP64 flops of one stiffness evaluation
   (solid + fluid elements), from the mesh: per element the geometry (6 x 25 reals), point ids,
   moduli (nmod x nslice x 25), attenuation moduli (2 x nslice x npa) and the SLS state read
   and written once; flops of the gradient, quadrature, stress and the two direct DFTs */
int  axg_stiffness_cost(const axg_solver *h, double *bytes, double *flops);
/* algorithmic bytes of one point update (stiff->accel + Newmark) */
int  axg_point_cost(const axg_solver *h, double *bytes);
/* run on the caller's CUDA stream (a cudaStream_t passed as void*; NULL = the
   handle's own stream). Invalidates a captured step graph. */
int  axg_set_stream(axg_solver *h, void *stream);
/* threads per element team for the nr class (0: nr<=3, 1: <=9, 2: <=25, 3: <=64,
   4: larger); 32, 64, 128 or 256; before axg_finalize (the autotuner's knob) */
int  axg_set_team_size(axg_solver *h, int32_t nr_class, int32_t team);

/* ---- boundary-stiffness exchange of a partitioned mesh ----
   The reference sums the stiffness of the points that MPI ranks share once per step, between
   the boundary conditions before assembly and those after it: Messaging::commGatherSendRecv /
   commWaitScatter (SOLVER/src/core/domain/Messaging.hpp:26-47), MessageRank::gatherFromPoints /
   scatterToPoints (MessageRank.cpp:40-63), SolidPoint::feedComm / extractComm
   (SolidPoint.hpp:55-67), called from NewmarkTimeScheme::solve (NewmarkTimeScheme.cpp:57-83).
   Here a handle holds one rank's sub-mesh; the host moves the buffers between ranks (NCCL or
   another transport). slots: DEVICE array of n indices, in complex values, into the handle's
   solid (solid = 1) or fluid (solid = 0) stiffness field (the layout of axg_field_size:
   [sum nu][3] or [sum nu]); buf: DEVICE buffer of n complex values in the stiffness precision
   (complex float for AXG_FP32 / AXG_MIXED, complex double for AXG_FP64). Both run on the
   handle's stream (axg_set_stream) and need one wavefield per handle. */
/* buf[i] = stiff[slots[i]] */
int  axg_gather_stiffness(axg_solver *h, int32_t solid, int64_t n, const int64_t *slots, void *buf);
/* stiff[slots[i]] += buf[i]; the slots of one call must be distinct */
int  axg_scatter_add_stiffness(axg_solver *h, int32_t solid, int64_t n, const int64_t *slots, const void *buf);
/* Element parts, so that a rank can hide the exchange behind element work: the elements that
   touch a shared point (part 0) first, the gather and the transfer, then the others (part 1)
   while the transfer runs. The reference overlaps its exchange with output and scanning only
   (NewmarkTimeScheme.cpp:57-83); this split has no counterpart there. part: 0 or 1 per solid /
   fluid element (NULL = all 0), after the element setters and before axg_finalize; no bucket
   mixes parts. */
int  axg_set_element_parts(axg_solver *h, const uint8_t *solid_part, const uint8_t *fluid_part);
/* Domain::computeStiffness (Domain.cpp:298-308) for the elements of one part (0 or 1): the two
   parts together add what axg_compute_stiffness adds */
int  axg_compute_stiffness_part(axg_solver *h, int32_t part);

/* ---- stiffness of a caller's field with no device allocation ----
   No counterpart in the reference. Adds -K x to f for every element of a finalized handle,
   as axg_compute_stiffness does for the handle's own displacement on a freshly created
   handle (SLS memory at rest). x and f are DEVICE pointers in the handle's field layout
   ([sum nu][3] complex for solid points, [sum nu] complex for fluid points, the sizes of
   axg_field_size) and in its stiffness precision: complex float for AXG_FP32 and AXG_MIXED,
   complex double for AXG_FP64; the fluid pair may be NULL when there are no fluid elements.
   The handle's own fields and attenuation state are not touched.
   For callers that must not allocate device memory: a process whose device memory is
   owned by another runtime (JAX/XLA reserves most of the GPU up front, serving frameworks
   run their own pools), where cudaMalloc fails or escapes the owner's accounting, and code
   called back from such a runtime. Working memory (the SLS memory variables of this one
   evaluation) lives in a fixed device array inside the library, AXG_NOALLOC_SCRATCH_BYTES
   large, which every GPU that loads the library keeps until the process exits; a model whose
   SLS state is larger gets AXG_E_ARG. The array is cleared at the start of each call. All
   calls on a device share it, so calls whose GPU work overlaps (other streams, other handles)
   race: order them on one stream or synchronize between them. The work is queued on the
   handle's stream (axg_set_stream). The first call on a device looks the array up
   (cudaGetSymbolAddress); make that first call before any stream capture. The address is kept
   for the life of the process: a device reset (cudaDeviceReset) after the first call on that
   device is not supported. */
#define AXG_NOALLOC_SCRATCH_BYTES (16u << 20)
int  axg_compute_stiffness_noalloc(axg_solver *h, const void *solid_x, void *solid_f,
                                   const void *fluid_x, void *fluid_f);

/* ---- operand construction (host, double), the preloop numbers ---- */
/* GLL/GLJ positions, weights and G matrices for nPol = 4, derived from their
   definitions and rounded to 12 decimals (spectrals.hpp:73-102) */
int  axg_spectral_tables(double *xgll, double *xglj, double *wgll, double *wglj,
                         double *ggll, double *gglj);
/* Quad::createGradient + Quad::computeIntegralFactor (Quad.hpp:155-184,
   Quad.cpp:403-435) for a quad with the given 4 nodes (s0 z0 s1 z1 s2 z2 s3 z3,
   counter-clockwise from (xi,eta)=(-1,-1)); out_geometry[6*25], out_sz[2*25] */
int  axg_quad_geometry(int32_t mapping, const double *nodal_sz, int32_t axial,
                       double *out_geometry, double *out_sz);
/* one point of a quad's mapping and its Jacobian d(s,z)/d(xi,eta): out[6] = s, z, J00, J01,
 * J10, J11 (Mapping::mapping, Mapping::jacobian; mapping/Mapping.hpp, MappingLinear.hpp,
 * MappingSpherical.hpp, MappingSemiSpherical.hpp) */
int  axg_quad_map(int32_t mapping, const double *nodal_sz, double xi, double eta, double *out);
/* axg_quad_geometry over n quads: nodal_sz [n*8], axial [n], out [n*150], [n*50] */
int  axg_quad_geometry_batch(int32_t n, int32_t mapping, const double *nodal_sz,
                             const uint8_t *axial, double *out_geometry, double *out_sz);
/* Quad::computeDt (Quad.cpp:271-349) for one quad: min neighbour distance / vmax */
int  axg_quad_dt(const double *sz, double vmax, double *dt);
/* AttBuilder::setAlphaBetaGamma (AttBuilder.cpp:183-198) */
int  axg_att_alpha_beta_gamma(int32_t nsls, const double *w, const double *y, double dt,
                              double *alpha, double *beta, double *gamma);
/* AttBuilder::createAttenuation (AttBuilder.cpp:102-178), FULL or CG4, for n samples:
   kp, mu are modified in place (relaxed -> unrelaxed moduli); dkp/dmu outputs are
   per sample (CG4 weighting is applied by the caller through weights_cg4 when cg4=1,
   on arrays of 25 points per sample) */
int  axg_att_moduli(int32_t nsls, const double *w, const double *y,
                    double fmin, double fmax, double fref,
                    int32_t n, const double *qkappa, const double *qmu,
                    double *kp, double *mu, double *dkp, double *dmu);

#ifdef __cplusplus
}
#endif
#endif /* AXG_H */
