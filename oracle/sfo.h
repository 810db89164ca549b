/*
 * sfo.h -- CPU oracle for the SoftFlow per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64, single-threaded
 * restatement of the reference engine's step (ramc77/SoftFlow,
 * src/engine/simulation.cpp:470-801) used as the checker for the CUDA
 * implementation in softflow_b200/.  Nothing in the product links it.
 *
 * Every function in sfo.c cites the reference file:line it restates.  The
 * restatement keeps the reference's expression order so that, compiled
 * without FMA contraction and without -ffast-math, it reproduces the
 * reference's own FP64 results bit for bit (pinned by
 * tests/test_oracle_vs_reference.py against the reference sources compiled
 * by oracle/Makefile).
 *
 * Scope: periodic-x channel (rows 0 and ny-1 SOLID, or periodic-y), a
 * closed box, or a Zou-He inlet / outlet channel, with optional moving top /
 * bottom walls; BGK /
 * MRT / regularized collision with Guo forcing, body force + force cap,
 * Peskin 4-point IBM spread / interpolate / multi-direct forcing, circular
 * capsules with Hookean / Neo-Hookean / Skalak / WLC stretching,
 * Laplacian or Helfrich bending, area / perimeter penalties, damping,
 * Kelvin-Voigt membrane viscosity, soft contact with the cell list, and the
 * single-species advection-diffusion step.
 */
#ifndef SFO_H
#define SFO_H

#ifdef __cplusplus
extern "C" {
#endif

/* Collision operator ids (reference src/core/parameters.h CollisionModel). */
enum { SF_BGK = 0, SF_MRT = 1, SF_REGULARIZED = 2 };
/* Membrane model ids (reference src/core/parameters.h MembraneModel). */
enum { SF_HOOKEAN = 0, SF_NEO_HOOKEAN = 1, SF_SKALAK = 2, SF_WLC = 3 };

/* Channel parameters: the subset of SimulationParams on the hot path
 * (reference src/core/parameters.h:41-342). */
typedef struct sf_params {
    int nx, ny;
    int collision;              /* SF_BGK / SF_MRT / SF_REGULARIZED        */
    double tau, rho0;
    double mrt_se, mrt_s_eps, mrt_sq;
    double body_fx, body_fy;
    int periodic_y;             /* 0: SOLID rows 0 and ny-1                 */
    double max_lattice_force;   /* force cap (|F| <= cap)                   */
    int ibm_iterations;         /* 1 = plain spread; K > 1 = MDF            */
    double dt;
    /* soft contact (RepulsionParams) */
    double rep_epsilon, rep_sigma, rep_r_cut;
    int rep_power;
    double rep_damping_normal, rep_friction;
    /* advection-diffusion (ScalarParams, one species) */
    int scalar_enabled;
    double scalar_D;
    int scalar_periodic_y;
    double scalar_inlet;
    /* fluid boundaries (FluidParams, parameters.h:44-46, 87-88):
     * boundary_type as BoundaryType (types.h:58-62): 0 INLET_OUTLET
     * (Zou-He velocity inlet at x = 0, pressure outlet at x = nx-1),
     * 1 PERIODIC, 2 CLOSED; moving top / bottom walls */
    int boundary_type;
    double inlet_velocity, outlet_density;
    double top_wall_velocity, bottom_wall_velocity;
    /* Bouzidi interpolated bounce-back at obstacle links
     * (FluidParams::use_interpolated_bb, parameters.h:89) */
    int use_interpolated_bb;
} sf_params;

/* Membrane parameters (reference MembraneParams, circle shape only). */
typedef struct sf_membrane {
    int model;
    double k_stretch, G_s, C_skalak;
    double wlc_L_max_ratio, wlc_kBT_p, wlc_k_pow;
    double k_bend;
    int use_helfrich;
    double kappa_0;
    double k_area, k_perimeter, gamma_visc, eta_membrane;
} sf_membrane;

typedef struct sfo_sim sfo_sim;

void sf_params_default(sf_params* p);
void sf_membrane_default(sf_membrane* m);

sfo_sim* sfo_create(const sf_params* p);
void sfo_destroy(sfo_sim* s);

/* Pillars of the channel geometry (ChannelBuilder::addCirclePillar /
 * addRectPillar, geometry/channel_builder.h:25-33), before sfo_initialize.
 * A channel with pillars has a ChannelBuilder in the reference's sense. */
void sfo_add_circle_pillar(sfo_sim* s, double cx, double cy, double radius);
void sfo_add_rect_pillar(sfo_sim* s, double x0, double y0, double x1, double y1);

/* Capsule chemistry of the scalar (AdvectionDiffusion::applySourceSink /
 * applyChemistry, advection_diffusion.cpp:225-437): per capsule type up to 8
 * entries; a count of 0 is an empty vector, which selects the reference's
 * branches (simulation.cpp:640-653: physics kinetics when k_leach or
 * k_adsorb is non-empty, else the constant rates when either is set). */
#define SF_CHEM_TYPES 8
typedef struct sf_chemistry {
    int n_release, n_absorb, n_k_leach, n_C_eq, n_M_p, n_k_adsorb, n_k_desorb, n_Gamma_max;
    double release[SF_CHEM_TYPES], absorb[SF_CHEM_TYPES], k_leach[SF_CHEM_TYPES];
    double C_eq[SF_CHEM_TYPES], M_p_initial[SF_CHEM_TYPES], k_adsorb[SF_CHEM_TYPES];
    double k_desorb[SF_CHEM_TYPES], Gamma_max[SF_CHEM_TYPES];
} sf_chemistry;
void sfo_set_chemistry(sfo_sim* s, const sf_chemistry* c);
/* Per capsule: cumulative released / absorbed amounts and the reservoir
 * mass (-1: infinite); per marker: the surface coverage Gamma. */
void sfo_chemistry_state(const sfo_sim* s, double* released, double* absorbed, double* Mp,
                         double* gamma);

/* Capsule construction (reference capsule.cpp:7-141), returns its index. */
int sfo_add_capsule(sfo_sim* s, double cx, double cy, double radius, int nn,
                    const sf_membrane* m, int type);
/* Seeded rejection placement (reference simulation.cpp:220-274).  With
 * check_walls != 0 the channel-builder wall test is applied (walls at y = 0
 * and y = ny - 1).  Returns the number placed. */
int sfo_add_capsule_random(sfo_sim* s, int count, double x0, double y0,
                           double x1, double y1, double rmin, double rmax,
                           int nn, const sf_membrane* m, int type, int seed,
                           double min_gap, int max_attempts, int check_walls);

void sfo_initialize(sfo_sim* s);
void sfo_step(sfo_sim* s, int nsteps);

/* Zero-copy views of the state (reference LatticeField / Capsule data). */
int sfo_num_capsules(const sfo_sim* s);
int sfo_num_markers(const sfo_sim* s);
const int* sfo_capsule_offsets(const sfo_sim* s);   /* [ncaps+1] */
double* sfo_f(sfo_sim* s);        /* [9][ny][nx] post-stream populations */
double* sfo_rho(sfo_sim* s);      /* [ny][nx] */
double* sfo_ux(sfo_sim* s);
double* sfo_uy(sfo_sim* s);
double* sfo_Fx(sfo_sim* s);       /* lattice force of the last step */
double* sfo_Fy(sfo_sim* s);
double* sfo_pos(sfo_sim* s);      /* [M][2] marker positions */
double* sfo_vel(sfo_sim* s);      /* [M][2] marker velocities */
double* sfo_force(sfo_sim* s);    /* [M][2] marker membrane + contact force */
double* sfo_prev_len(sfo_sim* s); /* [M] Kelvin-Voigt previous edge length */
double* sfo_g(sfo_sim* s);        /* [ny*nx][9] scalar populations (AoS)  */
double* sfo_C(sfo_sim* s);        /* [ny][nx] concentration */
int sfo_last_capped(const sfo_sim* s);
int sfo_has_prev(const sfo_sim* s, int capsule);

/* Capsule geometry (reference capsule.cpp:159-204). */
double sfo_capsule_area(const sfo_sim* s, int c);
double sfo_capsule_perimeter(const sfo_sim* s, int c);
/* Taylor deformation D and inclination of the equivalent ellipse
 * (Capsule::deformationIndex / inclinationAngle, capsule.cpp:209-266). */
double sfo_capsule_deformation(const sfo_sim* s, int c);
double sfo_capsule_inclination(const sfo_sim* s, int c);
void sfo_capsule_centroid(const sfo_sim* s, int c, double* cx, double* cy);
double sfo_capsule_rest_area(const sfo_sim* s, int c);

/* Set the scalar field and its equilibrium populations g = w C
 * (the seeding used by reference tests/verification/test_pure_diffusion.cpp). */
void sfo_set_concentration(sfo_sim* s, const double* C);

/* Individual phases, exposed for unit tests of single operators. */
void sfo_compute_macroscopic(sfo_sim* s);
void sfo_spread_forces(sfo_sim* s);
void sfo_compute_membrane_forces(sfo_sim* s);
void sfo_compute_repulsion(sfo_sim* s);
double sfo_phi(double r);

/* Contact cell-list contents after the last repulsion pass: per marker the
 * number of (other-capsule) neighbour markers visited, and the flat list of
 * visited neighbour marker indices in visiting order. */
int sfo_contact_pairs(const sfo_sim* s, int* counts, int* list, int list_cap);

#ifdef __cplusplus
}
#endif
#endif
