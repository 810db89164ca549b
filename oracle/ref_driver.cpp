// ref_driver.cpp -- drives the reference engine's own hot-path classes.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
// reference sources (src/lbm, src/coupling, src/membrane, src/core,
// src/geometry) into oracle/_ref/libsfref*.so.  The reference's
// engine/simulation.cpp includes a CMake-generated header
// (<softflow/build_info.h>), so it is not compiled; this driver instead
// calls the same classes in the same order as Simulation::step()
// (reference src/engine/simulation.cpp:470-801) and restates the seeded
// placement of Simulation::addCapsuleRandom (:220-274).
//
// The C entry points mirror oracle/sfo.h (prefix sfr_ instead of sfo_) so
// the tests can run either implementation through one wrapper.
#include "sfo.h"

#include "lbm/lbm_solver.h"
#include "lbm/advection_diffusion.h"
#include "coupling/immersed_boundary.h"
#include "membrane/capsule_system.h"
#include "membrane/repulsion.h"
#include "io/vtk_writer.h"
#include "geometry/channel_builder.h"
#include "io/global_stats_writer.h"

#include <omp.h>

#include <memory>
#include <random>
#include <vector>
#include <cstring>

using namespace softflow;

namespace {

struct RefSim {
    SimulationParams p;
    std::unique_ptr<LBMSolver> lbm;
    CapsuleSystem caps;
    std::unique_ptr<RepulsionForce> rep;
    ImmersedBoundary ibm;
    std::unique_ptr<AdvectionDiffusion> adr;
    int last_capped = 0;
    // flat marker mirrors, refreshed after every call that changes them
    std::vector<double> pos, vel, frc, prev_len;
    std::vector<int> offsets;
    std::vector<double> C_mirror;
    std::unique_ptr<ChannelBuilder> builder;   // Simulation::setChannelBuilder
    // Simulation::scalar_release_rates_ / scalar_absorption_rates_ and the
    // kinetic vectors of ScalarParams (simulation.cpp:925-945)
    bool chem_on = false;
    std::vector<Real> release_rates, absorption_rates;
};

MembraneParams to_mp(const sf_membrane* m) {
    MembraneParams mp;
    mp.model = static_cast<MembraneModel>(m->model);
    mp.k_stretch = m->k_stretch;
    mp.G_s = m->G_s;
    mp.C_skalak = m->C_skalak;
    mp.wlc_L_max_ratio = m->wlc_L_max_ratio;
    mp.wlc_kBT_p = m->wlc_kBT_p;
    mp.wlc_k_pow = m->wlc_k_pow;
    mp.k_bend = m->k_bend;
    mp.use_helfrich_bending = m->use_helfrich != 0;
    mp.kappa_0 = m->kappa_0;
    mp.k_area = m->k_area;
    mp.k_perimeter = m->k_perimeter;
    mp.gamma_visc = m->gamma_visc;
    mp.eta_membrane = m->eta_membrane;
    return mp;
}

void sync_markers(RefSim* s) {
    int M = s->caps.totalNodes();
    s->pos.resize(2 * M);
    s->vel.resize(2 * M);
    s->frc.resize(2 * M);
    s->offsets.assign(1, 0);
    int k = 0;
    for (int c = 0; c < s->caps.numCapsules(); ++c) {
        const Capsule& cp = s->caps[c];
        for (int i = 0; i < cp.numNodes(); ++i, ++k) {
            s->pos[2 * k] = cp.nodePosition(i).x;
            s->pos[2 * k + 1] = cp.nodePosition(i).y;
            s->vel[2 * k] = cp.nodeVelocity(i).x;
            s->vel[2 * k + 1] = cp.nodeVelocity(i).y;
            s->frc[2 * k] = cp.nodeForce(i).x;
            s->frc[2 * k + 1] = cp.nodeForce(i).y;
        }
        s->offsets.push_back(k);
    }
    if (s->adr) {
        int N = s->p.nx * s->p.ny;
        s->C_mirror.assign(s->adr->concentrationData(0), s->adr->concentrationData(0) + N);
    }
}

}  // namespace

extern "C" {

void* sfr_create(const sf_params* in) {
    auto* s = new RefSim();
    SimulationParams& p = s->p;
    p.nx = in->nx;
    p.ny = in->ny;
    p.dt = in->dt;
    p.ibm_iterations = in->ibm_iterations;
    p.max_lattice_force = in->max_lattice_force;
    p.fluid.tau = in->tau;
    p.fluid.rho0 = in->rho0;
    p.fluid.boundary_type = static_cast<BoundaryType>(in->boundary_type);
    p.fluid.inlet_velocity = in->inlet_velocity;
    p.fluid.outlet_density = in->outlet_density;
    p.fluid.top_wall_velocity = in->top_wall_velocity;
    p.fluid.bottom_wall_velocity = in->bottom_wall_velocity;
    p.fluid.use_interpolated_bb = in->use_interpolated_bb != 0;
    p.fluid.periodic_y = in->periodic_y != 0;
    p.fluid.body_force_x = in->body_fx;
    p.fluid.body_force_y = in->body_fy;
    p.fluid.collision_model = static_cast<CollisionModel>(in->collision);
    p.fluid.mrt_se = in->mrt_se;
    p.fluid.mrt_s_eps = in->mrt_s_eps;
    p.fluid.mrt_sq = in->mrt_sq;
    p.repulsion.epsilon = in->rep_epsilon;
    p.repulsion.sigma = in->rep_sigma;
    p.repulsion.r_cut = in->rep_r_cut;
    p.repulsion.power = in->rep_power;
    p.repulsion.damping_normal = in->rep_damping_normal;
    p.repulsion.friction_coeff = in->rep_friction;
    p.scalar.enabled = in->scalar_enabled != 0;
    p.scalar.n_species = 1;
    p.scalar.diffusivity = {in->scalar_D};
    p.scalar.inlet_concentration = {in->scalar_inlet};
    p.scalar.periodic_y = in->scalar_periodic_y != 0;
    // Simulation constructor (simulation.cpp:125-140)
    s->lbm = std::make_unique<LBMSolver>(p);
    s->rep = std::make_unique<RepulsionForce>(p.repulsion);
    if (p.fluid.boundary_type == BoundaryType::PERIODIC) {      // simulation.cpp:129-132
        s->rep->setPeriodicX(static_cast<Real>(p.nx));
        s->caps.setPeriodicX(p.nx);
    }
    if (p.scalar.enabled) s->adr = std::make_unique<AdvectionDiffusion>(p.nx, p.ny, p.scalar);
    return s;
}

void sfr_destroy(void* h) { delete static_cast<RefSim*>(h); }

int sfr_add_capsule(void* h, double cx, double cy, double r, int nn, const sf_membrane* m,
                    int type) {
    auto* s = static_cast<RefSim*>(h);
    s->caps.addCapsule({cx, cy}, r, nn, to_mp(m), type);
    sync_markers(s);
    return s->caps.numCapsules() - 1;
}

// Restates simulation.cpp:220-274 with the same <random> engine and
// distributions, so the draws are the reference's.
int sfr_add_capsule_random(void* h, int count, double x0, double y0, double x1, double y1,
                           double rmin, double rmax, int nn, const sf_membrane* m, int type,
                           int seed, double min_gap, int max_attempts, int check_walls) {
    auto* s = static_cast<RefSim*>(h);
    std::mt19937 rng(static_cast<unsigned>(seed));
    std::uniform_real_distribution<Real> dx(x0, x1), dy(y0, y1), dr(rmin, rmax);
    int placed = 0, attempts = 0;
    int total_max = (max_attempts > 0) ? max_attempts : count * 500;
    MembraneParams mp = to_mp(m);
    while (placed < count && attempts < total_max) {
        Real cx = dx(rng);
        Real cy = dy(rng);
        Real r = dr(rng);
        bool overlap = false;
        for (int c = 0; c < s->caps.numCapsules(); ++c) {
            Vec2d oc = s->caps[c].centroid();
            Real orad = s->caps[c].effectiveRadius();
            if ((Vec2d{cx, cy} - oc).norm() < r + orad + min_gap) { overlap = true; break; }
        }
        if (check_walls) {
            if (cy - r < 0.0 + min_gap || cy + r > static_cast<Real>(s->p.ny - 1) - min_gap)
                overlap = true;
            if (s->builder)                            // simulation.cpp:256-261
                for (const auto& obs : s->builder->getObstacles())
                    if (obs->signedDistance(cx, cy) < r + min_gap) { overlap = true; break; }
        }
        if (!overlap) {
            s->caps.addCapsule({cx, cy}, r, nn, mp, type);
            placed++;
        }
        attempts++;
    }
    sync_markers(s);
    return placed;
}

void sfr_add_circle_pillar(void* h, double cx, double cy, double r) {
    auto* s = static_cast<RefSim*>(h);
    if (!s->builder) s->builder = std::make_unique<ChannelBuilder>(s->p.nx, s->p.ny);
    s->builder->addCirclePillar(cx, cy, r);
}

void sfr_add_rect_pillar(void* h, double x0, double y0, double x1, double y1) {
    auto* s = static_cast<RefSim*>(h);
    if (!s->builder) s->builder = std::make_unique<ChannelBuilder>(s->p.nx, s->p.ny);
    s->builder->addRectPillar(x0, y0, x1, y1);
}

void sfr_initialize(void* h) {
    auto* s = static_cast<RefSim*>(h);
    if (s->builder) {                          // simulation.cpp:430-434
        s->builder->setBoundaryType(s->p.fluid.boundary_type);
        s->builder->applyToField(s->lbm->field());
    }
    s->lbm->initialize();                      // simulation.cpp:436
    if (s->builder && s->p.fluid.use_interpolated_bb)   // :439-442
        s->lbm->setObstacles(s->builder->getObstacles());
    if (s->adr) s->adr->initialize(0.0);       // :446-448
    if (s->p.fluid.boundary_type == BoundaryType::PERIODIC)
        s->caps.setPeriodicX(s->p.nx);             // :456-458
    sync_markers(s);
}

void sfr_set_concentration(void* h, const double* C) {
    auto* s = static_cast<RefSim*>(h);
    if (!s->adr) return;
    int N = s->p.nx * s->p.ny;
    double* Cd = s->adr->concentrationData(0);
    double* g = s->adr->gData(0);
    for (int n = 0; n < N; ++n) {
        Cd[n] = C[n];
        for (int q = 0; q < 9; ++q) g[n * 9 + q] = D2Q9::w[q] * C[n];
    }
    sync_markers(s);
}

// One engine step in the order of simulation.cpp:470-700 (features that
// are off in every configuration of this path are omitted).
static void one_step(RefSim* s) {
    auto& field = s->lbm->field();
    field.clearForces();
    s->caps.clearAllForces();
    s->caps.computeAllMembraneForces();
    s->rep->computeAll(s->caps, 0.5, static_cast<Real>(s->p.ny) - 1.5);
    if (s->builder)                                // simulation.cpp:494-498
        for (const auto& obs : s->builder->getObstacles())
            s->rep->computeObstacleRepulsion(s->caps, *obs);
    if (s->p.ibm_iterations > 1) s->ibm.multiDirectForcing(s->caps, field, s->p.ibm_iterations);
    else s->ibm.spreadForces(s->caps, field);
    {
        const Real bfx = s->p.fluid.body_force_x, bfy = s->p.fluid.body_force_y;
        if (bfx != 0.0 || bfy != 0.0) {
            const int N = field.size();
            for (int n = 0; n < N; ++n) {
                if (field.cellTypeData()[n] == CellType::FLUID) {
                    field.FxData()[n] += bfx;
                    field.FyData()[n] += bfy;
                }
            }
        }
    }
    {
        const Real Fm = s->p.max_lattice_force, Fm2 = Fm * Fm;
        const int N = field.size();
        int capped = 0;
        for (int n = 0; n < N; ++n) {
            Real fx = field.FxData()[n], fy = field.FyData()[n];
            Real f2 = fx * fx + fy * fy;
            if (f2 > Fm2) {
                Real sc = Fm / std::sqrt(f2);
                field.FxData()[n] *= sc;
                field.FyData()[n] *= sc;
                ++capped;
            }
        }
        s->last_capped = capped;
    }
    s->lbm->step();
    if (s->adr) {
        s->adr->step(field);
        if (s->chem_on) {                     // simulation.cpp:640-653
            bool has_physics = !s->p.scalar.k_leach.empty() || !s->p.scalar.k_adsorb.empty();
            if (has_physics)
                s->adr->applyChemistry(s->caps, s->release_rates, s->absorption_rates,
                                       s->p.scalar);
            else if (!s->release_rates.empty() || !s->absorption_rates.empty())
                s->adr->applySourceSink(s->caps, s->release_rates, s->absorption_rates);
        }
    }
    s->ibm.interpolateVelocity(field, s->caps);
    s->caps.moveAllNodes(s->p.dt);
    if (!s->p.fluid.periodic_y) {
        const Real ymin = 1.5, ymax = static_cast<Real>(s->p.ny) - 1.5;
        for (int c = 0; c < s->caps.numCapsules(); ++c)
            for (auto& q : s->caps[c].positions()) {
                if (q.y < ymin) q.y = ymin;
                if (q.y > ymax) q.y = ymax;
            }
    }
}

void sfr_step(void* h, int n) {
    auto* s = static_cast<RefSim*>(h);
    for (int i = 0; i < n; ++i) one_step(s);
    sync_markers(s);
}

int sfr_num_capsules(void* h) { return static_cast<RefSim*>(h)->caps.numCapsules(); }
int sfr_num_markers(void* h) { return static_cast<RefSim*>(h)->caps.totalNodes(); }
const int* sfr_capsule_offsets(void* h) { return static_cast<RefSim*>(h)->offsets.data(); }
double* sfr_f(void* h) { return static_cast<RefSim*>(h)->lbm->field().fData(); }
double* sfr_rho(void* h) { return static_cast<RefSim*>(h)->lbm->field().rhoData(); }
double* sfr_ux(void* h) { return static_cast<RefSim*>(h)->lbm->field().uxData(); }
double* sfr_uy(void* h) { return static_cast<RefSim*>(h)->lbm->field().uyData(); }
double* sfr_Fx(void* h) { return static_cast<RefSim*>(h)->lbm->field().FxData(); }
double* sfr_Fy(void* h) { return static_cast<RefSim*>(h)->lbm->field().FyData(); }
double* sfr_pos(void* h) { return static_cast<RefSim*>(h)->pos.data(); }
double* sfr_vel(void* h) { return static_cast<RefSim*>(h)->vel.data(); }
double* sfr_force(void* h) { return static_cast<RefSim*>(h)->frc.data(); }
double* sfr_C(void* h) {
    auto* s = static_cast<RefSim*>(h);
    return s->adr ? s->C_mirror.data() : nullptr;
}
double* sfr_g(void* h) {
    auto* s = static_cast<RefSim*>(h);
    return s->adr ? s->adr->gData(0) : nullptr;
}
int sfr_last_capped(void* h) { return static_cast<RefSim*>(h)->last_capped; }
double sfr_capsule_area(void* h, int c) { return static_cast<RefSim*>(h)->caps[c].area(); }
double sfr_capsule_perimeter(void* h, int c) { return static_cast<RefSim*>(h)->caps[c].perimeter(); }
double sfr_capsule_deformation(void* h, int c) { return static_cast<RefSim*>(h)->caps[c].deformationIndex(); }
double sfr_capsule_inclination(void* h, int c) { return static_cast<RefSim*>(h)->caps[c].inclinationAngle(); }
void sfr_capsule_centroid(void* h, int c, double* x, double* y) {
    Vec2d r = static_cast<RefSim*>(h)->caps[c].centroid();
    *x = r.x;
    *y = r.y;
}
double sfr_phi(double r) { return PeskinDelta::phi(r); }

void sfr_set_chemistry(void* h, const sf_chemistry* c) {
    auto* s = static_cast<RefSim*>(h);
    auto vec = [](const double* v, int n) { return std::vector<Real>(v, v + n); };
    s->release_rates = vec(c->release, c->n_release);
    s->absorption_rates = vec(c->absorb, c->n_absorb);
    s->p.scalar.k_leach = vec(c->k_leach, c->n_k_leach);
    s->p.scalar.C_eq = vec(c->C_eq, c->n_C_eq);
    s->p.scalar.M_p_initial = vec(c->M_p_initial, c->n_M_p);
    s->p.scalar.k_adsorb = vec(c->k_adsorb, c->n_k_adsorb);
    s->p.scalar.k_desorb = vec(c->k_desorb, c->n_k_desorb);
    s->p.scalar.Gamma_max = vec(c->Gamma_max, c->n_Gamma_max);
    s->chem_on = true;
}

void sfr_chemistry_state(void* h, double* released, double* absorbed, double* Mp,
                         double* gamma) {
    auto* s = static_cast<RefSim*>(h);
    int k = 0;
    for (int c = 0; c < s->caps.numCapsules(); ++c) {
        if (released) released[c] = s->adr ? s->adr->getCapsuleReleased(c) : 0.0;
        if (absorbed) absorbed[c] = s->adr ? s->adr->getCapsuleAbsorbed(c) : 0.0;
        if (Mp) Mp[c] = s->adr ? s->adr->getCapsuleMp(c) : -1.0;
        for (int i = 0; i < s->caps[c].numNodes(); ++i, ++k)
            if (gamma) gamma[k] = s->adr ? s->adr->getNodeGamma(c, i) : 0.0;
    }
}

// The reference's VTK writer on the current state (default fields, periodic
// x as Simulation's constructor sets it, simulation.cpp:177-186).
void sfr_write_vtk(void* h, const char* dir, int step, int legacy) {
    auto* s = static_cast<RefSim*>(h);
    VTKWriter w(dir);
    if (s->p.fluid.boundary_type == BoundaryType::PERIODIC) w.setPeriodicX(s->p.nx);
    w.setLegacyMode(legacy != 0);
    if (s->adr) w.setAdvectionDiffusion(s->adr.get());
    w.writeFluidField(s->lbm->field(), step);
    w.writeCapsules(s->caps, step);
}

// One row of the reference's global_stats.csv on the current state.
void sfr_write_global_stats(void* h, const char* dir, int step, double time) {
    auto* s = static_cast<RefSim*>(h);
    GlobalStatsWriter w(dir);
    w.writeTimestep(s->lbm->field(), s->caps, step, time, s->adr.get());
}

// OpenMP thread count of the reference loops.  One thread makes the
// reference's spread (per-thread buffers, dynamic schedule) reproducible.
void sfr_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int sfr_get_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
