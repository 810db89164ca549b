// ref_engine.cpp -- the C entry points of oracle/sfo.h (prefix sfe_) over the
// reference's own engine object, softflow::Simulation
// (src/engine/simulation.h:33-285, simulation.cpp:124-801), compiled
// unmodified together with every other reference source.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile builds it into
// oracle/_ref/libsfengine.so with the deterministic flags and a stand-in for
// the CMake-generated <softflow/build_info.h> (provenance strings written
// into run_manifest.json; nothing on the step path reads them).  Where
// ref_driver.cpp restates the order of Simulation::step, this driver calls
// Simulation::addCapsuleRandom / initialize / step themselves, so the
// orchestration, the seeded placement, the body force and force cap, the
// move and the y-clamp are the reference's own code.
//
// Every output of the engine is switched off (intervals 0) and its
// output directory is a fresh temporary one.  The engine keeps its count of
// capped cells private, so sfe_last_capped returns -1.
#include "sfo.h"

#include "engine/simulation.h"
#include "coupling/delta_function.h"
#include "lbm/lattice.h"
#include "geometry/channel_builder.h"
#include "lbm/advection_diffusion.h"

#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace softflow;

namespace {

struct EngSim {
    SimulationParams p;
    std::unique_ptr<Simulation> sim;
    std::unique_ptr<ChannelBuilder> builder;   // pillars, handed over at initialize
    std::string outdir;
    // flat marker mirrors, refreshed after every call that changes them
    std::vector<double> pos, vel, frc, C_mirror;
    std::vector<int> offsets;
};

MembraneParams membrane(const sf_membrane* m) {
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

void mirror(EngSim* s) {
    CapsuleSystem& caps = s->sim->capsules();
    const int M = caps.totalNodes();
    s->pos.resize(2 * (size_t)M);
    s->vel.resize(2 * (size_t)M);
    s->frc.resize(2 * (size_t)M);
    s->offsets.assign(1, 0);
    int k = 0;
    for (int c = 0; c < caps.numCapsules(); ++c) {
        const Capsule& cp = caps[c];
        for (int i = 0; i < cp.numNodes(); ++i, ++k) {
            const Vec2d x = cp.nodePosition(i), v = cp.nodeVelocity(i), f = cp.nodeForce(i);
            s->pos[2 * k] = x.x;
            s->pos[2 * k + 1] = x.y;
            s->vel[2 * k] = v.x;
            s->vel[2 * k + 1] = v.y;
            s->frc[2 * k] = f.x;
            s->frc[2 * k + 1] = f.y;
        }
        s->offsets.push_back(k);
    }
    if (AdvectionDiffusion* adr = s->sim->advectionDiffusion()) {
        const int N = s->p.nx * s->p.ny;
        s->C_mirror.assign(adr->concentrationData(0), adr->concentrationData(0) + N);
    }
}

LatticeField& field(void* h) { return static_cast<EngSim*>(h)->sim->lbmSolver().field(); }

}  // namespace

extern "C" {

void* sfe_create(const sf_params* in) {
    auto* s = new EngSim();
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
    // no output of any kind, into a directory of its own
    char tmpl[] = "/tmp/sfengine_XXXXXX";
    const char* dir = mkdtemp(tmpl);
    s->outdir = dir ? dir : "/tmp";
    p.output_dir = s->outdir;
    p.output_interval = 0;
    p.vtk_dump_every = 0;
    p.csv_dump_every = 0;
    p.probe_dump_every = 0;
    p.stats_dump_every = 0;
    p.checkpoint_interval = 0;
    p.metrics_interval = 0;
    s->sim = std::make_unique<Simulation>(p);
    return s;
}

void sfe_destroy(void* h) { delete static_cast<EngSim*>(h); }

int sfe_add_capsule(void* h, double cx, double cy, double r, int nn, const sf_membrane* m,
                    int type) {
    auto* s = static_cast<EngSim*>(h);
    s->sim->addCapsule({cx, cy}, r, nn, membrane(m), type);
    mirror(s);
    return s->sim->capsules().numCapsules() - 1;
}

// Simulation::addCapsuleRandom itself (its wall test is always on; the
// pillars join the rejection once they are handed over, so callers add
// pillars through the engine before placing among them).
int sfe_add_capsule_random(void* h, int count, double x0, double y0, double x1, double y1,
                           double rmin, double rmax, int nn, const sf_membrane* m, int type,
                           int seed, double min_gap, int max_attempts, int check_walls) {
    auto* s = static_cast<EngSim*>(h);
    if (!check_walls) return -1;
    if (s->builder) s->sim->setChannelBuilder(*s->builder);
    const int before = s->sim->capsules().numCapsules();
    s->sim->addCapsuleRandom(count, x0, y0, x1, y1, rmin, rmax, nn, membrane(m), type, seed,
                             min_gap, max_attempts);
    mirror(s);
    return s->sim->capsules().numCapsules() - before;
}

void sfe_add_circle_pillar(void* h, double cx, double cy, double r) {
    auto* s = static_cast<EngSim*>(h);
    if (!s->builder) s->builder = std::make_unique<ChannelBuilder>(s->p.nx, s->p.ny);
    s->builder->addCirclePillar(cx, cy, r);
}

void sfe_add_rect_pillar(void* h, double x0, double y0, double x1, double y1) {
    auto* s = static_cast<EngSim*>(h);
    if (!s->builder) s->builder = std::make_unique<ChannelBuilder>(s->p.nx, s->p.ny);
    s->builder->addRectPillar(x0, y0, x1, y1);
}

void sfe_initialize(void* h) {
    auto* s = static_cast<EngSim*>(h);
    if (s->builder) s->sim->setChannelBuilder(*s->builder);
    s->sim->initialize();
    mirror(s);
}

void sfe_set_concentration(void* h, const double* C) {
    auto* s = static_cast<EngSim*>(h);
    AdvectionDiffusion* adr = s->sim->advectionDiffusion();
    if (!adr) return;
    const int N = s->p.nx * s->p.ny;
    double* Cd = adr->concentrationData(0);
    double* g = adr->gData(0);
    for (int n = 0; n < N; ++n) {
        Cd[n] = C[n];
        for (int q = 0; q < 9; ++q) g[n * 9 + q] = D2Q9::w[q] * C[n];
    }
    mirror(s);
}

void sfe_step(void* h, int n) {
    auto* s = static_cast<EngSim*>(h);
    for (int i = 0; i < n; ++i) s->sim->step();
    mirror(s);
}

int sfe_num_capsules(void* h) { return static_cast<EngSim*>(h)->sim->capsules().numCapsules(); }
int sfe_num_markers(void* h) { return static_cast<EngSim*>(h)->sim->capsules().totalNodes(); }
const int* sfe_capsule_offsets(void* h) { return static_cast<EngSim*>(h)->offsets.data(); }
double* sfe_f(void* h) { return field(h).fData(); }
double* sfe_rho(void* h) { return field(h).rhoData(); }
double* sfe_ux(void* h) { return field(h).uxData(); }
double* sfe_uy(void* h) { return field(h).uyData(); }
double* sfe_Fx(void* h) { return field(h).FxData(); }
double* sfe_Fy(void* h) { return field(h).FyData(); }
double* sfe_pos(void* h) { return static_cast<EngSim*>(h)->pos.data(); }
double* sfe_vel(void* h) { return static_cast<EngSim*>(h)->vel.data(); }
double* sfe_force(void* h) { return static_cast<EngSim*>(h)->frc.data(); }
double* sfe_C(void* h) {
    auto* s = static_cast<EngSim*>(h);
    return s->sim->advectionDiffusion() ? s->C_mirror.data() : nullptr;
}
double* sfe_g(void* h) {
    AdvectionDiffusion* adr = static_cast<EngSim*>(h)->sim->advectionDiffusion();
    return adr ? adr->gData(0) : nullptr;
}
int sfe_last_capped(void*) { return -1; }
double sfe_capsule_area(void* h, int c) {
    return static_cast<EngSim*>(h)->sim->capsules()[c].area();
}
double sfe_capsule_perimeter(void* h, int c) {
    return static_cast<EngSim*>(h)->sim->capsules()[c].perimeter();
}
double sfe_capsule_deformation(void* h, int c) {
    return static_cast<EngSim*>(h)->sim->capsules()[c].deformationIndex();
}
double sfe_capsule_inclination(void* h, int c) {
    return static_cast<EngSim*>(h)->sim->capsules()[c].inclinationAngle();
}
void sfe_capsule_centroid(void* h, int c, double* x, double* y) {
    const Vec2d r = static_cast<EngSim*>(h)->sim->capsules()[c].centroid();
    *x = r.x;
    *y = r.y;
}
double sfe_phi(double r) { return PeskinDelta::phi(r); }

// The engine's own chemistry setters (simulation.cpp:930-970), one capsule
// type per vector entry.
void sfe_set_chemistry(void* h, const sf_chemistry* c) {
    auto* s = static_cast<EngSim*>(h);
    for (int t = 0; t < c->n_release; ++t) s->sim->setScalarReleaseRate(t, c->release[t]);
    for (int t = 0; t < c->n_absorb; ++t) s->sim->setScalarAbsorptionRate(t, c->absorb[t]);
    for (int t = 0; t < c->n_k_leach; ++t)
        s->sim->setLeachingParams(t, c->k_leach[t], t < c->n_C_eq ? c->C_eq[t] : 0.0);
    for (int t = 0; t < c->n_k_adsorb; ++t)
        s->sim->setAdsorptionParams(t, c->k_adsorb[t], t < c->n_k_desorb ? c->k_desorb[t] : 0.0,
                                    t < c->n_Gamma_max ? c->Gamma_max[t] : 0.0);
    for (int t = 0; t < c->n_M_p; ++t) s->sim->setParticleMass(t, c->M_p_initial[t]);
}

void sfe_chemistry_state(void* h, double* released, double* absorbed, double* Mp,
                         double* gamma) {
    auto* s = static_cast<EngSim*>(h);
    AdvectionDiffusion* adr = s->sim->advectionDiffusion();
    CapsuleSystem& caps = s->sim->capsules();
    int k = 0;
    for (int c = 0; c < caps.numCapsules(); ++c) {
        if (released) released[c] = adr ? adr->getCapsuleReleased(c) : 0.0;
        if (absorbed) absorbed[c] = adr ? adr->getCapsuleAbsorbed(c) : 0.0;
        if (Mp) Mp[c] = adr ? adr->getCapsuleMp(c) : -1.0;
        for (int i = 0; i < caps[c].numNodes(); ++i, ++k)
            if (gamma) gamma[k] = adr ? adr->getNodeGamma(c, i) : 0.0;
    }
}

void sfe_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int sfe_get_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
