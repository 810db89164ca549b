// engine_gpu_hook.cpp -- the reference's own Python module (python/bindings.cpp
// with the engine, compiled unmodified) with its step routed through
// libsoftflow_b200.so.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile links this file into
// oracle/_ref/pybind/softflow_core*.so together with the reference's
// bindings.cpp and every engine source, with the linker's symbol wrapping
// (-Wl,--wrap) on six Simulation members the binding calls.  No reference
// source is copied or edited: the binding's calls land here first.
//
//   Simulation(params)       forgets any hook state left at the same address
//   addCapsule(...)          records the capsule (centre, radius, nodes,
//                            membrane, type), then adds it
//   setChannelBuilder(...)   marks the simulation for the CPU path (pillars)
//   addCapsuleRandom(...)    places with the library's seeded placement
//                            (sfg_place_random: the reference's std::mt19937
//                            draws and rejection test, simulation.cpp:220-274)
//                            and adds each capsule through addCapsule
//   step() / run(n)          on the CPU as the reference does, or, with the
//                            environment variable SOFTFLOW_GPU set to fp64,
//                            fp32 or fp16s when the simulation takes its
//                            first step, through the GPU library
//
// The GPU path replaces steps 0-10 of Simulation::step (simulation.cpp:
// 470-675): a context is built from params() and the recorded capsules at
// the first step, the host state (populations, markers, scalar) is uploaded
// whenever it differs from what the last step left, the steps run on the
// device, and every host mirror the binding exposes (populations, rho, u, F,
// marker positions, velocities, forces, concentration) is written back, so
// Python sees the state the CPU path would have.  run(n) makes one upload
// and one download around n device steps and ends with finalize(), as
// Simulation::run does.  The interval-gated tail of step (output writers,
// checkpoints, stability checks, the step callback, simulation.cpp:700-786)
// and the reference features this library does not build (pillars set
// through setChannelBuilder, inserters, lubrication, adhesion, free
// surface, viscosity fields, non-periodic capsule channels) stay on the CPU
// path: a simulation that uses them runs on the CPU, with a notice.
#include "engine/simulation.h"
#include "geometry/channel_builder.h"
#include "lbm/advection_diffusion.h"
#include "softflow_gpu.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

using softflow::MembraneParams;
using softflow::Simulation;
using softflow::SimulationParams;
using softflow::Vec2d;

extern "C" {
// the reference's members (Itanium C++ ABI: `this` first)
void __real__ZN8softflow10SimulationC1ERKNS_16SimulationParamsE(Simulation*,
                                                                 const SimulationParams&);
void __real__ZN8softflow10Simulation10addCapsuleENS_5Vec2dEdiRKNS_14MembraneParamsEi(
    Simulation*, Vec2d, double, int, const MembraneParams&, int);
void __real__ZN8softflow10Simulation16addCapsuleRandomEiddddddiRKNS_14MembraneParamsEiidi(
    Simulation*, int, double, double, double, double, double, double, int,
    const MembraneParams&, int, int, double, int);
void __real__ZN8softflow10Simulation4stepEv(Simulation*);
void __real__ZN8softflow10Simulation17setChannelBuilderERKNS_14ChannelBuilderE(
    Simulation*, const softflow::ChannelBuilder&);
void __real__ZN8softflow10Simulation3runEi(Simulation*, int);
}

namespace {

struct CapsuleSpec {
    double cx, cy, r;
    int nodes;
    MembraneParams mp;
    int type;
};

struct Hook {
    std::vector<CapsuleSpec> caps;
    bool unsupported = false;       // a feature only the CPU path has
    bool decided = false;           // GPU or CPU chosen at the first step
    bool gpu = false;
    sfg_context* ctx = nullptr;
    int M = 0;
    // host state as the last device step left it (upload only on change)
    std::vector<double> f, pos, vel, C, g;
};

std::mutex g_mu;
std::unordered_map<const Simulation*, Hook> g_hooks;

void check(int rc) {
    if (rc != SFG_OK) throw std::runtime_error(std::string("softflow_b200: ") + sfg_last_error());
}

sfg_membrane_params to_sfg(const MembraneParams& m) {
    sfg_membrane_params o{};
    o.model = static_cast<int>(m.model);
    o.k_stretch = m.k_stretch;
    o.G_s = m.G_s;
    o.C_skalak = m.C_skalak;
    o.wlc_L_max_ratio = m.wlc_L_max_ratio;
    o.wlc_kBT_p = m.wlc_kBT_p;
    o.wlc_k_pow = m.wlc_k_pow;
    o.k_bend = m.k_bend;
    o.use_helfrich = m.use_helfrich_bending ? 1 : 0;
    o.kappa_0 = m.kappa_0;
    o.k_area = m.k_area;
    o.k_perimeter = m.k_perimeter;
    o.gamma_visc = m.gamma_visc;
    o.eta_membrane = m.eta_membrane;
    return o;
}

int precision_from_env() {
    const char* v = std::getenv("SOFTFLOW_GPU");
    if (!v || !*v) return -1;
    if (!std::strcmp(v, "fp64")) return SFG_FP64;
    if (!std::strcmp(v, "fp32")) return SFG_FP32;
    if (!std::strcmp(v, "fp16s")) return SFG_FP16S;
    throw std::runtime_error("SOFTFLOW_GPU must be fp64, fp32 or fp16s");
}

// What the CPU path would need that this library does not build.
const char* unsupported_feature(const Simulation& s, const Hook& h) {
    const SimulationParams& p = s.params();
    if (h.unsupported) return "pillars (setChannelBuilder) or inserters";
    if (p.fluid.boundary_type != softflow::BoundaryType::PERIODIC && !h.caps.empty())
        return "capsules in a non-periodic channel";
    if (p.lubrication.enabled) return "lubrication";
    if (p.adhesion.enabled) return "adhesion";
    if (p.shan_chen.enabled) return "Shan-Chen";
    if (p.fluid.viscosity_contrast) return "viscosity contrast";
    if (p.fluid.non_newtonian_model != softflow::NonNewtonianModel::NONE) return "non-Newtonian";
    if ((p.fluid.gravity_x != 0.0 || p.fluid.gravity_y != 0.0) &&
        (p.fluid.apply_gravity_to_capsules || p.fluid.apply_gravity_to_fluid))
        return "gravity";
    if (p.scalar.enabled && p.scalar.n_species != 1) return "several scalar species";
    if (p.ml.enabled) return "the engine's surrogate training";
    if ((int)h.caps.size() != s.capsules().numCapsules()) return "capsules added outside the binding";
    for (const CapsuleSpec& c : h.caps)
        if (c.mp.shape != softflow::CapsuleShape::CIRCLE || c.mp.is_rigid || c.mp.density != 1.0 ||
            c.mp.viscosity_ratio != 1.0)
            return "non-circular, rigid, buoyant or viscosity-contrast capsules";
    return nullptr;
}

void build_context(Simulation& s, Hook& h, int precision) {
    const SimulationParams& p = s.params();
    check(sfg_create(0, precision, &h.ctx));
    sfg_channel_params cp{};
    cp.nx = p.nx;
    cp.ny = p.ny;
    cp.collision = static_cast<int>(p.fluid.collision_model);
    cp.tau = p.fluid.tau;
    cp.rho0 = p.fluid.rho0;
    cp.mrt_se = p.fluid.mrt_se;
    cp.mrt_s_eps = p.fluid.mrt_s_eps;
    cp.mrt_sq = p.fluid.mrt_sq;
    cp.body_fx = p.fluid.body_force_x;
    cp.body_fy = p.fluid.body_force_y;
    cp.periodic_y = p.fluid.periodic_y ? 1 : 0;
    cp.max_lattice_force = p.max_lattice_force;
    cp.ibm_iterations = p.ibm_iterations;
    cp.dt = p.dt;
    cp.rep_epsilon = p.repulsion.epsilon;
    cp.rep_sigma = p.repulsion.sigma;
    cp.rep_r_cut = p.repulsion.r_cut;
    cp.rep_power = p.repulsion.power;
    cp.rep_damping_normal = p.repulsion.damping_normal;
    cp.rep_friction = p.repulsion.friction_coeff;
    cp.scalar_enabled = p.scalar.enabled ? 1 : 0;
    cp.scalar_D = p.scalar.diffusivity.empty() ? 0.01 : p.scalar.diffusivity[0];
    cp.scalar_periodic_y = p.scalar.periodic_y ? 1 : 0;
    cp.scalar_inlet = p.scalar.inlet_concentration.empty() ? 0.0 : p.scalar.inlet_concentration[0];
    cp.boundary_type = static_cast<int>(p.fluid.boundary_type);
    cp.inlet_velocity = p.fluid.inlet_velocity;
    cp.outlet_density = p.fluid.outlet_density;
    cp.top_wall_velocity = p.fluid.top_wall_velocity;
    cp.bottom_wall_velocity = p.fluid.bottom_wall_velocity;
    cp.use_interpolated_bb = p.fluid.use_interpolated_bb ? 1 : 0;
    int ch = 0;
    check(sfg_add_channel(h.ctx, &cp, &ch));
    for (const CapsuleSpec& c : h.caps) {
        const sfg_membrane_params mp = to_sfg(c.mp);
        sfg_capsule_rest rest{};
        const int cap = 4096;
        std::vector<double> pos(2 * cap), len(cap), ang(cap), ds(cap);
        check(sfg_build_circle_capsule(c.cx, c.cy, c.r, c.nodes, &mp, &rest, pos.data(),
                                       len.data(), ang.data(), ds.data(), cap));
        int id = 0;
        check(sfg_add_capsule(h.ctx, ch, &mp, &rest, pos.data(), len.data(), ang.data(),
                              ds.data(), &id));
        if (c.type != 0) check(sfg_set_capsule_type(h.ctx, ch, id, c.type));
    }
    check(sfg_initialize(h.ctx));
    h.M = s.capsules().totalNodes();
}

void gather_markers(Simulation& s, std::vector<double>& pos, std::vector<double>& vel) {
    softflow::CapsuleSystem& caps = s.capsules();
    pos.clear();
    vel.clear();
    for (int c = 0; c < caps.numCapsules(); ++c) {
        for (const Vec2d& x : caps[c].positions()) { pos.push_back(x.x); pos.push_back(x.y); }
        for (const Vec2d& v : caps[c].velocities()) { vel.push_back(v.x); vel.push_back(v.y); }
    }
}

// Host -> device where the host differs from what the last device step left.
void upload(Simulation& s, Hook& h) {
    softflow::LatticeField& fld = s.lbmSolver().field();
    const size_t nf = 9 * (size_t)fld.size();
    if (h.f.size() != nf || std::memcmp(h.f.data(), fld.fData(), nf * sizeof(double)))
        check(sfg_set_populations(h.ctx, 0, fld.fData()));
    std::vector<double> pos, vel;
    gather_markers(s, pos, vel);
    if (pos != h.pos || vel != h.vel)
        check(sfg_set_markers(h.ctx, 0, pos.data(), vel.data()));
    if (softflow::AdvectionDiffusion* adr = s.advectionDiffusion()) {
        const size_t N = (size_t)fld.size();
        if (h.C.size() != N || std::memcmp(h.C.data(), adr->concentrationData(0), N * 8) ||
            std::memcmp(h.g.data(), adr->gData(0), 9 * N * 8))
            check(sfg_set_scalar_state(h.ctx, 0, adr->concentrationData(0), adr->gData(0)));
    }
}

// Device -> every host mirror the binding exposes.
void download(Simulation& s, Hook& h) {
    softflow::LatticeField& fld = s.lbmSolver().field();
    const size_t N = (size_t)fld.size();
    check(sfg_get_populations(h.ctx, 0, fld.fData()));
    check(sfg_get_macroscopic(h.ctx, 0, fld.rhoData(), fld.uxData(), fld.uyData(), fld.FxData(),
                              fld.FyData()));
    std::vector<double> pos(2 * (size_t)h.M), vel(2 * (size_t)h.M), frc(2 * (size_t)h.M);
    if (h.M > 0) check(sfg_get_markers(h.ctx, 0, pos.data(), vel.data(), frc.data()));
    softflow::CapsuleSystem& caps = s.capsules();
    size_t k = 0;
    for (int c = 0; c < caps.numCapsules(); ++c) {
        auto& X = caps[c].positions();
        auto& V = caps[c].velocities();
        auto& F = caps[c].forces();
        for (size_t i = 0; i < X.size(); ++i, ++k) {
            X[i] = Vec2d(pos[2 * k], pos[2 * k + 1]);
            V[i] = Vec2d(vel[2 * k], vel[2 * k + 1]);
            F[i] = Vec2d(frc[2 * k], frc[2 * k + 1]);
        }
    }
    h.f.assign(fld.fData(), fld.fData() + 9 * N);
    h.pos = std::move(pos);
    h.vel = std::move(vel);
    if (softflow::AdvectionDiffusion* adr = s.advectionDiffusion()) {
        check(sfg_get_concentration(h.ctx, 0, adr->concentrationData(0), adr->gData(0)));
        h.C.assign(adr->concentrationData(0), adr->concentrationData(0) + N);
        h.g.assign(adr->gData(0), adr->gData(0) + 9 * N);
    }
}

// Runs n steps on the device if this simulation takes the GPU path; false
// when it runs on the CPU.
bool gpu_steps(Simulation& s, int n) {
    std::lock_guard<std::mutex> lock(g_mu);
    Hook& h = g_hooks[&s];
    if (!h.decided) {
        h.decided = true;
        const int prec = precision_from_env();
        if (prec >= 0) {
            if (const char* why = unsupported_feature(s, h)) {
                std::cerr << "softflow_b200: " << why << " runs on the CPU path\n";
            } else {
                build_context(s, h, prec);
                h.gpu = true;
            }
        }
    }
    if (!h.gpu) return false;
    upload(s, h);
    check(sfg_step(h.ctx, n));
    unsigned st = 0;
    check(sfg_synchronize(h.ctx, &st));
    download(s, h);
    s.setCurrentStep(s.currentStep() + n);
    return true;
}

void forget(const Simulation* s) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_hooks.find(s);
    if (it == g_hooks.end()) return;
    if (it->second.ctx) sfg_destroy(it->second.ctx);
    g_hooks.erase(it);
}

}  // namespace

extern "C" {

void __wrap__ZN8softflow10SimulationC1ERKNS_16SimulationParamsE(Simulation* s,
                                                                 const SimulationParams& p) {
    forget(s);                                // an earlier object at this address
    __real__ZN8softflow10SimulationC1ERKNS_16SimulationParamsE(s, p);
}

void __wrap__ZN8softflow10Simulation10addCapsuleENS_5Vec2dEdiRKNS_14MembraneParamsEi(
    Simulation* s, Vec2d center, double radius, int num_nodes, const MembraneParams& mp,
    int type) {
    {
        std::lock_guard<std::mutex> lock(g_mu);
        Hook& h = g_hooks[s];
        if (h.decided) h.unsupported = true;  // added after the first step
        h.caps.push_back({center.x, center.y, radius, num_nodes, mp, type});
    }
    __real__ZN8softflow10Simulation10addCapsuleENS_5Vec2dEdiRKNS_14MembraneParamsEi(
        s, center, radius, num_nodes, mp, type);
}

void __wrap__ZN8softflow10Simulation16addCapsuleRandomEiddddddiRKNS_14MembraneParamsEiidi(
    Simulation* s, int count, double x0, double y0, double x1, double y1, double rmin,
    double rmax, int num_nodes, const MembraneParams& mp, int type, int seed, double min_gap,
    int max_attempts) {
    softflow::CapsuleSystem& caps = s->capsules();
    const int n0 = caps.numCapsules();
    std::vector<double> cen(2 * (size_t)n0), rad((size_t)n0);
    for (int c = 0; c < n0; ++c) {
        const Vec2d g = caps[c].centroid();
        cen[2 * c] = g.x;
        cen[2 * c + 1] = g.y;
        rad[c] = caps[c].effectiveRadius();
    }
    std::vector<double> oc(2 * (size_t)std::max(count, 1)), orad((size_t)std::max(count, 1));
    int placed = 0, attempts = 0;
    check(sfg_place_random(count, x0, y0, x1, y1, rmin, rmax, num_nodes, seed, min_gap,
                           max_attempts, 1, s->params().nx, s->params().ny, n0, cen.data(),
                           rad.data(), std::max(count, 1), oc.data(), orad.data(), &placed,
                           &attempts));
    for (int i = 0; i < placed; ++i)
        __wrap__ZN8softflow10Simulation10addCapsuleENS_5Vec2dEdiRKNS_14MembraneParamsEi(
            s, Vec2d(oc[2 * i], oc[2 * i + 1]), orad[i], num_nodes, mp, type);
    std::cout << "Placed " << placed << "/" << count << " capsules (" << attempts
              << " attempts)" << std::endl;
}

void __wrap__ZN8softflow10Simulation17setChannelBuilderERKNS_14ChannelBuilderE(
    Simulation* s, const softflow::ChannelBuilder& b) {
    {
        std::lock_guard<std::mutex> lock(g_mu);
        g_hooks[s].unsupported = true;        // pillars: the CPU path
    }
    __real__ZN8softflow10Simulation17setChannelBuilderERKNS_14ChannelBuilderE(s, b);
}

void __wrap__ZN8softflow10Simulation4stepEv(Simulation* s) {
    if (!gpu_steps(*s, 1)) __real__ZN8softflow10Simulation4stepEv(s);
}

void __wrap__ZN8softflow10Simulation3runEi(Simulation* s, int num_steps) {
    if (num_steps > 0 && gpu_steps(*s, num_steps)) {
        s->finalize();
        return;
    }
    __real__ZN8softflow10Simulation3runEi(s, num_steps);
}

}  // extern "C"
