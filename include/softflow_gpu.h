/*
 * softflow_gpu.h -- C ABI of the B200 implementation of the SoftFlow
 * per-timestep hot path (libsoftflow_b200.so).
 *
 * The library replaces the bodies of the reference engine's step
 * (ramc77/SoftFlow src/engine/simulation.cpp:470-801): lattice moments,
 * BGK / MRT / regularized collision with Guo forcing, streaming with
 * halfway bounce-back, body force and force cap, Peskin 4-point IBM spread /
 * interpolation / multi-direct forcing, membrane forces, soft contact,
 * marker motion, and the advection-diffusion scalar step.
 *
 * Conventions
 *   - Every entry point returns an int status: SFG_OK (0) or an SFG_ERR_*
 *     code; sfg_last_error() gives the message.  No exception crosses the
 *     ABI.  A caller maps a nonzero status to its own error type (the
 *     reference engine throws std::runtime_error, which pybind11 turns into
 *     a Python exception).
 *   - Host arrays are FP64 in the reference's canonical layouts:
 *     populations [9][ny][nx] (LatticeField::f_, lattice_field.h:53-56),
 *     scalar fields [ny][nx], marker vectors [markers][2] in capsule-major,
 *     node-minor order (CapsuleSystem iteration order).
 *   - A context holds one or more independent channels ("ensemble"); every
 *     step advances all of them with one launch per kernel phase.
 *   - A context is driven by one host thread.
 */
#ifndef SOFTFLOW_GPU_H
#define SOFTFLOW_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SFG_ABI_VERSION 2

enum sfg_status {
    SFG_OK = 0,
    SFG_ERR_ARG = 1,       /* invalid argument (caller error)                 */
    SFG_ERR_STATE = 2,     /* call not valid in the context's current state   */
    SFG_ERR_CUDA = 3,      /* CUDA runtime error (message has the CUDA text)  */
    SFG_ERR_CAPACITY = 4,  /* a fixed capacity was exceeded                   */
    SFG_ERR_NUMERIC = 5    /* non-finite marker state was detected            */
};

/* Storage precision of the lattice populations. */
enum sfg_precision {
    SFG_FP64 = 0,   /* FP64 storage and arithmetic                              */
    SFG_FP32 = 1,   /* FP32 storage and arithmetic                              */
    SFG_FP16S = 2   /* binary16 storage of (f - w) * 2^12 with stochastic rounding
                       inside the time loop, FP32 arithmetic                    */
};

enum sfg_collision { SFG_BGK = 0, SFG_MRT = 1, SFG_REGULARIZED = 2 };
enum sfg_membrane_model { SFG_HOOKEAN = 0, SFG_NEO_HOOKEAN = 1, SFG_SKALAK = 2, SFG_WLC = 3 };

/* Channel parameters: the fields of the reference SimulationParams that the
 * path reads (src/core/parameters.h:41-342): SOLID rows 0 and ny-1 (or
 * periodic in y); periodic in x, a Zou-He inlet / outlet pair of columns,
 * or SOLID columns (closed box). */
typedef struct sfg_channel_params {
    int nx, ny;
    int collision;              /* sfg_collision                               */
    double tau, rho0;
    double mrt_se, mrt_s_eps, mrt_sq;
    double body_fx, body_fy;
    int periodic_y;
    double max_lattice_force;
    int ibm_iterations;
    double dt;
    double rep_epsilon, rep_sigma, rep_r_cut;
    int rep_power;
    double rep_damping_normal, rep_friction;
    int scalar_enabled;
    double scalar_D;
    int scalar_periodic_y;
    double scalar_inlet;
    /* fluid boundaries (FluidParams, parameters.h:44-46, 87-88):
     * boundary_type is sfg_boundary; inlet_velocity is the centre-line
     * speed of the parabolic Zou-He inlet profile, outlet_density the Zou-He
     * outlet pressure (zou_he_boundary.cpp:17-85); moving top / bottom wall
     * speeds along x (moving_wall.cpp:14-64).  Channels other than PERIODIC
     * carry no capsules and no scalar here. */
    int boundary_type;
    double inlet_velocity, outlet_density;
    double top_wall_velocity, bottom_wall_velocity;
    /* Bouzidi interpolated bounce-back on the links of a channel with
     * pillars (FluidParams::use_interpolated_bb, parameters.h:89;
     * interpolated_bounce_back.cpp); no effect without pillars */
    int use_interpolated_bb;
} sfg_channel_params;

/* BoundaryType (reference core/types.h:58-62). */
enum sfg_boundary { SFG_INLET_OUTLET = 0, SFG_PERIODIC = 1, SFG_CLOSED = 2 };

/* Membrane parameters (reference MembraneParams, parameters.h:82-136). */
typedef struct sfg_membrane_params {
    int model;                  /* sfg_membrane_model */
    double k_stretch, G_s, C_skalak;
    double wlc_L_max_ratio, wlc_kBT_p, wlc_k_pow;
    double k_bend;
    int use_helfrich;
    double kappa_0;
    double k_area, k_perimeter, gamma_visc, eta_membrane;
} sfg_membrane_params;

/* Rest state of one capsule (reference Capsule constructor,
 * src/membrane/capsule.cpp:7-141). */
typedef struct sfg_capsule_rest {
    int num_nodes;
    double rest_area, rest_perimeter;
    double wlc_kBT_p, wlc_k_pow;    /* resolved WLC constants (capsule.cpp:92-123) */
} sfg_capsule_rest;

typedef struct sfg_context sfg_context;

/* ---- library ------------------------------------------------------------ */
int sfg_abi_version(void);
/* Message of the last failed call on this thread (empty if none). */
const char* sfg_last_error(void);

/* ---- host-side setup helpers (no device work) ---------------------------
 * Rest geometry of a circular capsule: replaces Capsule::Capsule
 * (capsule.cpp:7-141) for CapsuleShape::CIRCLE.  num_nodes <= 0 selects
 * Capsule::computeOptimalNodes (capsule.h:14-17); *rest_out->num_nodes
 * reports the count used.  Output arrays hold at least that many nodes
 * (pos: 2 per node).  rest_ang / rest_ds are zero unless use_helfrich. */
int sfg_build_circle_capsule(double cx, double cy, double radius, int num_nodes,
                             const sfg_membrane_params* mp, sfg_capsule_rest* rest_out,
                             double* pos_out, double* rest_len_out, double* rest_ang_out,
                             double* rest_ds_out, int capacity);

/* Seeded rejection placement: replaces Simulation::addCapsuleRandom
 * (simulation.cpp:220-274), same std::mt19937 draws.  existing_centroid
 * [n_existing][2] and existing_radius [n_existing] describe capsules already
 * in the channel.  Placed centres/radii go to out_center [cap][2] and
 * out_radius [cap]; *n_placed and *n_attempts are set. */
int sfg_place_random(int count, double x0, double y0, double x1, double y1, double rmin,
                     double rmax, int num_nodes, int seed, double min_gap, int max_attempts,
                     int check_walls, int nx, int ny, int n_existing,
                     const double* existing_centroid, const double* existing_radius,
                     int capacity, double* out_center, double* out_radius, int* n_placed,
                     int* n_attempts);

/* sfg_place_random with the channel's pillars ([n_pillars][5]: kind 0 circle
 * (a, b) radius c, kind 1 rectangle (a, b)-(c, d)): with check_walls a
 * candidate whose centre lies closer than r + min_gap to a pillar is
 * rejected, as Simulation::addCapsuleRandom does with a channel builder
 * (simulation.cpp:250-262). */
int sfg_place_random_pillars(int count, double x0, double y0, double x1, double y1,
                             double rmin, double rmax, int num_nodes, int seed, double min_gap,
                             int max_attempts, int check_walls, int nx, int ny, int n_existing,
                             const double* existing_centroid, const double* existing_radius,
                             int capacity, double* out_center, double* out_radius, int* n_placed,
                             int* n_attempts, int n_pillars, const double* pillars);

/* ---- context ------------------------------------------------------------ */
int sfg_create(int device, int precision, sfg_context** out);
int sfg_destroy(sfg_context* ctx);

/* Adds a channel (before sfg_initialize).  Replaces LBMSolver construction
 * (lbm_solver.cpp:12-67) and the parameter plumbing of Simulation. */
int sfg_add_channel(sfg_context* ctx, const sfg_channel_params* p, int* channel_out);

/* Adds one capsule to a channel (before sfg_initialize): node positions
 * pos [n][2], rest edge lengths, Helfrich rest angles and arc lengths (may be
 * NULL when use_helfrich == 0).  Replaces CapsuleSystem::addCapsule
 * (capsule_system.cpp:5-9). */
int sfg_add_capsule(sfg_context* ctx, int channel, const sfg_membrane_params* mp,
                    const sfg_capsule_rest* rest, const double* pos, const double* rest_len,
                    const double* rest_ang, const double* rest_ds, int* capsule_out);

/* Adds a pillar to a channel's geometry (before sfg_initialize): kind 0 a
 * circle of centre (a, b) and radius c, kind 1 the rectangle spanned by
 * (a, b) and (c, d).  Replaces ChannelBuilder::addCirclePillar /
 * addRectPillar with Simulation::setChannelBuilder (geometry/
 * channel_builder.h:25-33, simulation.cpp:211-213, 430-442): lattice nodes
 * inside a pillar are SOLID (halfway bounce-back, or interpolated with
 * use_interpolated_bb); markers are repelled from the pillars as
 * RepulsionForce::computeObstacleRepulsion does (repulsion.cpp:180-235). */
enum sfg_pillar { SFG_PILLAR_CIRCLE = 0, SFG_PILLAR_RECT = 1 };
int sfg_add_pillar(sfg_context* ctx, int channel, int kind, double a, double b, double c,
                   double d);

/* Capsule chemistry of the scalar, before sfg_initialize (the channel needs
 * the scalar): AdvectionDiffusion::applySourceSink / applyChemistry
 * (advection_diffusion.cpp:225-437) after every scalar step, as
 * Simulation::step calls them (simulation.cpp:640-653).  Vectors are per
 * capsule type (at most SFG_CHEM_TYPES entries); a count of 0 is an empty
 * vector, which selects the reference's branches: Fick leaching from
 * finite reservoirs and Langmuir adsorption with Peskin-weighted exchange
 * when k_leach or k_adsorb is non-empty, else constant release /
 * absorption at the nearest node when either rate vector is non-empty.
 * Capsules are applied in order; capsules whose stencils overlap run one
 * after the other, so results equal the reference's serial loop. */
#define SFG_CHEM_TYPES 8
typedef struct sfg_chemistry {
    int n_release, n_absorb, n_k_leach, n_C_eq, n_M_p, n_k_adsorb, n_k_desorb, n_Gamma_max;
    double release[SFG_CHEM_TYPES], absorb[SFG_CHEM_TYPES], k_leach[SFG_CHEM_TYPES];
    double C_eq[SFG_CHEM_TYPES], M_p_initial[SFG_CHEM_TYPES], k_adsorb[SFG_CHEM_TYPES];
    double k_desorb[SFG_CHEM_TYPES], Gamma_max[SFG_CHEM_TYPES];
} sfg_chemistry;
int sfg_set_chemistry(sfg_context* ctx, int channel, const sfg_chemistry* chem);
/* Type id of a capsule (Capsule::getTypeId), index within its channel,
 * before sfg_initialize; 0 by default. */
int sfg_set_capsule_type(sfg_context* ctx, int channel, int capsule, int type);
/* Chemistry state of a channel: per capsule the cumulative released and
 * absorbed amounts and the reservoir mass (-1: infinite), per marker the
 * surface coverage (AdvectionDiffusion::getCapsuleReleased / Absorbed / Mp,
 * getNodeGamma).  Any pointer may be NULL. */
int sfg_get_chemistry_state(sfg_context* ctx, int channel, double* released, double* absorbed,
                            double* Mp, double* gamma);

/* Allocates device state and sets every channel to equilibrium at rho0 with
 * u = 0 (LBMSolver::initialize, lbm_solver.cpp:130-170; scalar initialised to
 * zero, advection_diffusion.cpp:46-57). */
int sfg_initialize(sfg_context* ctx);

/* Advances every channel by nsteps steps of Simulation::step
 * (simulation.cpp:470-700).  Asynchronous: returns after enqueueing. */
int sfg_step(sfg_context* ctx, int nsteps);

/* Waits for queued work; reports kernel status bits (see softflow docs) and
 * returns SFG_ERR_NUMERIC if a non-finite marker was seen. */
int sfg_synchronize(sfg_context* ctx, unsigned* status_out);

/* ---- state transfer (synchronous) ---------------------------------------- */
int sfg_get_populations(sfg_context* ctx, int channel, double* f);
int sfg_set_populations(sfg_context* ctx, int channel, const double* f);
/* Every channel's populations in one call: f holds the channels' [9][ny][nx]
 * FP64 arrays back to back in channel order (the LatticeField::fData()
 * layout of each, python/bindings.cpp:348-355).  The copies of channel i + 1
 * overlap the device-side import of channel i (two staging buffers, a copy
 * stream); synchronous on return like sfg_set_populations. */
int sfg_set_all_populations(sfg_context* ctx, const double* f);
/* rho, u and the lattice force of the last step (any pointer may be NULL),
 * as LatticeField::computeMacroscopic leaves them (lattice_field.cpp:28-73). */
int sfg_get_macroscopic(sfg_context* ctx, int channel, double* rho, double* ux, double* uy,
                        double* Fx, double* Fy);
int sfg_get_markers(sfg_context* ctx, int channel, double* pos, double* vel, double* force);
int sfg_set_markers(sfg_context* ctx, int channel, const double* pos, const double* vel);
/* Marker positions / velocities of every channel at once (channel-major). */
int sfg_get_all_markers(sfg_context* ctx, double* pos, double* vel);
/* The same copy without waiting, for a host loop that consumes every step's
 * markers while the next steps run: a snapshot after the steps enqueued so
 * far is taken on the context stream and copied to pos / vel (page-locked
 * host memory, [M][2] each, either may be NULL) on a separate copy stream.
 * slot (0 or 1) selects one of two snapshot buffers; the host buffers must
 * stay valid and unread until sfg_wait_markers(slot) returns.  Reusing a
 * slot first waits for its previous copy.  No reference counterpart (the
 * reference's host owns the markers). */
int sfg_get_all_markers_async(sfg_context* ctx, int slot, double* pos, double* vel);
int sfg_wait_markers(sfg_context* ctx, int slot);
/* Concentration field and equilibrium populations g = w C
 * (AdvectionDiffusion::setRegion semantics, advection_diffusion.cpp:59-71). */
int sfg_set_concentration(sfg_context* ctx, int channel, const double* C);
/* Declares, before the first step, that the populations set with
 * sfg_set_populations are a saved state after a step: the first collision
 * then takes the uniform (capped) body force as the previous step's force
 * in u = (j + F/2) / rho, as the reference's restored u includes it
 * (Checkpoint::load restores rho and u, io/checkpoint.cpp:249-255).  The
 * previous step's spread (capsule) force is not part of a saved state and
 * counts as zero there. */
int sfg_mark_restored(sfg_context* ctx);
/* Scalar state restored from a saved state: concentration C [ny][nx] and
 * populations g [9][ny][nx] as they were (Checkpoint::load,
 * io/checkpoint.cpp:312-330). */
int sfg_set_scalar_state(sfg_context* ctx, int channel, const double* C, const double* g);
/* Concentration (and, if g != NULL, the scalar populations [9][ny][nx]). */
int sfg_get_concentration(sfg_context* ctx, int channel, double* C, double* g);
/* Cells whose force was capped in the last step (Simulation::
 * last_capped_nodes_, simulation.cpp:588-609). */
int sfg_get_capped_count(sfg_context* ctx, int channel, int* count);
/* Contact pairs visited per marker in the last step (cell-list bookkeeping). */
int sfg_get_contact_counts(sfg_context* ctx, int channel, int* counts);

/* ---- standalone operators on caller buffers ------------------------------ */
/* Spreads marker forces onto a lattice force field: the operation of
 * ImmersedBoundary::spreadForces (reference immersed_boundary.cpp:25-100)
 * on caller-provided DEVICE buffers, enqueued on `stream` (a cudaStream_t,
 * NULL for the default stream).
 *   nx, ny       lattice size; x is periodic (arc lengths use the minimum image)
 *   ncaps        number of closed marker rings
 *   d_offsets    [ncaps + 1] first marker of each ring, d_offsets[ncaps] = M
 *   d_pos        [M][2] marker positions      d_force  [M][2] marker forces
 *   d_Fx, d_Fy   [ny][nx] lattice force; the spread sum is added (F += sum)
 *   num_markers  M; must equal d_offsets[ncaps] (markers past the last
 *                ring are skipped, never read)
 * Deterministic: each cell sums its contributions in ascending marker order
 * (the reference's serial order) without floating-point atomics.  Scratch
 * memory is taken with cudaMallocAsync on the stream and released on it. */
int sfg_spread_forces(int nx, int ny, int ncaps, const int* d_offsets, const double* d_pos,
                      const double* d_force, double* d_Fx, double* d_Fy, int num_markers,
                      void* stream);

/* The spread of sfg_spread_forces for callers that cannot allocate device
 * memory inside a call (a host engine or framework that owns the device
 * memory budget through its own pool, or a loop that must not stall on
 * cudaMalloc / cudaFree).  No counterpart in the reference, which runs on the
 * CPU.  It allocates nothing: its scratch is a fixed 2 MiB device array held
 * by every GPU that loads the library until the process exits.
 * Limits: num_markers <= 32768 and ceil(nx/32) * ceil(ny/8) <= 32768 force
 * tiles; larger calls return SFG_ERR_CAPACITY.  All calls share the array:
 * calls whose GPU work overlaps (other streams or host threads on the same
 * device) race and must be serialized by the caller.  The first call on each
 * device looks up the array's device address with that device current; make
 * it before any stream capture on that device.  Results equal
 * sfg_spread_forces bit for bit. */
int sfg_spread_forces_noalloc(int nx, int ny, int ncaps, const int* d_offsets,
                              const double* d_pos, const double* d_force, double* d_Fx,
                              double* d_Fy, int num_markers, void* stream);

/* ---- learned multi-direct forcing: the per-marker network ------------------
 * An 8 -> 64 -> 64 -> 2 ReLU network (4866 FP32 parameters: W1 [64x8], b1,
 * W2 [64x64], b2, W3 [2x64], b3) trained and evaluated on the tensor cores
 * with BF16 operands and FP32 accumulation.  The reference's counterpart is
 * the FP64 surrogate SimpleNN (src/ml/simple_nn.cpp:10-262: same layer
 * shapes with 9 inputs, He initialisation, mean/std normalisation, MSE
 * gradient), trained there with SGD on the CPU and not used by its step.
 * Device pointers are given as `d_`; calls are ordered on `stream` and return
 * after it has finished.  Features are raw (the network normalises them);
 * targets are raw (normalised inside). */
typedef struct sfg_mlp sfg_mlp;
#define SFG_MLP_NUM_PARAMS 4866
int sfg_mlp_create(int device, sfg_mlp** out);
int sfg_mlp_destroy(sfg_mlp* m);
/* Sets the FP32 parameters (host array) and resets the Adam state. */
int sfg_mlp_set_params(sfg_mlp* m, const float* params);
int sfg_mlp_get_params(sfg_mlp* m, float* params);
/* Input mean/std [8] and output mean/std [2]; every std must be > 0. */
int sfg_mlp_set_normalization(sfg_mlp* m, const float* in_mean, const float* in_std,
                              const float* out_mean, const float* out_std);
/* d_y [n x 2] = network(d_x [n x 8]), de-normalised. */
int sfg_mlp_forward(sfg_mlp* m, const float* d_x, int n, float* d_y, void* stream);
/* Gradient of the loss mean((y - t)^2) over the n samples and both outputs
 * (normalised targets) into the host array grad [4866]; loss optional. */
int sfg_mlp_gradients(sfg_mlp* m, const float* d_x, const float* d_t, int n, float* grad,
                      float* loss, void* stream);
/* floor(n / batch) Adam steps (beta 0.9 / 0.999, eps 1e-8) over consecutive
 * batches of the given data; losses (host, optional) receives each step's
 * batch loss. */
int sfg_mlp_train(sfg_mlp* m, const float* d_x, const float* d_t, int n, int batch, float lr,
                  float* losses, void* stream);
int sfg_mlp_step_count(sfg_mlp* m, int* steps);

/* Learned multi-direct forcing in the step.  On every channel with
 * ibm_iterations = K >= 3 and capsules, replaces the first K-2 correction
 * sweeps of ImmersedBoundary::multiDirectForcing (immersed_boundary.cpp:
 * 231-286) by the network's prediction of their summed correction (seed),
 * spread like a sweep; the last plain sweep follows.  The no-slip residual
 * max |U_prev - U_interp| over the channel's markers, taken at that sweep's
 * interpolation, gates the result: above residual_threshold (lu/step) the
 * channel redoes the plain K-1 sweeps from its membrane-force spread, so its
 * result is the plain one.  The network's current parameters are copied into
 * the context; net == NULL turns the learned form off.  The reference has no
 * counterpart (it always runs the plain sweeps). */
int sfg_set_mdf_model(sfg_context* ctx, sfg_mlp* net, double residual_threshold);
/* Last step's residuals of a channel (learned gate; plain iteration's last
 * sweep, 0 when it did not run) and cumulative learned / fallback steps. */
int sfg_get_mdf_stats(sfg_context* ctx, int channel, float* resid_learned, float* resid_plain,
                      long long* learned_steps, long long* fallbacks);
/* Training data: when enabled, every step records for each marker the
 * network inputs (with the velocity interpolated at the plain iteration's
 * first sweep) and the label, the correction summed over the sweeps before
 * the last one, in the marker's local frame (learned steps record the
 * seed).  sfg_get_harvest copies the last step's records:
 * features [M][8], labels [M][2], valid [M] (M = all markers of the context,
 * capsule-major).  Any pointer may be NULL. */
int sfg_set_harvest(sfg_context* ctx, int enabled);
int sfg_get_harvest(sfg_context* ctx, float* features, float* labels, int* valid);

/* ---- launch shapes ------------------------------------------------------
 * sfg_autotune times whole steps (CUDA events) for each candidate launch
 * shape -- CTAs per SM of the persistent lattice kernel, of the spread and of
 * the learned seed, and the block size of the per-marker kernels -- one
 * tunable at a time, and keeps the fastest.  The trials are real steps: the
 * context advances by *steps_run steps (call it in place of warm-up steps).
 * No reference counterpart (the reference has no launch shapes). */
int sfg_autotune(sfg_context* ctx, int steps_per_trial, int* steps_run);
int sfg_get_launch_config(sfg_context* ctx, int* lattice_ctas_per_sm, int* spread_ctas_per_sm,
                          int* marker_block, int* learned_ctas_per_sm);

/* ---- thermo: device-side reductions of the state -------------------------
 * One record per channel, reduced on the device over the state after the
 * last step.  Cell sums run in a fixed tree order (run-to-run identical;
 * they differ from the reference's row-major serial sums by rounding only);
 * minima, maxima, counts and the capsule sums are exact. */
typedef struct sfg_thermo_record {
    /* sqrt(max |u|^2) over non-SOLID cells: Simulation::getMaxSpeed
     * (simulation.cpp:892-907), the thermo line's u_max (setup.py:1969) */
    double max_speed;
    /* over non-SOLID cells, as GlobalStatsWriter::writeTimestep
     * (global_stats_writer.cpp:52-81): mean rho, mean |u|, sum 0.5 rho |u|^2,
     * smallest and largest rho */
    double mean_rho, mean_velocity, kinetic_energy, min_rho, max_rho;
    /* sum of the concentration over all cells (0 without the scalar):
     * total_dissolved_mass (global_stats_writer.cpp:92-103) */
    double total_scalar;
    /* Taylor deformation over the channel's capsules, summed in capsule
     * order (global_stats_writer.cpp:84-90); 0 without capsules */
    double mean_deformation, max_deformation;
    long long fluid_cells;      /* non-SOLID cells */
    /* y * nx + x of the first cell in row-major order whose rho or u is not
     * finite (Simulation::checkStability, simulation.cpp:818-845), or -1 */
    long long first_nonfinite;
    long long capped_nodes;     /* as sfg_get_capped_count */
    int num_capsules;
    int reserved;
} sfg_thermo_record;

/* Geometry of one capsule (FP64, the reference's evaluation order):
 * Capsule::centroid, area, perimeter, deformationIndex, inclinationAngle
 * (capsule.cpp:159-266). */
typedef struct sfg_capsule_stats {
    double cx, cy, area, perimeter, deformation, inclination;
} sfg_capsule_stats;

/* Thermo of every channel (chans [num_channels], may be NULL) and the
 * geometry of every capsule (caps [total capsules, channel-major], may be
 * NULL), synchronous.  Runs a pending scalar step first, as every host read
 * of the scalar does. */
int sfg_thermo(sfg_context* ctx, sfg_thermo_record* chans, sfg_capsule_stats* caps);

/* Called by sfg_run after every thermo interval with the records of
 * sfg_thermo; a nonzero return stops the run after that interval. */
typedef int (*sfg_thermo_fn)(long long step, const sfg_thermo_record* chans, int num_channels,
                             const sfg_capsule_stats* caps, int num_capsules, void* user);

/* Runs nsteps steps in one call: the multi-step loop of Simulation::run
 * (simulation.cpp:788-800) and of the Python driver's run loop
 * (setup.py:1957-1969), with the per-interval thermo (max speed, capsule
 * deformation) reduced on the device.  Every thermo_every steps and after
 * the last step (thermo_every <= 0: only after the last step) the records are
 * copied to the host and passed to cb (may be NULL).  *steps_done (may be
 * NULL) receives the steps run, fewer than nsteps when cb stopped the run.
 * Returns after the last interval has finished on the device. */
int sfg_run(sfg_context* ctx, int nsteps, int thermo_every, sfg_thermo_fn cb, void* user,
            int* steps_done);

/* ---- output: VTK files of a channel --------------------------------------
 * Written on the host from the device state of the last step (pulled by the
 * call), with the file names, layout and "%.6e" formatting of the
 * reference's VTKWriter: XML ImageData <dir>/fluid/fluid_%06d.vti and
 * PolyData <dir>/particles/particles_%06d.vtp, or with legacy != 0 the
 * legacy files <dir>/fluid_%06d.vtk and <dir>/particles_%06d.vtk
 * (vtk_writer.cpp:75-209, 230-471, 549-929).  fields selects the fluid
 * arrays (FluidOutputFields, io/output_config.h:10-21); SFG_VTK_DEFAULT is the
 * reference's default set. */
enum sfg_vtk_field {
    SFG_VTK_DENSITY = 1, SFG_VTK_VELOCITY = 2, SFG_VTK_VELOCITY_MAG = 4,
    SFG_VTK_PRESSURE = 8, SFG_VTK_VORTICITY = 16, SFG_VTK_STRAIN_RATE = 32,
    SFG_VTK_IBM_FORCE = 64, SFG_VTK_NODE_TYPE = 128, SFG_VTK_CONCENTRATION = 256,
    SFG_VTK_DEFAULT = 1 | 2 | 4 | 8 | 128 | 256
};
int sfg_write_vtk_fluid(sfg_context* ctx, int channel, const char* output_dir, int step,
                        int legacy, unsigned fields);
/* Capsule polygons split at the periodic seam as the reference does;
 * type_ids [capsules of the channel] (may be NULL: type 0). */
int sfg_write_vtk_capsules(sfg_context* ctx, int channel, const char* output_dir, int step,
                           int legacy, const int* type_ids);

/* ---- diagnostics ---------------------------------------------------------- */
/* The parameters a channel was added with. */
int sfg_get_channel_params(const sfg_context* ctx, int channel, sfg_channel_params* out);
/* Nodes of each capsule of a channel (nodes [capsules of the channel]). */
int sfg_get_capsule_nodes(const sfg_context* ctx, int channel, int* nodes);
/* Index of the channel's first capsule in the context-wide capsule order. */
int sfg_get_capsule_base(const sfg_context* ctx, int channel, int* first_capsule);
int sfg_num_channels(const sfg_context* ctx, int* n);
int sfg_channel_counts(const sfg_context* ctx, int channel, int* num_capsules, int* num_markers);
int sfg_step_count(const sfg_context* ctx, long long* steps);
/* Kernel launches issued per step (for launch accounting). */
int sfg_launches_per_step(const sfg_context* ctx, int* launches);
/* Host-visible timing of the last sfg_step call in milliseconds, measured
 * with CUDA events on the context stream (valid after sfg_synchronize). */
int sfg_last_step_ms(sfg_context* ctx, float* ms);
/* Per-phase timing, the counterpart of the reference's per-module Profiler
 * timers (simulation.cpp:194-208, io/profiler.h:12-90).  With profiling on,
 * sfg_step runs each step eagerly and accumulates CUDA-event times per
 * phase (milliseconds, indexed by sfg_phase). */
enum sfg_phase {
    SFG_PHASE_MEMBRANE = 0,     /* "Membrane forces"                          */
    SFG_PHASE_CONTACT = 1,      /* "Repulsion forces" (cell list + contact)   */
    SFG_PHASE_IBM_TILES = 2,    /* force-tile occupancy and marker lists      */
    SFG_PHASE_IBM_SPREAD = 3,   /* "IBM spread" (all MDF sweeps)              */
    SFG_PHASE_MDF_INTERP = 4,   /* MDF interpolation sweeps                   */
    SFG_PHASE_LATTICE = 5,      /* "LBM step" (+ fused scalar step)           */
    SFG_PHASE_BOOKKEEPING = 6,  /* per-step flags                             */
    SFG_PHASE_INTERP_MOVE = 7,  /* "IBM interpolate" + marker move            */
    SFG_PHASE_MDF_LEARNED = 8,  /* learned forcing: interpolation + network   */
    SFG_NUM_PHASES = 9
};
int sfg_set_profiling(sfg_context* ctx, int on);
int sfg_get_phase_times(sfg_context* ctx, float* ms, int n);
int sfg_reset_phase_times(sfg_context* ctx);
/* Lattice kernel variant, before sfg_initialize: 0 (default) = the widest
 * vectorised form the channels allow (eight cells per lane in FP16-shifted
 * storage without the scalar when every nx % 8 == 0, otherwise four cells
 * per lane when every nx % 4 == 0), 1 = one cell per thread, 2 = four cells
 * per lane, 3 = as 0 with the eight-cell kernel's cells in force tiles
 * untouched by the step's markers stepped beside the forcing on a side
 * stream.  FP64 and FP32 results are identical across variants; FP16-shifted
 * results of the four- and eight-cell forms differ only in the stochastic
 * rounding's random bits (variants 0 and 3 are identical).  The choice
 * exists for measurements. */
int sfg_set_lattice_variant(sfg_context* ctx, int variant);
/* CUDA stream of the context (cudaStream_t), for callers that interleave
 * their own work. */
int sfg_get_stream(const sfg_context* ctx, void** stream);

#ifdef __cplusplus
}
#endif
#endif /* SOFTFLOW_GPU_H */
