// sfg_internal.h -- device buffer bundles and launch wrappers shared by the
// translation units of libsoftflow_b200.so (not part of the C ABI).
#pragma once
#include "../../include/softflow_gpu.h"
#include "common.cuh"
#include "markers.cuh"

namespace sfg {

struct ContactBufs {
    int* cell_of = nullptr;     // [M] global contact cell of each marker
    int* cell_cnt = nullptr;    // [ncells]
    int* cell_start = nullptr;  // [ncells]
    int* cursor = nullptr;      // [ncells]
    int* list = nullptr;        // [M]
    int* scan_tmp = nullptr;
};

// Per-slot record of the step's force tiles (written by k_tile_slots).
struct SlotInfo {
    int tile, chan, x0, y0, cnt, off, nx, ny;
};

struct TileBufs {
    int T = 0;                  // force tiles over all channels
    int max_slots = 0;
    int* tile_chan = nullptr;   // [T]
    int* tile_flag = nullptr;   // [T]
    int* tile_cnt = nullptr;    // [T] markers whose stencil covers the tile
    int* cursor = nullptr;      // [T]
    int* slot_scan = nullptr;   // [T]
    int* list_off = nullptr;    // [T]
    int* tile_slot[2] = {nullptr, nullptr};  // [T] per step parity
    int* slot_tile = nullptr;   // [max_slots]
    int* n_slots = nullptr;     // [1]
    int* list = nullptr;        // [8 M]
    int* scan_tmp = nullptr;
    double* acc = nullptr;      // [max_slots][TILE_CELLS][2]: (x, y) per cell
    void* gsnap = nullptr;      // [max_slots][2][TILE_CELLS] (R)
    void* fin[2] = {nullptr, nullptr};
    int* capped = nullptr;      // [nchan]
    int* fluid_touched = nullptr;
    double* acc0 = nullptr;     // [max_slots][TILE_CELLS][2] force after the membrane spread
    void* mom = nullptr;        // [max_slots][TILE_CELLS] (rho, jx, jy, 0) of R (step's moments)
    int marker_block = 128;         // block size of the per-marker kernels (tuned)
    SlotInfo* slot_info = nullptr;  // [max_slots]
    // The order in which the spread warps take the slots: by descending
    // class of list length (passes of 8 markers), so that each warp's share
    // of the step's tiles sums to about the same work.
    int* slot_order = nullptr;      // [max_slots]
    int* slot_rank = nullptr;       // [max_slots] rank of the slot within its class
    int* cls_cnt = nullptr;         // [SLOT_CLASSES] slots per class
    int* spread_ctr = nullptr;      // [n_spread_ctr] slot counters, one per spread launch of a
                                    // step (zeroed at the start of the step)
    int n_spread_ctr = 0;
    int* plain_needed = nullptr;  // [1] set when some channel needs the plain sweeps; null
                                  // (always run them) unless a channel is learned
    unsigned* resid_gate = nullptr;   // [nchan] learned form's no-slip residual (float bits)
    unsigned* resid_plain = nullptr;  // [nchan] plain iteration's last-sweep residual
};

// Exclusive prefix sum of n ints (three kernels, graph-capturable);
// `total` (device int, may be null) receives the sum.
void scan_exclusive(const int* in, int* out, int n, int* tmp, int* total, cudaStream_t st);
size_t scan_tmp_ints(int n);

// Capsules of up to maxn nodes; > 48 KB of shared memory needs opting in.
size_t membrane_smem_bytes(int maxn);
cudaError_t prepare_membrane(int maxn);
// Opts the spread kernels into their shared-memory size (once per device).
cudaError_t prepare_spread();
// Resident spread CTAs per SM (after prepare_spread).
int spread_blocks_per_sm(bool fp64);
void launch_membrane(const CapsuleDev* caps, int ncaps, const MarkerBufs& mb, int* has_prev,
                     int maxn, unsigned* status, cudaStream_t st);
void launch_contact(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                    int ncells, cudaStream_t st);
// The cell list (binning, scan, fill, sort: positions only) and the pair
// forces (added to the membrane forces) as separate launch groups.
void launch_contact_prep(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                         int ncells, cudaStream_t st);
void launch_contact_force(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                          cudaStream_t st);
// Repulsion of markers from the pillars of their channel (after the pairs).
void launch_obstacle_repulsion(const ChannelDev* chans, int M, const MarkerBufs& mb,
                               cudaStream_t st);
// `slots_ready` (may be null) is recorded once the slot records exist (the
// tile moments need no more).
void launch_tiles(const ChannelDev* chans, const CapsuleDev* caps, int M, const MarkerBufs& mb,
                  TileBufs& tb, int T, int parity, const double* phi_tbl, unsigned* status,
                  cudaStream_t st, cudaEvent_t slots_ready = nullptr);
// Spread of sweep `sweep` in forcing mode `mode` (MdfMode); sweep 0 spreads
// the membrane and contact forces of every channel.  launch_idx: the
// launch's slot counter in tb.spread_ctr (distinct per launch of a step).
template <typename R>
void launch_spread(const ChannelDev* chans, const MarkerBufs& mb, TileBufs& tb, int parity,
                   int sweep, int mode, int launch_idx, int grid, unsigned* status,
                   cudaStream_t st);
template <typename S, typename R>
void launch_mdf_interp(const ChannelDev* chans, int M, const MarkerBufs& mb, const S* f,
                       TileBufs& tb, int parity, int sweep, int mode, cudaStream_t st);
// Learned forcing: interpolation after the membrane spread and network
// inputs (feat [M][8], frame [M]), then tensor-core inference and rotation
// back to the lattice frame -> dF, dFsum, u0 of every marker of a learned
// channel.  `model` is a mlp::ModelDev.
template <typename S, typename R>
void launch_mdf_learned(const ChannelDev* chans, const CapsuleDev* caps, int M,
                        const MarkerBufs& mb, const S* f, TileBufs& tb, int parity,
                        const void* model, float* feat, double2* frame, int grid,
                        unsigned* status, cudaStream_t st);
// Training data of the step: inputs [M x 8], labels [M x 2] (the step's total
// correction in the local frame), valid [M].
void launch_harvest(const ChannelDev* chans, const CapsuleDev* caps, int M, const MarkerBufs& mb,
                    float* feat, float* label, int* valid, cudaStream_t st);
cudaError_t prepare_mdf_learned();
// Sets tb.plain_needed from the gate residuals (learned contexts).
void launch_plain_needed(const ChannelDev* chans, int nch, TileBufs& tb, cudaStream_t st);
// Moments of the step's force tiles (before the first forcing sweep).
template <typename S, typename R>
void launch_tile_moments(const ChannelDev* chans, const S* f, TileBufs& tb, int grid,
                         cudaStream_t st);
template <typename S, typename R>
void launch_interp_move(const ChannelDev* chans, const CapsuleDev* caps, int ncaps, int M,
                        const MarkerBufs& mb, const S* f, TileBufs& tb, int parity,
                        const double* phi_tbl, cudaStream_t st);

// Lattice kernels (lattice_f64.cu / lattice_f32.cu).
struct LatticeLaunch {
    const RowItem* items;
    int n_items;
    const ChannelDev* chans;
    const void* src;
    void* dst;
    const void* gsrc;
    void* gdst;
    const void* cfield;
    const int* stepped;
    const int* adr_pending;
    const int* c_fresh;
    const unsigned* step_ctr;   // device step counter (stochastic-rounding seed)
    bool any_adr;
    const RowItem* items4;      // 128-cell runs for the vectorised kernel
    int n_items4;
    bool use_vec4;              // every channel has nx % 4 == 0
    int persistent_ctas;        // grid of the persistent vectorised kernel
    int collision;              // shared collision model of all channels, -1 if mixed
    bool any_bc = false;        // some channel has Zou-He / closed columns or moving walls
    const RowItem* zh_rows = nullptr;  // (channel, y) rows of the Zou-He columns
    int n_zh = 0;
    const IbbLink* ibb = nullptr;      // interpolated bounce-back links, by level
    const int* ibb_level_start = nullptr;  // host array [n_ibb_levels + 1]
    int n_ibb_levels = 0;
    const RowItem* items8 = nullptr;   // 256-cell runs for the 8-cell FP16-shifted kernel
    int n_items8 = 0;
    bool use_vec8 = false;             // FP16-shifted storage, every channel nx % 8 == 0
    int pass = 0;                      // 8-cell kernel: 0 all cells, 1 cells of untouched
                                       // force tiles, 2 cells of touched ones
    int n_chans = 0;                   // channel count (run records are checked against it)
    unsigned* status = nullptr;        // status word (ST_* bits)
};
struct TileViewArgs {
    const int* cur_slot;
    const int* prev_slot;
    const void* cur_fin;
    const void* cur_G;
    const void* prev_fin;
};
// Resident CTAs per SM of the persistent lattice kernel (occupancy query).
int lattice_ctas_per_sm(int precision, bool adr, bool vec8);
template <typename S, typename R>
int lattice_ctas_per_sm_t(bool adr, bool vec8);
template <typename S, typename R>
void launch_lattice_step(const LatticeLaunch& L, const TileViewArgs& tv, cudaStream_t st);
template <typename S, typename R>
void launch_scalar_flush(const LatticeLaunch& L, const TileViewArgs& tv_last, cudaStream_t st);
// Scalar step of the current step on its streamed populations (L.dst) and
// forces (contexts with capsule chemistry).
template <typename S, typename R>
void launch_scalar_now(const LatticeLaunch& L, const TileViewArgs& tv, unsigned char* cov,
                       cudaStream_t st);
// Capsule chemistry of every channel that has it (chemistry.cu).
size_t chem_box_bytes();
template <typename R>
void launch_chemistry(const ChannelDev* chans, int nch, const sfg_chemistry* params,
                      const CapsuleDev* caps, const double2* pos, const double* phi, void* g_new,
                      void* g_old, void* cfield, unsigned char* cov, double* released,
                      double* absorbed, double* Mp, double* gamma, int* wave_buf,
                      void* box_buf, int box_cap, unsigned* status, cudaStream_t st);
template <typename S, typename R>
void launch_pop_import(const double* in, void* out, const ChannelDev& ch, cudaStream_t st);
template <typename S, typename R>
void launch_pop_export(const void* in, double* out, const ChannelDev& ch, cudaStream_t st);
template <typename S, typename R>
void launch_macro_export(const void* in, const ChannelDev& ch, const TileViewArgs& tv_last,
                         int stepped, double* rho, double* ux, double* uy, double* Fx, double* Fy,
                         cudaStream_t st);
// Per-block partial thermo sums of every channel (parts [nch][blocks_per_chan]).
template <typename S, typename R>
void launch_thermo_cells(const void* in, const void* g, const ChannelDev* chans, int nch,
                         int blocks_per_chan, const TileViewArgs& tv_last, int stepped,
                         ThermoPart* parts, const void* cfield, const unsigned char* cov,
                         cudaStream_t st);
// Geometry of every capsule: out [ncaps][6] = centroid x, y, area, perimeter,
// deformation, inclination.
void launch_capsule_stats(const CapsuleDev* caps, int ncaps, const double2* pos, double* out,
                          cudaStream_t st);

}  // namespace sfg
