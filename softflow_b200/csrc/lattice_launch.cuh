// lattice_launch.cuh -- host launch wrappers of the lattice kernels; included
// by lattice_f64.cu (FP64, no FMA contraction) and lattice_f32.cu (FP32 and
// FP16-shifted storage).
#pragma once
#include <algorithm>

#include "lattice.cuh"
#include "sfg_internal.h"

namespace sfg {

inline TileView to_view(const TileViewArgs& a) {
    TileView v;
    v.cur_slot = a.cur_slot;
    v.prev_slot = a.prev_slot;
    v.cur_fin = a.cur_fin;
    v.cur_G = a.cur_G;
    v.prev_fin = a.prev_fin;
    return v;
}

template <typename S, typename R, bool ADR, int COLL>
static void launch_step4(const LatticeLaunch& L, const TileViewArgs& tv, int grid,
                         cudaStream_t st) {
    k_lattice_step4<S, R, ADR, COLL><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
        L.items4, L.n_items4, L.chans, static_cast<const S*>(L.src), static_cast<S*>(L.dst),
        static_cast<const R*>(L.gsrc), static_cast<R*>(L.gdst), static_cast<const R*>(L.cfield),
        to_view(tv), L.stepped, L.adr_pending, L.c_fresh, L.step_ctr);
}

template <typename S, typename R, bool ADR>
static void launch_step4_coll(const LatticeLaunch& L, const TileViewArgs& tv, int grid,
                              cudaStream_t st) {
    switch (L.collision) {
        case 0: launch_step4<S, R, ADR, 0>(L, tv, grid, st); break;
        case 1: launch_step4<S, R, ADR, 1>(L, tv, grid, st); break;
        case 2: launch_step4<S, R, ADR, 2>(L, tv, grid, st); break;
        default: launch_step4<S, R, ADR, -1>(L, tv, grid, st); break;
    }
}

template <typename S, typename R>
void launch_lattice_step(const LatticeLaunch& L, const TileViewArgs& tv, cudaStream_t st) {
    if (L.any_bc) {
        // boundary-aware kernel (no scalar transport in such contexts), then
        // the Zou-He columns on the streamed populations
        if (L.n_items == 0) return;
        k_lattice_step_bc<S, R><<<(L.n_items + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA,
                                  32 * ITEMS_PER_CTA, 0, st>>>(
            L.items, L.n_items, L.chans, static_cast<const S*>(L.src), static_cast<S*>(L.dst),
            to_view(tv), L.stepped, L.step_ctr);
        for (int lv = 0; lv < L.n_ibb_levels; ++lv) {
            const int a = L.ibb_level_start[lv], n = L.ibb_level_start[lv + 1] - a;
            if (n > 0)
                k_ibb<S, R><<<(n + 127) / 128, 128, 0, st>>>(L.ibb + a, n, L.chans,
                                                             static_cast<S*>(L.dst),
                                                             L.step_ctr);
        }
        if (L.n_zh > 0)
            k_zou_he<S, R><<<(L.n_zh + 127) / 128, 128, 0, st>>>(L.zh_rows, L.n_zh, L.chans,
                                                                 static_cast<S*>(L.dst),
                                                                 L.step_ctr);
        return;
    }
    if constexpr (std::is_same<S, __half>::value && std::is_same<R, float>::value) {
        if (L.use_vec8 && !L.any_adr) {
            if (L.n_items8 == 0) return;
            const int grid = std::max(1, std::min(L.persistent_ctas,
                                                  (L.n_items8 + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA));
            const TileView v = to_view(tv);
            const __half* src = static_cast<const __half*>(L.src);
            __half* dst = static_cast<__half*>(L.dst);
            switch (L.collision) {
                case 0: k_lattice_step8h<0><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
                            L.items8, L.n_items8, L.chans, L.n_chans, src, dst, v, L.stepped, L.step_ctr, L.pass, L.status);
                        break;
                case 1: k_lattice_step8h<1><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
                            L.items8, L.n_items8, L.chans, L.n_chans, src, dst, v, L.stepped, L.step_ctr, L.pass, L.status);
                        break;
                case 2: k_lattice_step8h<2><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
                            L.items8, L.n_items8, L.chans, L.n_chans, src, dst, v, L.stepped, L.step_ctr, L.pass, L.status);
                        break;
                default: k_lattice_step8h<-1><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
                             L.items8, L.n_items8, L.chans, L.n_chans, src, dst, v, L.stepped, L.step_ctr, L.pass, L.status);
                         break;
            }
            return;
        }
    }
    if (L.use_vec4) {
        if (L.n_items4 == 0) return;
        const int grid = std::max(1, std::min(L.persistent_ctas,
                                              (L.n_items4 + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA));
        if (L.any_adr) launch_step4_coll<S, R, true>(L, tv, grid, st);
        else launch_step4_coll<S, R, false>(L, tv, grid, st);
        return;
    }
    if (L.n_items == 0) return;
    const int grid = (L.n_items + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA;
    if (L.any_adr)
        k_lattice_step<S, R, true><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
            L.items, L.n_items, L.chans, static_cast<const S*>(L.src), static_cast<S*>(L.dst),
            static_cast<const R*>(L.gsrc), static_cast<R*>(L.gdst),
            static_cast<const R*>(L.cfield), to_view(tv), L.stepped, L.adr_pending, L.c_fresh,
            L.step_ctr);
    else
        k_lattice_step<S, R, false><<<grid, 32 * ITEMS_PER_CTA, 0, st>>>(
            L.items, L.n_items, L.chans, static_cast<const S*>(L.src), static_cast<S*>(L.dst),
            nullptr, nullptr, nullptr, to_view(tv), L.stepped, L.adr_pending, L.c_fresh,
            L.step_ctr);
}

template <typename S, typename R>
void launch_scalar_now(const LatticeLaunch& L, const TileViewArgs& tv, unsigned char* cov,
                       cudaStream_t st) {
    if (L.n_items == 0) return;
    k_scalar_now<S, R><<<(L.n_items + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA, 32 * ITEMS_PER_CTA, 0,
                         st>>>(L.items, L.n_items, L.chans, static_cast<const S*>(L.dst),
                               static_cast<const R*>(L.gsrc), static_cast<R*>(L.gdst),
                               static_cast<const R*>(L.cfield), cov, to_view(tv), L.c_fresh);
}

template <typename S, typename R>
void launch_scalar_flush(const LatticeLaunch& L, const TileViewArgs& tv_last, cudaStream_t st) {
    if (L.n_items == 0 || !L.any_adr) return;
    k_scalar_flush<S, R><<<(L.n_items + ITEMS_PER_CTA - 1) / ITEMS_PER_CTA,
                           32 * ITEMS_PER_CTA, 0, st>>>(
        L.items, L.n_items, L.chans, static_cast<const S*>(L.src), static_cast<const R*>(L.gsrc),
        static_cast<R*>(L.gdst), static_cast<const R*>(L.cfield), to_view(tv_last),
        L.adr_pending, L.c_fresh);
}

inline int io_grid(long long n) {
    long long g = (n + 255) / 256;
    return (int)(g > 4096 ? 4096 : (g < 1 ? 1 : g));
}

template <typename S, typename R>
void launch_pop_import(const double* in, void* out, const ChannelDev& ch, cudaStream_t st) {
    k_pop_import<S, R><<<io_grid(9LL * ch.nx * ch.ny), 256, 0, st>>>(in, static_cast<S*>(out), ch);
}

template <typename S, typename R>
void launch_pop_export(const void* in, double* out, const ChannelDev& ch, cudaStream_t st) {
    k_pop_export<S><<<io_grid(9LL * ch.nx * ch.ny), 256, 0, st>>>(static_cast<const S*>(in), out,
                                                                  ch);
}

template <typename S, typename R>
void launch_macro_export(const void* in, const ChannelDev& ch, const TileViewArgs& tv_last,
                         int stepped, double* rho, double* ux, double* uy, double* Fx, double* Fy,
                         cudaStream_t st) {
    k_macro_export<S, R><<<io_grid((long long)ch.nx * ch.ny), 256, 0, st>>>(
        static_cast<const S*>(in), ch, to_view(tv_last), stepped, rho, ux, uy, Fx, Fy);
}

template <typename S, typename R>
void launch_thermo_cells(const void* in, const void* g, const ChannelDev* chans, int nch,
                         int blocks_per_chan, const TileViewArgs& tv_last, int stepped,
                         ThermoPart* parts, const void* cfield, const unsigned char* cov,
                         cudaStream_t st) {
    k_thermo_cells<S, R><<<dim3(blocks_per_chan, nch), THERMO_THREADS, 0, st>>>(
        static_cast<const S*>(in), static_cast<const R*>(g), chans, to_view(tv_last), stepped,
        parts, static_cast<const R*>(cfield), cov);
}

template <typename S, typename R>
int lattice_ctas_per_sm_t(bool adr, bool vec8) {
    // the generic-collision instance has the largest footprint
    int n = 0;
    if constexpr (std::is_same<S, __half>::value && std::is_same<R, float>::value) {
        if (vec8 && !adr) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lattice_step8h<-1>,
                                                          32 * ITEMS_PER_CTA, 0);
            return n > 0 ? n : 1;
        }
    }
    if (adr)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lattice_step4<S, R, true, -1>,
                                                      32 * ITEMS_PER_CTA, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lattice_step4<S, R, false, -1>,
                                                      32 * ITEMS_PER_CTA, 0);
    return n > 0 ? n : 1;
}

#define SFG_LATTICE_INST(S, R)                                                                   \
    template int lattice_ctas_per_sm_t<S, R>(bool, bool);                                            \
    template void launch_lattice_step<S, R>(const LatticeLaunch&, const TileViewArgs&,           \
                                            cudaStream_t);                                        \
    template void launch_scalar_flush<S, R>(const LatticeLaunch&, const TileViewArgs&,           \
                                            cudaStream_t);                                        \
    template void launch_scalar_now<S, R>(const LatticeLaunch&, const TileViewArgs&,             \
                                          unsigned char*, cudaStream_t);                          \
    template void launch_pop_import<S, R>(const double*, void*, const ChannelDev&, cudaStream_t); \
    template void launch_pop_export<S, R>(const void*, double*, const ChannelDev&, cudaStream_t); \
    template void launch_macro_export<S, R>(const void*, const ChannelDev&, const TileViewArgs&,  \
                                            int, double*, double*, double*, double*, double*,     \
                                            cudaStream_t);                                        \
    template void launch_thermo_cells<S, R>(const void*, const void*, const ChannelDev*, int, int, \
                                            const TileViewArgs&, int, ThermoPart*, const void*,   \
                                            const unsigned char*, cudaStream_t);

}  // namespace sfg
