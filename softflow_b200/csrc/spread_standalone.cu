// spread_standalone.cu -- sfg_spread_forces: ImmersedBoundary::spreadForces
// (reference immersed_boundary.cpp:25-100) on caller-provided device buffers.
//
// Deterministic gather without floating-point atomics: markers are binned by
// the 32 x 8 force tiles their 4 x 4 stencil covers; one warp per tile sorts
// the tile's marker list and applies the markers in ascending order, so every
// cell sums its contributions in the reference's serial order.  The sum is
// added to the caller's field as the reference's OpenMP reduction does
// (F += sum, immersed_boundary.cpp:70-79).  Built with --fmad=false.
#include <climits>
#include <string>
#include <algorithm>
#include <cmath>

#include "../../include/softflow_gpu.h"
#include "markers.cuh"
#include "sfg_internal.h"
#include "spread_standalone.cuh"

namespace sfg_host {
void set_error(const std::string& msg);
}

namespace sfg {

__device__ __forceinline__ int ring_of(const int* __restrict__ off, int ncaps, int m) {
    int lo = 0, hi = ncaps - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= m) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int sa_tiles(int nx, int ny, int tiles_x, int ix0, int iy0, int out[8]) {
    int tys[2], nty = 0;
    for (int iy = iy0 - 1; iy <= iy0 + 2; ++iy) {
        if (iy < 0 || iy >= ny) continue;
        const int ty = iy / TILE_H;
        if (nty == 0 || tys[nty - 1] != ty) tys[nty++] = ty;
    }
    int txs[4], ntx = 0;
    for (int ix = ix0 - 1; ix <= ix0 + 2; ++ix) {
        int jx = ix;
        if (jx < 0) jx += nx;
        if (jx >= nx) jx -= nx;
        if (jx < 0 || jx >= nx) continue;
        const int tx = jx / TILE_W;
        bool dup = false;
        for (int a = 0; a < ntx; ++a) dup |= (txs[a] == tx);
        if (!dup) txs[ntx++] = tx;
    }
    int n = 0;
    for (int a = 0; a < nty; ++a)
        for (int b = 0; b < ntx; ++b) out[n++] = tys[a] * tiles_x + txs[b];
    return n;
}

// Arc length (min image, Lx = nx), stencil origin and tile counts.
__global__ void k_sa_prep(int nx, int ny, int tiles_x, int ncaps, const int* __restrict__ off,
                          const double2* __restrict__ pos, const double2* __restrict__ frc, int M,
                          SpreadScratch sc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    // num_markers must equal off[ncaps]; a marker beyond the rings (a larger
    // count) is skipped instead of reading past the caller's arrays
    if (m >= off[ncaps]) {
        sc.ds[m] = 0.0;
        sc.ix0[m] = INT_MIN;
        sc.iy0[m] = 0;
        return;
    }
    const int c = ring_of(off, ncaps, m);
    const int o = off[c], n = off[c + 1] - o, k = m - o;
    const double Lx = (double)nx;
    const double2 p = pos[m];
    const double dp = norm_d(min_image_d(p, pos[o + (k - 1 + n) % n], Lx));
    const double dn = norm_d(min_image_d(pos[o + (k + 1) % n], p, Lx));
    sc.ds[m] = 0.5 * (dp + dn);
    int ix0 = INT_MIN, iy0 = 0;
    const double2 f = frc[m];
    // NaN / Inf guards of immersed_boundary.cpp:248-252 and the stencil row
    // test of :257-258; markers beyond one period outside are skipped
    if (finite2(p) && !(isnan(f.x) || isnan(f.y)) && p.x >= -Lx + 2.0 && p.x < 2.0 * Lx - 3.0 &&
        fabs(p.y) < 1e9) {
        const int a = (int)floor(p.x), b = (int)floor(p.y);
        if (!(b < -2 || b >= ny + 2)) {
            ix0 = a;
            iy0 = b;
        }
    }
    sc.ix0[m] = ix0;
    sc.iy0[m] = iy0;
    if (ix0 == INT_MIN) return;
    int t[8];
    const int nt = sa_tiles(nx, ny, tiles_x, ix0, iy0, t);
    for (int i = 0; i < nt; ++i) atomicAdd(&sc.tile_cnt[t[i]], 1);
}

// Clears the per-tile counters and writes the Peskin table
// (delta_function.h:29-37: phi on 1025 points of [0, 2]) into the scratch.
// Every operation is exact in double except the square root, which is
// correctly rounded on the device as in the host library, and the unit is
// built without contraction, so the table equals the host-built one of the
// simulation contexts bit for bit.
__global__ void k_sa_init(int T, SpreadScratch sc) {
    const int n = T > 1025 ? T : 1025;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < T) {
            sc.tile_cnt[i] = 0;
            sc.cursor[i] = 0;
        }
        if (i <= 1024) {
            const double ar = 2.0 * static_cast<double>(i) / 1024;
            double v = 0.0;
            if (ar <= 1.0) v = 0.125 * (3.0 - 2.0 * ar + sqrt(1.0 + 4.0 * ar - 4.0 * ar * ar));
            else v = 0.125 * (5.0 - 2.0 * ar - sqrt(-7.0 + 12.0 * ar - 4.0 * ar * ar));
            sc.phi[i] = v;
        }
    }
}

__global__ void k_sa_fill(int nx, int ny, int tiles_x, int M, SpreadScratch sc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M || sc.ix0[m] == INT_MIN) return;
    int t[8];
    const int nt = sa_tiles(nx, ny, tiles_x, sc.ix0[m], sc.iy0[m], t);
    for (int i = 0; i < nt; ++i)
        sc.list[sc.tile_off[t[i]] + atomicAdd(&sc.cursor[t[i]], 1)] = m;
}

constexpr int SA_WARPS = 8;
constexpr int SA_LCAP = 256;  // a power of two: the bitonic sort pads to one

__global__ void __launch_bounds__(SA_WARPS * 32)
k_sa_gather(int nx, int ny, int tiles_x, int T, const double2* __restrict__ pos,
            const double2* __restrict__ frc, const double* __restrict__ phi_tbl,
            SpreadScratch sc, double* __restrict__ Fx, double* __restrict__ Fy) {
    __shared__ double s_acc[SA_WARPS][2][TILE_CELLS];
    __shared__ int s_list[SA_WARPS][SA_LCAP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* ax = s_acc[warp][0];
    double* ay = s_acc[warp][1];
    int* sl = s_list[warp];
    const int sx = lane & 3, sy = (lane >> 2) & 3;
    for (int t = blockIdx.x * SA_WARPS + warp; t < T; t += gridDim.x * SA_WARPS) {
        int cnt = sc.tile_cnt[t];
        if (cnt == 0) continue;
        const int off = sc.tile_off[t];
        const int x0 = (t % tiles_x) * TILE_W, y0 = (t / tiles_x) * TILE_H;
        const int* lst;
        if (cnt <= SA_LCAP) {
            int pow2 = 1;
            while (pow2 < cnt) pow2 <<= 1;
            for (int i = lane; i < pow2; i += 32) sl[i] = i < cnt ? sc.list[off + i] : INT_MAX;
            __syncwarp();
            for (int k = 2; k <= pow2; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < pow2; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int a = sl[i], b = sl[l];
                            if ((a > b) == ((i & k) == 0)) { sl[i] = b; sl[l] = a; }
                        }
                    }
                    __syncwarp();
                }
            lst = sl;
        } else {
            if (lane == 0) {
                int* a = sc.list + off;
                for (int i = 1; i < cnt; ++i) {
                    const int v = a[i];
                    int j = i - 1;
                    while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
                    a[j + 1] = v;
                }
            }
            __syncwarp();
            lst = sc.list + off;
        }
        for (int c = lane; c < TILE_CELLS; c += 32) {
            ax[c] = 0.0;
            ay[c] = 0.0;
        }
        __syncwarp();
        for (int i = 0; i < cnt; ++i) {
            const int m = lst[i];
            if (lane < 16) {
                const int ix = sc.ix0[m] - 1 + sx, iy = sc.iy0[m] - 1 + sy;
                int jx = ix;
                if (jx < 0) jx += nx;
                if (jx >= nx) jx -= nx;
                const int cxl = jx - x0, cyl = iy - y0;
                if (iy >= 0 && iy < ny && cxl >= 0 && cxl < TILE_W && cyl >= 0 && cyl < TILE_H) {
                    const double2 p = pos[m];
                    const double w = phi_lut(phi_tbl, p.x - (double)ix) *
                                     phi_lut(phi_tbl, p.y - (double)iy);
                    if (w > 1e-15) {
                        const double2 f = frc[m];
                        const double ds = sc.ds[m];
                        const int c = cyl * TILE_W + cxl;
                        ax[c] += f.x * w * ds;
                        ay[c] += f.y * w * ds;
                    }
                }
            }
            __syncwarp();
        }
        for (int c = lane; c < TILE_CELLS; c += 32) {
            const int jx = x0 + (c % TILE_W), jy = y0 + (c / TILE_W);
            if (jx < nx && jy < ny) {
                const size_t n = (size_t)jy * nx + jx;
                Fx[n] = Fx[n] + ax[c];
                Fy[n] = Fy[n] + ay[c];
            }
        }
        __syncwarp();
    }
}

size_t spread_scratch_bytes(int M, int T) {
    const size_t a = 256;
    auto up = [a](size_t b) { return (b + a - 1) / a * a; };
    return up(sizeof(double) * M) + 2 * up(sizeof(int) * M) + up(sizeof(int) * 8 * (size_t)M) +
           3 * up(sizeof(int) * T) + up(sizeof(int) * scan_tmp_ints(T)) + up(sizeof(double) * 1025);
}

SpreadScratch carve_spread_scratch(void* base, int M, int T) {
    const size_t a = 256;
    auto up = [a](size_t b) { return (b + a - 1) / a * a; };
    char* p = static_cast<char*>(base);
    SpreadScratch sc;
    sc.ds = reinterpret_cast<double*>(p);         p += up(sizeof(double) * M);
    sc.ix0 = reinterpret_cast<int*>(p);           p += up(sizeof(int) * M);
    sc.iy0 = reinterpret_cast<int*>(p);           p += up(sizeof(int) * M);
    sc.list = reinterpret_cast<int*>(p);          p += up(sizeof(int) * 8 * (size_t)M);
    sc.tile_cnt = reinterpret_cast<int*>(p);      p += up(sizeof(int) * T);
    sc.tile_off = reinterpret_cast<int*>(p);      p += up(sizeof(int) * T);
    sc.cursor = reinterpret_cast<int*>(p);        p += up(sizeof(int) * T);
    sc.scan_tmp = reinterpret_cast<int*>(p);      p += up(sizeof(int) * scan_tmp_ints(T));
    sc.phi = reinterpret_cast<double*>(p);
    return sc;
}

// Enqueues the whole spread on `st` with the scratch in `sc`.  Everything the
// scratch must start with (zero counters, the Peskin table) is written by
// k_sa_init on the stream, so the scratch may hold anything on entry.
int run_spread(int nx, int ny, int ncaps, const int* off, const double* pos, const double* frc,
               double* Fx, double* Fy, SpreadScratch sc, int M, int T, int tiles_x,
               cudaStream_t st) {
    int nsm = 0, dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        sfg_host::set_error(std::string("spread: ") + cudaGetErrorString(e));
        return SFG_ERR_CUDA;
    }
    const int B = 256, G = (M + B - 1) / B;
    const int Gi = std::min((std::max(T, 1025) + B - 1) / B, nsm * 8);
    k_sa_init<<<Gi, B, 0, st>>>(T, sc);
    k_sa_prep<<<G, B, 0, st>>>(nx, ny, tiles_x, ncaps, off,
                               reinterpret_cast<const double2*>(pos),
                               reinterpret_cast<const double2*>(frc), M, sc);
    scan_exclusive(sc.tile_cnt, sc.tile_off, T, sc.scan_tmp, nullptr, st);
    k_sa_fill<<<G, B, 0, st>>>(nx, ny, tiles_x, M, sc);
    const int grid = std::max(1, std::min((T + SA_WARPS - 1) / SA_WARPS, nsm * 4));
    k_sa_gather<<<grid, SA_WARPS * 32, 0, st>>>(nx, ny, tiles_x, T,
                                                reinterpret_cast<const double2*>(pos),
                                                reinterpret_cast<const double2*>(frc), sc.phi, sc,
                                                Fx, Fy);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        sfg_host::set_error(std::string("spread: ") + cudaGetErrorString(e));
        return SFG_ERR_CUDA;
    }
    return SFG_OK;
}

int check_spread_args(int nx, int ny, int ncaps, const int* off, const double* pos,
                      const double* frc, const double* Fx, const double* Fy, const char* who) {
    if (nx < 4 || ny < 1) {
        sfg_host::set_error(std::string(who) + ": need nx >= 4 and ny >= 1");
        return SFG_ERR_ARG;
    }
    if (ncaps < 0 || (ncaps > 0 && (!off || !pos || !frc)) || !Fx || !Fy) {
        sfg_host::set_error(std::string(who) + ": null or negative argument");
        return SFG_ERR_ARG;
    }
    return SFG_OK;
}

}  // namespace sfg

using namespace sfg;

extern "C" int sfg_spread_forces(int nx, int ny, int ncaps, const int* d_offsets,
                                 const double* d_pos, const double* d_force, double* d_Fx,
                                 double* d_Fy, int num_markers, void* stream) {
    int rc = check_spread_args(nx, ny, ncaps, d_offsets, d_pos, d_force, d_Fx, d_Fy,
                               "sfg_spread_forces");
    if (rc) return rc;
    if (ncaps == 0 || num_markers <= 0) return SFG_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int tiles_x = (nx + TILE_W - 1) / TILE_W, tiles_y = (ny + TILE_H - 1) / TILE_H;
    const int T = tiles_x * tiles_y, M = num_markers;
    void* base = nullptr;
    cudaError_t e = cudaMallocAsync(&base, spread_scratch_bytes(M, T), st);
    if (e != cudaSuccess) {
        sfg_host::set_error(std::string("sfg_spread_forces: ") + cudaGetErrorString(e));
        return SFG_ERR_CUDA;
    }
    rc = run_spread(nx, ny, ncaps, d_offsets, d_pos, d_force, d_Fx, d_Fy,
                    carve_spread_scratch(base, M, T), M, T, tiles_x, st);
    e = cudaFreeAsync(base, st);
    if (rc == SFG_OK && e != cudaSuccess) {
        sfg_host::set_error(std::string("sfg_spread_forces: ") + cudaGetErrorString(e));
        return SFG_ERR_CUDA;
    }
    return rc;
}
