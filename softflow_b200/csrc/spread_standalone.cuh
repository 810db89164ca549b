// spread_standalone.cuh -- scratch layout and helpers of sfg_spread_forces.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace sfg {

// Scratch of one standalone spread call (global memory beyond the caller's
// inputs and outputs).
struct SpreadScratch {
    double* ds = nullptr;       // [M] arc length per marker
    int* ix0 = nullptr;         // [M] stencil origin (INT_MIN: marker skipped)
    int* iy0 = nullptr;         // [M]
    int* list = nullptr;        // [8 M] markers per covered tile
    int* tile_cnt = nullptr;    // [T]
    int* tile_off = nullptr;    // [T]
    int* cursor = nullptr;      // [T]
    int* scan_tmp = nullptr;
    double* phi = nullptr;      // [1025] Peskin table
};

size_t spread_scratch_bytes(int M, int T);
SpreadScratch carve_spread_scratch(void* base, int M, int T);
int run_spread(int nx, int ny, int ncaps, const int* off, const double* pos, const double* frc,
               double* Fx, double* Fy, SpreadScratch sc, int M, int T, int tiles_x,
               cudaStream_t st);
int check_spread_args(int nx, int ny, int ncaps, const int* off, const double* pos,
                      const double* frc, const double* Fx, const double* Fy, const char* who);

}  // namespace sfg
