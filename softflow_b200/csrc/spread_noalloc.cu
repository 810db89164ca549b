// spread_noalloc.cu -- sfg_spread_forces_noalloc: the deterministic spread of
// sfg_spread_forces with its scratch in a fixed device array instead of
// cudaMallocAsync.
//
// Who needs it: callers that must not allocate device memory during a call,
// for example a host engine or framework that owns the whole device memory
// budget through its own pool (a direct cudaMalloc would fail or fragment that
// pool), or a time-stepping loop that must not stall: cudaMalloc / cudaFree
// can synchronize the device.  Such callers pass only their input and output
// buffers.
//
// Limits and sharing:
//   - at most NOALLOC_MAX_MARKERS markers and NOALLOC_MAX_TILES force tiles
//     (32 x 8 cells each, so ceil(nx/32) * ceil(ny/8) <= NOALLOC_MAX_TILES);
//     larger calls are rejected with SFG_ERR_CAPACITY;
//   - the array is NOALLOC_SCRATCH_BYTES (2 MiB) of device memory on every GPU
//     that loads the library, held until the process exits;
//   - every call uses the same array and it keeps the last call's contents;
//     each call clears the parts that must start at zero.  Calls whose GPU
//     work overlaps (different streams, or different host threads on one
//     device) race on the array and must be serialized by the caller;
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture on the device.
#include <mutex>
#include <string>

#include "../../include/softflow_gpu.h"
#include "spread_standalone.cuh"
#include "common.cuh"

namespace sfg_host {
void set_error(const std::string& msg);
}

namespace {

constexpr int NOALLOC_MAX_MARKERS = 32768;
constexpr int NOALLOC_MAX_TILES = 32768;
constexpr size_t NOALLOC_SCRATCH_BYTES = 2u << 20;

// The scratch itself.  In host code this name is only a host-side stand-in,
// never a device address: the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_spread_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

int fail(int code, const std::string& msg) {
    sfg_host::set_error(msg);
    return code;
}

// Device address of the scratch on the current device (looked up once per
// device, with that device current).
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(SFG_ERR_CUDA, std::string("sfg_spread_forces_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(SFG_ERR_ARG, "sfg_spread_forces_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_spread_scratch);
        if (e != cudaSuccess || p == nullptr)
            return fail(SFG_ERR_CUDA, std::string("sfg_spread_forces_noalloc: scratch lookup: ") +
                                          cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SFG_OK;
}

}  // namespace

extern "C" int sfg_spread_forces_noalloc(int nx, int ny, int ncaps, const int* d_offsets,
                                         const double* d_pos, const double* d_force,
                                         double* d_Fx, double* d_Fy, int num_markers,
                                         void* stream) {
    using namespace sfg;
    int rc = check_spread_args(nx, ny, ncaps, d_offsets, d_pos, d_force, d_Fx, d_Fy,
                               "sfg_spread_forces_noalloc");
    if (rc) return rc;
    if (ncaps == 0 || num_markers <= 0) return SFG_OK;
    const int tiles_x = (nx + TILE_W - 1) / TILE_W, tiles_y = (ny + TILE_H - 1) / TILE_H;
    const long long T = (long long)tiles_x * tiles_y;
    if (num_markers > NOALLOC_MAX_MARKERS)
        return fail(SFG_ERR_CAPACITY, "sfg_spread_forces_noalloc: " +
                                          std::to_string(num_markers) + " markers exceed the " +
                                          std::to_string(NOALLOC_MAX_MARKERS) + "-marker limit");
    if (T > NOALLOC_MAX_TILES)
        return fail(SFG_ERR_CAPACITY, "sfg_spread_forces_noalloc: lattice " + std::to_string(nx) +
                                          " x " + std::to_string(ny) + " needs " +
                                          std::to_string(T) + " force tiles, limit " +
                                          std::to_string(NOALLOC_MAX_TILES));
    if (spread_scratch_bytes(num_markers, (int)T) > NOALLOC_SCRATCH_BYTES)
        return fail(SFG_ERR_CAPACITY, "sfg_spread_forces_noalloc: scratch exceeds 2 MiB");
    void* base = nullptr;
    if ((rc = scratch_address(&base))) return rc;
    return run_spread(nx, ny, ncaps, d_offsets, d_pos, d_force, d_Fx, d_Fy,
                      carve_spread_scratch(base, num_markers, (int)T), num_markers, (int)T,
                      tiles_x, static_cast<cudaStream_t>(stream));
}
