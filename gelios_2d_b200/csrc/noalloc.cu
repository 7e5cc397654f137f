// Allocation-free entry point: one plain single-fluid step (the Go_stationary
// form) on grid and state arrays that the caller already holds in device
// memory.
//
// Who needs it: callers that cannot call cudaMalloc at the time they step —
// for example a host code whose device memory is all handed out up front by
// its own pool, or a driver that steps from inside a region where the CUDA
// allocator must not be touched.  gelios_create/gelios_upload_* allocate the
// context's buffers; this entry point allocates nothing.  Its scratch (the
// per-face-slot fluxes, the cell centroids and the dt/status words of the
// step) lives in one file-scope __device__ array of fixed size, so a grid is
// accepted only up to GELIOS_NOALLOC_MAX_CELLS cells and
// GELIOS_NOALLOC_MAX_SLOTS face slots.
//
// The kernels are the ones gelios_step runs for GELIOS_FORM_STATIONARY; only
// the scratch pointers differ.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/gelios_b200.h"
#include "physics.cuh"
#include "step_kernels.cuh"

namespace gelios {
void set_error(const std::string& msg);
}
using namespace gelios;

namespace {

// scratch layout (doubles): flux slots [5 * MAX_SLOTS], centroids and
// |centroid|^(2 gamma) [3 * MAX_CELLS],
// then 8 doubles of dt/status words (T unused, acc, counters[2], status)
constexpr size_t kFluxDoubles = 5ull * GELIOS_NOALLOC_MAX_SLOTS;
constexpr size_t kCenDoubles = 3ull * GELIOS_NOALLOC_MAX_CELLS;
constexpr size_t kWordDoubles = 8;
constexpr size_t kScratchDoubles = kFluxDoubles + kCenDoubles + kWordDoubles;

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch per device, resolved once per device.
constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

__global__ void noalloc_words_init(unsigned long long* acc, unsigned long long* counters, int* status) {
    *acc = 0x7ff0000000000000ULL;  // +inf: no CFL candidate yet
    counters[0] = 0;
    counters[1] = 0;
    *status = 0;
}

// Go_stationary leaves C_centr cells as they are (Setka.cpp:5239); the
// context path keeps both state buffers equal there.  Here state_out may be a
// fresh array, so those cells are copied through from state_in.
__global__ void noalloc_copy_centr(const uint32_t* __restrict__ flags, int n, StepBuffers b) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || !(flags[c] & CF_CENTR)) return;
    for (int k = 0; k < 5; k++) b.nxt[k][c] = b.cur[k][c];
}

}  // namespace

extern "C" int gelios_stationary_step_noalloc(const gelios_params* prm, const gelios_device_grid* g,
                                              const double* const* state_in, double* const* state_out,
                                              const double* dt_in, double* dt_out, void* stream) {
    if (!prm || !g || !state_in || !state_out || !dt_in || !dt_out) {
        set_error("gelios_stationary_step_noalloc: null argument");
        return GELIOS_E_ARG;
    }
    for (int k = 0; k < 5; k++)
        if (!state_in[k] || !state_out[k]) {
            set_error("gelios_stationary_step_noalloc: null state array");
            return GELIOS_E_ARG;
        }
    if (g->n_cells <= 0 || g->n_slots <= 0 || g->n_units <= 0 || !g->x || !g->y || !g->contour_start ||
        !g->contour || !g->gran_start || !g->cell_flags || !g->slot_A || !g->slot_B || !g->slot_nb ||
        !g->slot_info || !g->unit_slot || !g->unit_cell || !g->unit_twin) {
        set_error("gelios_stationary_step_noalloc: incomplete device grid");
        return GELIOS_E_ARG;
    }
    if (g->n_cells > GELIOS_NOALLOC_MAX_CELLS || g->n_slots > GELIOS_NOALLOC_MAX_SLOTS) {
        set_error("gelios_stationary_step_noalloc: grid of " + std::to_string(g->n_cells) + " cells / " +
                  std::to_string(g->n_slots) + " face slots exceeds the fixed scratch (" +
                  std::to_string(GELIOS_NOALLOC_MAX_CELLS) + " cells, " +
                  std::to_string(GELIOS_NOALLOC_MAX_SLOTS) + " slots)");
        return GELIOS_E_LIMIT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("gelios_stationary_step_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        return GELIOS_E_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("gelios_stationary_step_noalloc: device index beyond the supported range");
        return GELIOS_E_LIMIT;
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            // first call on this device (the current one): resolve the device
            // address of the file-scope array
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                set_error(std::string("gelios_stationary_step_noalloc: cudaGetSymbolAddress: ") +
                          cudaGetErrorString(e));
                return GELIOS_E_CUDA;
            }
            g_scratch_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevMesh d;
    d.n_cells = g->n_cells;
    d.n_slots = g->n_slots;
    d.n_units = g->n_units;
    d.X = const_cast<double*>(g->x);
    d.Y = const_cast<double*>(g->y);
    d.cstart = g->contour_start;
    d.contour = g->contour;
    d.gstart = g->gran_start;
    d.cflags = g->cell_flags;
    d.sA = g->slot_A;
    d.sB = g->slot_B;
    d.snb = g->slot_nb;
    d.sinfo = g->slot_info;
    d.u_slot = g->unit_slot;
    d.u_cell = g->unit_cell;
    d.u_twin = g->unit_twin;
    double* flux = scratch;
    double* cen = scratch + kFluxDoubles;
    char* words = reinterpret_cast<char*>(scratch + kFluxDoubles + kCenDoubles);
    StepBuffers b;
    for (int k = 0; k < 5; k++) {
        b.cur[k] = state_in[k];
        b.nxt[k] = state_out[k];
    }
    b.cx = cen;
    b.cy = cen + GELIOS_NOALLOC_MAX_CELLS;
    b.rp = cen + 2 * GELIOS_NOALLOC_MAX_CELLS;
    b.dt_cur = dt_in;
    b.dt_next = dt_out;
    b.dt_acc = reinterpret_cast<unsigned long long*>(words + 8);
    b.counters = reinterpret_cast<unsigned long long*>(words + 16);
    b.status = reinterpret_cast<int*>(words + 32);
    // the array keeps the last call's contents: re-arm the words first
    noalloc_words_init<<<1, 1, 0, s>>>(b.dt_acc, b.counters, b.status);
    launch_centroid(d, d.X, d.Y, cen, cen + GELIOS_NOALLOC_MAX_CELLS, cen + 2 * GELIOS_NOALLOC_MAX_CELLS, prm->gamma,
                    s);
    launch_stationary_units(d, *prm, b, flux, s);
    launch_stationary_update(d, *prm, b, flux, s);
    noalloc_copy_centr<<<(d.n_cells + 127) / 128, 128, 0, s>>>(d.cflags, d.n_cells, b);
    launch_dt_finalize(b, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("gelios_stationary_step_noalloc: launch: ") + cudaGetErrorString(e));
        return GELIOS_E_CUDA;
    }
    return GELIOS_OK;
}
