// C ABI of the hot path (include/als_b200.h): plug-in level calls that
// mirror one virtual call of the reference interfaces each, the fused
// solver that runs whole time steps of one grid or of several grid levels
// on the device, and the FP64 ensemble statistics.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "als_b200.h"
#include "aux_kernels.cuh"
#include "scratch.h"
#include "stage_dispatch.cuh"

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define ALS_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t err_ = (call);                                                      \
        if (err_ != cudaSuccess) {                                                      \
            std::ostringstream os_;                                                     \
            os_ << #call << ": " << cudaGetErrorString(err_);                           \
            return fail(ALS_E_CUDA, os_.str());                                         \
        }                                                                               \
    } while (0)

int grid_blocks(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    if (b < 1) {
        b = 1;
    }
    // enough blocks for every SM several times over, then grid-stride
    return int(std::min<long long>(b, 148LL * 32));
}

bool valid_choice(int flux, int recon) {
    return flux >= ALS_FLUX_HLL && flux <= ALS_FLUX_TECNO6 && recon >= ALS_RECON_NONE &&
        recon <= ALS_RECON_WENO3;
}

// The TeCNO fluxes are built with reconstruction "none", the way the
// reference pairs them (the high-order part of the TeCNO scheme sits in its
// diffusion operator); the stencil fluxes tecno4/6 read the cell values.
int check_supported(int flux, int recon) {
    if (flux >= ALS_FLUX_TECNO1 && recon != ALS_RECON_NONE) {
        return fail(ALS_E_UNSUPPORTED, "the TeCNO fluxes are built for reconstruction \"none\"");
    }
    return ALS_OK;
}

cudaError_t launch_stage(int precision, int dim, int recon, int flux, int kind,
    const als::StageParams& P, int blocks_per_sm, cudaStream_t s, int shape = 0) {
    if (precision == ALS_FP64) {
        switch (dim) {
        case 1: return als::launch_stage_f64_1d(recon, flux, kind, shape, P, blocks_per_sm, s);
        case 2: return als::launch_stage_f64_2d(recon, flux, kind, shape, P, blocks_per_sm, s);
        default: return als::launch_stage_f64_3d(recon, flux, kind, shape, P, blocks_per_sm, s);
        }
    }
    switch (dim) {
    case 1: return als::launch_stage_f32_1d(recon, flux, kind, shape, P, blocks_per_sm, s);
    case 2: return als::launch_stage_f32_2d(recon, flux, kind, shape, P, blocks_per_sm, s);
    default: return als::launch_stage_f32_3d(recon, flux, kind, shape, P, blocks_per_sm, s);
    }
}

// Tile extent along d of tile shape `shape` of the kernels built for
// (precision, dim), as reported by the unit that holds them.
int tile_extent(int precision, int dim, int d, int shape = 0) {
    if (d >= dim) {
        return 1;
    }
    int tile[3] = {1, 1, 1};
    if (precision == ALS_FP64) {
        dim == 1 ? als::stage_tile_f64_1d(shape, tile)
                 : (dim == 2 ? als::stage_tile_f64_2d(shape, tile) : als::stage_tile_f64_3d(shape, tile));
    } else {
        dim == 1 ? als::stage_tile_f32_1d(shape, tile)
                 : (dim == 2 ? als::stage_tile_f32_2d(shape, tile) : als::stage_tile_f32_3d(shape, tile));
    }
    return tile[d];
}

// Geometry of a padded grid and the tiles (of shape `shape`) covering the
// region [lo, hi).
als::GridDesc make_grid(int dim, const int* n, int g, const int* lo, const int* hi,
    int precision = ALS_FP64, int shape = 0) {
    als::GridDesc gd;
    for (int d = 0; d < 3; ++d) {
        gd.n[d] = d < dim ? n[d] : 1;
        gd.N[d] = gd.n[d] + (d < dim ? 2 * g : 0);
        gd.lo[d] = d < dim ? lo[d] : 0;
        gd.hi[d] = d < dim ? hi[d] : 1;
        const int t = tile_extent(precision, dim, d, shape);
        gd.tiles[d] = std::max(1, (gd.hi[d] - gd.lo[d] + t - 1) / t);
    }
    gd.plane = (long long)gd.N[0] * gd.N[1] * gd.N[2];
    gd.ghosts = g;
    return gd;
}

int check_grid(const als_grid* g) {
    if (!g || g->dimension < 1 || g->dimension > 3 || g->ghosts < 1) {
        return fail(ALS_E_INVALID, "invalid grid");
    }
    for (int d = 0; d < g->dimension; ++d) {
        if (g->n[d] < g->ghosts) {
            return fail(ALS_E_INVALID, "every active direction needs at least `ghosts` interior cells");
        }
    }
    return ALS_OK;
}

int check_planes(const void* const* planes, int nvar) {
    if (!planes) {
        return fail(ALS_E_INVALID, "null plane array");
    }
    for (int v = 0; v < nvar; ++v) {
        if (!planes[v]) {
            return fail(ALS_E_INVALID, "null plane pointer");
        }
    }
    return ALS_OK;
}

// A level of one state given as one pointer per variable.
als::LevelDesc plane_level(const als::GridDesc& gd, int nvar, const void* const* in,
    const void* const* un, void* const* out) {
    als::LevelDesc L;
    std::memset(&L, 0, sizeof(L));
    L.grid = gd;
    for (int v = 0; v < nvar; ++v) {
        L.in[v] = in[v];
        L.un[v] = un[v];
        L.out[v] = out[v];
    }
    L.member_stride = 0;
    L.members = 1;
    L.tiles_per_member = gd.tiles[0] * gd.tiles[1] * gd.tiles[2];
    return L;
}

// Fills work_begin of every level and the total work of the launch.
void finish_params(als::StageParams& P) {
    long long w = 0;
    for (int l = 0; l < P.nlevels; ++l) {
        P.level[l].work_begin = w;
        w += (long long)P.level[l].members * P.level[l].tiles_per_member;
    }
    P.total_work = w;
}

template<class R>
als::Planes<R> planes_of(void* const* p, int nvar) {
    als::Planes<R> out;
    std::memset(&out, 0, sizeof(out));
    for (int v = 0; v < nvar; ++v) {
        out.p[v] = static_cast<R*>(p[v]);
    }
    return out;
}

template<class R>
als::Planes<R> contiguous_planes(void* base, int nvar, long long plane) {
    als::Planes<R> out;
    std::memset(&out, 0, sizeof(out));
    for (int v = 0; v < nvar; ++v) {
        out.p[v] = static_cast<R*>(base) + v * plane;
    }
    return out;
}

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        cudaSetDevice(prev);
    }
};

} // namespace

namespace als {
// Error text for the other translation units of the library (one message
// per host thread, read by als_last_error).
int report_error(int code, const char* msg) {
    return fail(code, msg);
}

// One retaining pool per device: the release threshold is unlimited, so
// the scratch of repeated calls is not unmapped and re-mapped at every
// synchronisation; als_scratch_trim hands the unused part back.
std::mutex g_scratch_mutex;
cudaMemPool_t g_scratch_pools[256] = {};

// The library's pool on the current device, created on first use.
static cudaError_t scratch_pool(cudaMemPool_t* pool) {
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) {
        return err;
    }
    if (device < 0 || device >= 256) {
        return cudaErrorInvalidDevice;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_pools[device]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        err = cudaMemPoolCreate(&p, &props);
        if (err != cudaSuccess) {
            return err;
        }
        unsigned long long keep = ~0ULL;   // the attribute is a 64-bit unsigned value
        err = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (err != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return err;
        }
        g_scratch_pools[device] = p;
    }
    *pool = g_scratch_pools[device];
    return cudaSuccess;
}

cudaError_t scratch_alloc(void** ptr, size_t bytes, cudaStream_t stream) {
    cudaMemPool_t pool = nullptr;
    const cudaError_t err = scratch_pool(&pool);
    if (err != cudaSuccess) {
        return err;
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
}

cudaError_t scratch_free(void* ptr, cudaStream_t stream) {
    return cudaFreeAsync(ptr, stream);
}
} // namespace als

extern "C" {

const char* als_last_error(void) {
    return g_error.c_str();
}

int als_scratch_trim(int device, unsigned long long keep_bytes) {
    if (device < 0 || device >= 256) {
        return fail(ALS_E_INVALID, "invalid device");
    }
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(als::g_scratch_mutex);
        pool = als::g_scratch_pools[device];
    }
    if (!pool) {
        return ALS_OK;
    }
    DeviceGuard guard(device);
    ALS_CUDA(cudaMemPoolTrimTo(pool, size_t(keep_bytes)));
    return ALS_OK;
}

int als_version(void) {
    return 2;
}

int als_ghost_cells(int flux, int reconstruction) {
    if (!valid_choice(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "unknown flux or reconstruction");
    }
    const int rc = check_supported(flux, reconstruction);
    if (rc != ALS_OK) {
        return rc;
    }
    // max(stencil size - 1, reconstruction ghosts) (NumericalFluxCPU.cpp:225-231)
    return als::stage_ghosts(reconstruction, flux);
}

} // extern "C"

namespace {

// Three wave-speed accumulators per host thread and device for
// als_compute_flux, allocated on first use and kept: a per-call
// cudaMallocAsync/cudaFreeAsync pair costs a pool release and re-map at
// every synchronisation (the default pool keeps nothing), several hundred
// microseconds per call.  A call that reads them back synchronises before
// it returns, so one thread never has two calls using them at once.
struct ThreadWaveSpeeds {
    std::vector<unsigned long long*> by_device;
    ~ThreadWaveSpeeds() {
        for (unsigned long long* p : by_device) {
            if (p) {
                cudaFree(p);   // at process exit the context may be gone: ignored
            }
        }
    }
};

int thread_wave_speed_scratch(unsigned long long** out) {
    thread_local ThreadWaveSpeeds slots;
    int device = 0;
    ALS_CUDA(cudaGetDevice(&device));
    if (device < 0) {
        return fail(ALS_E_CUDA, "no current device");
    }
    if (size_t(device) >= slots.by_device.size()) {
        slots.by_device.resize(size_t(device) + 1, nullptr);
    }
    if (!slots.by_device[device]) {
        ALS_CUDA(cudaMalloc((void**)&slots.by_device[device], 3 * sizeof(unsigned long long)));
    }
    *out = slots.by_device[device];
    return ALS_OK;
}

// Write-only accumulators of the calls that want no wave speeds (one array
// per device; concurrent calls only race on values nobody reads), and its
// address per device, looked up once.
static __device__ unsigned long long g_discarded_wave_speeds[3];
std::mutex g_discard_mutex;
void* g_discard_address[256] = {};

unsigned long long* discard_wave_speeds() {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 256) {
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_discard_mutex);
    if (!g_discard_address[device] &&
        cudaGetSymbolAddress(&g_discard_address[device], g_discarded_wave_speeds) != cudaSuccess) {
        g_discard_address[device] = nullptr;
    }
    return static_cast<unsigned long long*>(g_discard_address[device]);
}

} // namespace

extern "C" {

int als_fill_ghosts(const als_grid* grid, int boundary, double* const* planes, int nvar,
    void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (nvar < 1 || nvar > als::kMaxVars || (boundary != ALS_BC_NEUMANN && boundary != ALS_BC_PERIODIC)) {
        return fail(ALS_E_INVALID, "invalid ghost-fill arguments");
    }
    rc = check_planes((const void* const*)planes, nvar);
    if (rc != ALS_OK) {
        return rc;
    }
    int lo[3] = {0, 0, 0};
    als::GridDesc gd = make_grid(grid->dimension, grid->n, grid->ghosts, lo, grid->n);
    dim3 blocks(grid_blocks(als::ghost_shell_cells(grid->dimension, gd.n[0], gd.n[1], gd.n[2],
        grid->ghosts), 256), 1);
    als::fill_ghosts<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(
        planes_of<double>((void* const*)planes, nvar), nvar, gd.plane, 0, grid->dimension,
        gd.n[0], gd.n[1], gd.n[2], grid->ghosts, boundary);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int als_compute_flux(const als_grid* grid, int flux, int reconstruction, const double* const* in,
    double* const* out, const int* start, const int* end, double* wave_speed, void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!valid_choice(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "invalid flux arguments");
    }
    rc = check_supported(flux, reconstruction);
    if (rc != ALS_OK) {
        return rc;
    }
    const int nvar = grid->dimension + 2;
    rc = check_planes((const void* const*)in, nvar);
    if (rc == ALS_OK) {
        rc = check_planes((const void* const*)out, nvar);
    }
    if (rc != ALS_OK) {
        return rc;
    }
    // wider planes are fine: the reference sizes ghosts as the maximum of
    // the flux's and the diffusion operator's (ConservedSystem.cpp:109-114)
    if (grid->ghosts < als_ghost_cells(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "planes have fewer ghost cells than the flux needs");
    }
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
        const int n = d < grid->dimension ? grid->n[d] : 1;
        lo[d] = start ? start[d] : 0;
        hi[d] = n + (end ? end[d] : 0);
        if (d < grid->dimension && (lo[d] < 0 || hi[d] > n || lo[d] >= hi[d])) {
            return fail(ALS_E_INVALID, "region must lie inside the interior");
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    als::StageParams P;
    std::memset(&P, 0, sizeof(P));
    als::GridDesc gd = make_grid(grid->dimension, grid->n, grid->ghosts, lo, hi);
    P.level[0] = plane_level(gd, nvar, (const void* const*)in, (const void* const*)in,
        (void* const*)out);
    P.nlevels = 1;
    P.bc = ALS_BC_NEUMANN;
    P.write_ghosts = 0;
    P.gamma = grid->gamma;
    unsigned long long* ws_dev = nullptr;
    if (wave_speed) {
        rc = thread_wave_speed_scratch(&ws_dev);
        if (rc != ALS_OK) {
            return rc;
        }
        ALS_CUDA(cudaMemsetAsync(ws_dev, 0, 3 * sizeof(unsigned long long), s));
    }
    // without a destination the kernel still reduces the face speeds; the
    // level's accumulators then go to a slot nobody reads
    P.level[0].ws_out = ws_dev ? ws_dev : discard_wave_speeds();
    finish_params(P);
    if (!P.level[0].ws_out) {
        return fail(ALS_E_CUDA, "wave-speed scratch unavailable");
    }
    ALS_CUDA(launch_stage(ALS_FP64, grid->dimension, reconstruction, flux, als::KIND_FLUX0, P, 0, s));
    if (!wave_speed) {
        return ALS_OK;
    }
    unsigned long long host[3] = {0, 0, 0};
    ALS_CUDA(cudaMemcpyAsync(host, ws_dev, sizeof(host), cudaMemcpyDeviceToHost, s));
    ALS_CUDA(cudaStreamSynchronize(s));
    for (int d = 0; d < 3; ++d) {
        double w;
        std::memcpy(&w, &host[d], sizeof(w));
        wave_speed[d] = w;
    }
    return ALS_OK;
}

int als_reconstruct(const als_grid* grid, int reconstruction, int direction,
    const double* const* in, double* const* left, double* const* right, void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    const int nvar = grid->dimension + 2;
    if (direction < 0 || direction >= grid->dimension || reconstruction < ALS_RECON_NONE ||
        reconstruction > ALS_RECON_WENO3) {
        return fail(ALS_E_INVALID, "invalid reconstruction arguments");
    }
    rc = check_planes((const void* const*)in, nvar);
    if (rc == ALS_OK) {
        rc = check_planes((const void* const*)left, nvar);
    }
    if (rc == ALS_OK) {
        rc = check_planes((const void* const*)right, nvar);
    }
    if (rc != ALS_OK) {
        return rc;
    }
    const int G = grid->ghosts;
    if (G != std::max(1, als::recon_ghosts(reconstruction))) {
        return fail(ALS_E_UNSUPPORTED, "planes must have exactly the ghost width of the reconstruction");
    }
    int N[3];
    long long plane = 1;
    for (int d = 0; d < 3; ++d) {
        N[d] = d < grid->dimension ? grid->n[d] + 2 * G : 1;
        plane *= N[d];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int dim = grid->dimension;
    if (reconstruction == ALS_RECON_NONE) {
        // NoReconstruction copies every cell, ghosts included (NoReconstruction.cpp:51-61)
        for (int v = 0; v < nvar; ++v) {
            ALS_CUDA(cudaMemcpyAsync(left[v], in[v], sizeof(double) * plane, cudaMemcpyDeviceToDevice, s));
            ALS_CUDA(cudaMemcpyAsync(right[v], in[v], sizeof(double) * plane, cudaMemcpyDeviceToDevice, s));
        }
        return ALS_OK;
    }
    const int blocks = grid_blocks(plane, 256);
    const als::Planes<double> pin = planes_of<double>((void* const*)in, nvar);
    const als::Planes<double> pl = planes_of<double>((void* const*)left, nvar);
    const als::Planes<double> pr = planes_of<double>((void* const*)right, nvar);
#define ALS_RECON_CASE(NV, RC)                                                               \
    als::reconstruct_dir<double, NV, RC><<<blocks, 256, 0, s>>>(pin, pl, pr, dim, N[0], N[1], \
        N[2], G, direction, grid->gamma)
#define ALS_RECON_NV(NV)                                                                     \
    switch (reconstruction) {                                                                \
    case ALS_RECON_WENO2: ALS_RECON_CASE(NV, als::RECON_WENO2); break;                       \
    case ALS_RECON_ENO2: ALS_RECON_CASE(NV, als::RECON_ENO2); break;                         \
    case ALS_RECON_ENO3: ALS_RECON_CASE(NV, als::RECON_ENO3); break;                         \
    case ALS_RECON_MC: ALS_RECON_CASE(NV, als::RECON_MC); break;                             \
    case ALS_RECON_MM: ALS_RECON_CASE(NV, als::RECON_MM); break;                             \
    case ALS_RECON_WENOF2: ALS_RECON_CASE(NV, als::RECON_WENOF2); break;                     \
    case ALS_RECON_WENO3: ALS_RECON_CASE(NV, als::RECON_WENO3); break;                       \
    default: ALS_RECON_CASE(NV, als::RECON_ENO4); break;                                     \
    }
    if (dim == 1) {
        ALS_RECON_NV(3)
    } else if (dim == 2) {
        ALS_RECON_NV(4)
    } else {
        ALS_RECON_NV(5)
    }
#undef ALS_RECON_NV
#undef ALS_RECON_CASE
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int als_integrator_combine(int integrator, int substep, double* out, const double* us,
    const double* u0, size_t count, double c, void* stream) {
    const int substeps = integrator + 1;
    if (integrator < ALS_INT_FORWARD_EULER || integrator > ALS_INT_RK4 || substep < 0 ||
        substep >= substeps || !out || !us || ((substep > 0 || integrator == ALS_INT_RK4) && !u0)) {
        return fail(ALS_E_INVALID, "invalid combine arguments");
    }
    if (integrator == ALS_INT_RK4 && substep == 3) {
        return fail(ALS_E_INVALID, "RK4's last stage combines five volumes: als_integrator_combine_rk4");
    }
    als::combine<double><<<grid_blocks((long long)count, 256), 256, 0, (cudaStream_t)stream>>>(
        out, us, u0, (long long)count, c, integrator, substep);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int als_integrator_combine_rk4(double* out, const double* u0, const double* u1, const double* u2,
    const double* u3, size_t count, double c, void* stream) {
    if (!out || !u0 || !u1 || !u2 || !u3) {
        return fail(ALS_E_INVALID, "invalid combine arguments");
    }
    // a1 = (1.0 / 6.0) * cellScaling.x (RungeKutta4.cpp:81)
    const double a1 = (1.0 / 6.0) * c;
    als::combine_rk4_final<double><<<grid_blocks((long long)count, 256), 256, 0,
        (cudaStream_t)stream>>>(out, u0, u1, u2, u3, (long long)count, a1);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

double als_compute_timestep(const double* wave_speed, const double* cell_lengths, double cfl,
    double t, double end_time) {
    double total = 0;
    for (int d = 0; d < 3; ++d) {
        if (cell_lengths[d] == 0) {
            continue;
        }
        total += wave_speed[d] / cell_lengths[d];
    }
    const double dt = cfl / total;
    const double rest = end_time - t;
    return rest < dt ? rest : dt;
}

} // extern "C"

// ------------------------------------------------------------------ solver

namespace {

// One grid level of a solver: its geometry, its members and its buffers.
struct SolverLevel {
    als_solver_config cfg;        // this level's n, lower, upper, members
    als::GridDesc grid;           // tiles of this level's tile shape
    int shape = 0;                // tile shape of its stage kernels (stage_kernel.cuh)
    int first = 0;                // global index of its first member
    long long member_elems = 0;   // nvar * plane
    double dx[3];
    void* buf[3] = {nullptr, nullptr, nullptr};  // state A, flux L, state B
};

} // namespace

struct als_solver {
    als_solver_config cfg;        // shared settings (level 0's config)
    int device = 0;
    int g = 0;
    int nv = 0;
    size_t elem = 8;
    std::vector<SolverLevel> levels;
    std::vector<int> order;       // order of the levels in the work list
    int blocks_per_sm = 0;        // 0: one block per work item; > 0: persistent, blocks per SM
    unsigned long long* counter = nullptr;  // work counter of the persistent launches
    int members = 0;              // over all levels
    int subdomains = 0;           // 1: the members are subdomains of one grid (als_solver_decompose)
    int procs[3] = {1, 1, 1};     // subdomains per direction
    bool needs_state = false;     // split after its state was set: advancing waits for a new one
    int cur = 0;                  // RK2 ping-pong: 1 when U^n of active members sits in B
    als::StepState* state = nullptr;
    als::StepState* host_state = nullptr;  // pinned mirror
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int graph_cur = 0;

    ~als_solver() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (graph) {
            cudaGraphExecDestroy(graph);
        }
        for (SolverLevel& L : levels) {
            for (void* p : L.buf) {
                if (p) {
                    cudaFree(p);
                }
            }
        }
        if (state) {
            cudaFree(state);
        }
        if (counter) {
            cudaFree(counter);
        }
        if (host_state) {
            cudaFreeHost(host_state);
        }
        if (stream) {
            cudaStreamDestroy(stream);
        }
        cudaSetDevice(prev);
    }

    void* current(const SolverLevel& L) const {
        return cfg.integrator == ALS_INT_RK2 && cur == 1 ? L.buf[2] : L.buf[0];
    }
    void* other(const SolverLevel& L) const {
        return cfg.integrator == ALS_INT_RK2 && cur == 1 ? L.buf[0] : L.buf[2];
    }
    int level_of(int member) const {
        for (size_t l = 0; l < levels.size(); ++l) {
            if (member >= levels[l].first && member < levels[l].first + levels[l].cfg.members) {
                return int(l);
            }
        }
        return -1;
    }
};

namespace {

als::LevelDesc solver_level(const als_solver* s, const SolverLevel& L, const void* in,
    const void* un, void* out) {
    als::LevelDesc D;
    std::memset(&D, 0, sizeof(D));
    D.grid = L.grid;
    const long long plane = L.grid.plane;
    for (int v = 0; v < s->nv; ++v) {
        D.in[v] = static_cast<const char*>(in) + size_t(v) * plane * s->elem;
        D.un[v] = static_cast<const char*>(un) + size_t(v) * plane * s->elem;
        D.out[v] = static_cast<char*>(out) + size_t(v) * plane * s->elem;
    }
    D.member_stride = L.member_elems;
    D.state = s->state + L.first;
    D.members = L.cfg.members;
    D.tiles_per_member = L.grid.tiles[0] * L.grid.tiles[1] * L.grid.tiles[2];
    D.subdomains = s->subdomains;
    for (int d = 0; d < 3; ++d) {
        D.procs[d] = s->procs[d];
    }
    return D;
}

// Parameters of one stage over the levels of tile shape `shape`, in the
// solver's level order; `pick` chooses (in, un, out) per level.
template<class Pick>
als::StageParams solver_params(const als_solver* s, Pick pick, int shape = 0) {
    als::StageParams P;
    std::memset(&P, 0, sizeof(P));
    P.nlevels = 0;
    for (size_t k = 0; k < s->levels.size(); ++k) {
        const SolverLevel& L = s->levels[s->order[k]];
        if (L.shape != shape) {
            continue;
        }
        const void* in;
        const void* un;
        void* out;
        pick(L, in, un, out);
        P.level[P.nlevels++] = solver_level(s, L, in, un, out);
    }
    P.bc = s->cfg.boundary;
    P.write_ghosts = 1;
    P.gamma = s->cfg.gamma;
    P.counter = s->blocks_per_sm > 0 ? s->counter : nullptr;
    finish_params(P);
    return P;
}

template<class R, int NV>
cudaError_t launch_fe_update(als_solver* s, const SolverLevel& L) {
    dim3 blocks(grid_blocks(L.grid.plane, 256), L.cfg.members);
    als::fe_update<R, NV><<<blocks, 256, 0, s->stream>>>(static_cast<const R*>(L.buf[1]),
        static_cast<R*>(s->current(L)), L.grid.plane, L.member_elems, s->state + L.first,
        s->cfg.gamma);
    return cudaGetLastError();
}

// Enqueues one time step of every level, each stage as one launch over all
// levels of one tile shape (levels of different shapes take one launch per
// shape, in shape order).  FE: FLUX0 + fe_update.  RK2: FLUX0 + RK2_1 into
// the other buffer (ping-pong).  RK3: FLUX0 + RK3_1 + RK3_2 in place.  With
// `ev` (stages+1 events), records ev[0] before the first kernel and ev[k]
// after the launches of stage k.
template<class Pick>
cudaError_t launch_stage_all(const als_solver* s, int kind, Pick pick) {
    for (int shape = 0; shape < als::kMaxShapes; ++shape) {
        als::StageParams P = solver_params(s, pick, shape);
        if (P.nlevels == 0) {
            continue;
        }
        cudaError_t err = launch_stage(s->cfg.precision, s->cfg.dimension, s->cfg.reconstruction,
            s->cfg.flux, kind, P, s->blocks_per_sm, s->stream, shape);
        if (err != cudaSuccess) {
            return err;
        }
    }
    return cudaSuccess;
}

int enqueue_step(als_solver* s, cudaEvent_t* ev = nullptr) {
    const int prec = s->cfg.precision;
    const int dim = s->cfg.dimension;
    if (ev) {
        ALS_CUDA(cudaEventRecord(ev[0], s->stream));
    }
    ALS_CUDA(launch_stage_all(s, als::KIND_FLUX0, [s](const SolverLevel& L, const void*& in,
                                                      const void*& un, void*& out) {
        in = s->current(L);
        un = in;
        out = L.buf[1];
    }));
    if (ev) {
        ALS_CUDA(cudaEventRecord(ev[1], s->stream));
    }
    if (s->cfg.integrator == ALS_INT_FORWARD_EULER) {
        for (const SolverLevel& L : s->levels) {
            cudaError_t err;
            if (prec == ALS_FP64) {
                err = dim == 1 ? launch_fe_update<double, 3>(s, L)
                    : (dim == 2 ? launch_fe_update<double, 4>(s, L) : launch_fe_update<double, 5>(s, L));
            } else {
                err = dim == 1 ? launch_fe_update<float, 3>(s, L)
                    : (dim == 2 ? launch_fe_update<float, 4>(s, L) : launch_fe_update<float, 5>(s, L));
            }
            ALS_CUDA(err);
        }
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
    } else if (s->cfg.integrator == ALS_INT_RK2) {
        ALS_CUDA(launch_stage_all(s, als::KIND_RK2_1, [s](const SolverLevel& L, const void*& in,
                                                          const void*& un, void*& out) {
            in = L.buf[1];
            un = s->current(L);
            out = s->other(L);
        }));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
        s->cur ^= 1;
    } else {
        ALS_CUDA(launch_stage_all(s, als::KIND_RK3_1, [](const SolverLevel& L, const void*& in,
                                                         const void*& un, void*& out) {
            in = L.buf[1];
            un = L.buf[0];
            out = L.buf[2];
        }));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
        ALS_CUDA(launch_stage_all(s, als::KIND_RK3_2, [](const SolverLevel& L, const void*& in,
                                                         const void*& un, void*& out) {
            in = L.buf[2];
            un = L.buf[0];
            out = L.buf[0];
        }));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[3], s->stream));
        }
    }
    return ALS_OK;
}

template<class R>
int fill_member_ghosts(als_solver* s, const SolverLevel& L, void* base, int first_local,
    int count) {
    dim3 blocks(grid_blocks(als::ghost_shell_cells(s->cfg.dimension, L.grid.n[0], L.grid.n[1],
        L.grid.n[2], s->g), 256), count);
    void* start = static_cast<char*>(base) + size_t(first_local) * L.member_elems * s->elem;
    als::fill_ghosts<R><<<blocks, 256, 0, s->stream>>>(contiguous_planes<R>(start, s->nv, L.grid.plane),
        s->nv, L.grid.plane, L.member_elems, s->cfg.dimension, L.grid.n[0], L.grid.n[1],
        L.grid.n[2], s->g, s->cfg.boundary);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int reset_members(als_solver* s, int first, int count) {
    for (int m = first; m < first + count; ++m) {
        const SolverLevel& L = s->levels[s->level_of(m)];
        als::StepState& st = s->host_state[m];
        std::memset(&st, 0, sizeof(st));
        st.end_time = s->cfg.end_time;
        st.cfl = s->cfg.cfl;
        st.max_steps = s->cfg.max_steps > 0 ? s->cfg.max_steps : LLONG_MAX;
        st.done = (0 >= s->cfg.end_time) ? 1 : 0;
        st.bad_index = -1;  // as unsigned: the largest value, lowered by atomicMin
        st.bad_step = -1;
        for (int d = 0; d < 3; ++d) {
            st.dx[d] = L.dx[d];
        }
    }
    ALS_CUDA(cudaMemcpyAsync(s->state + first, s->host_state + first,
        sizeof(als::StepState) * count, cudaMemcpyHostToDevice, s->stream));
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int refresh_host_state(als_solver* s) {
    ALS_CUDA(cudaMemcpyAsync(s->host_state, s->state, sizeof(als::StepState) * s->members,
        cudaMemcpyDeviceToHost, s->stream));
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    // subdomains advance on member 0's state: every member reports it
    for (int m = 1; s->subdomains && m < s->members; ++m) {
        s->host_state[m] = s->host_state[0];
    }
    return ALS_OK;
}

void drop_graph(als_solver* s) {
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
}

// Whether the stage kernels of this solver's configuration are built with
// tile shape `shape`.
bool shape_available(const als_solver* s, int shape) {
    return shape >= 0 && shape < als::kMaxShapes &&
        als::shape_built(s->cfg.dimension, s->cfg.reconstruction, s->cfg.flux, shape);
}

// Gives level l tile shape shapes[l] (available shapes only) and recovers
// its tiles; the captured step graph no longer matches.
void set_level_shapes(als_solver* s, const int* shapes) {
    for (size_t l = 0; l < s->levels.size(); ++l) {
        SolverLevel& L = s->levels[l];
        L.shape = shapes[l];
        int lo[3] = {0, 0, 0};
        L.grid = make_grid(s->cfg.dimension, L.grid.n, s->g, lo, L.grid.n, s->cfg.precision,
            L.shape);
    }
    drop_graph(s);
}

// members [first, first+count) must lie in one level; returns it or -1
int range_level(const als_solver* s, int first, int count) {
    if (first < 0 || count < 1 || first + count > s->members) {
        return -1;
    }
    const int l = s->level_of(first);
    const SolverLevel& L = s->levels[l];
    return first + count <= L.first + L.cfg.members ? l : -1;
}

int check_config(const als_solver_config* cfg) {
    if (cfg->integrator == ALS_INT_RK4) {
        return fail(ALS_E_UNSUPPORTED,
            "RK4 runs through the plug-in integrator (als_integrator_combine, als_integrator_combine_rk4)");
    }
    if (cfg->dimension < 1 || cfg->dimension > 3 || !valid_choice(cfg->flux, cfg->reconstruction) ||
        cfg->integrator < ALS_INT_FORWARD_EULER || cfg->integrator > ALS_INT_RK3 ||
        (cfg->boundary != ALS_BC_NEUMANN && cfg->boundary != ALS_BC_PERIODIC) ||
        (cfg->precision != ALS_FP64 && cfg->precision != ALS_FP32) || cfg->members < 1 ||
        !(cfg->gamma > 1) || !(cfg->cfl > 0)) {
        return fail(ALS_E_INVALID, "invalid solver configuration");
    }
    const int g = als_ghost_cells(cfg->flux, cfg->reconstruction);
    if (g < 0) {
        return g;
    }
    for (int d = 0; d < cfg->dimension; ++d) {
        // ConservedSystem splits the update into an interior and 2*dim side
        // regions of width g (ConservedSystem.cpp:59-96); with fewer than 2g
        // cells those regions reach into the ghost layer, which this solver
        // does not reproduce.
        if (cfg->n[d] < 2 * g) {
            return fail(ALS_E_INVALID, "every active direction needs at least 2*ghosts interior cells");
        }
    }
    return ALS_OK;
}

} // namespace

extern "C" {

int als_solver_create_levels(const als_solver_config* cfgs, int nlevels, int device,
    als_solver** out) {
    if (!cfgs || !out) {
        return fail(ALS_E_INVALID, "null argument");
    }
    *out = nullptr;
    if (nlevels < 1 || nlevels > als::kMaxLevels) {
        return fail(ALS_E_INVALID, "1 to 4 grid levels");
    }
    for (int l = 0; l < nlevels; ++l) {
        int rc = check_config(&cfgs[l]);
        if (rc != ALS_OK) {
            return rc;
        }
        const als_solver_config& a = cfgs[0];
        const als_solver_config& b = cfgs[l];
        if (b.dimension != a.dimension || b.flux != a.flux || b.reconstruction != a.reconstruction ||
            b.integrator != a.integrator || b.boundary != a.boundary || b.precision != a.precision ||
            b.gamma != a.gamma || b.cfl != a.cfl || b.end_time != a.end_time ||
            b.max_steps != a.max_steps) {
            return fail(ALS_E_INVALID, "levels may differ only in grid size, domain and members");
        }
    }
    std::unique_ptr<als_solver> s(new (std::nothrow) als_solver());
    if (!s) {
        return fail(ALS_E_NOMEM, "out of host memory");
    }
    const als_solver_config& cfg = cfgs[0];
    s->cfg = cfg;
    s->device = device;
    s->g = als_ghost_cells(cfg.flux, cfg.reconstruction);
    s->nv = cfg.dimension + 2;
    s->elem = cfg.precision == ALS_FP64 ? 8 : 4;
    DeviceGuard guard(device);
    ALS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    int first = 0;
    for (int l = 0; l < nlevels; ++l) {
        SolverLevel L;
        L.cfg = cfgs[l];
        int lo[3] = {0, 0, 0};
        int n[3];
        for (int d = 0; d < 3; ++d) {
            n[d] = d < cfg.dimension ? cfgs[l].n[d] : 1;
        }
        // 3-D levels start on the z-marching columns where they are built
        // (measured faster than the boxes on KH 128^3); the tuner may change it
        L.shape = cfg.dimension == 3 &&
            als::shape_built(3, cfg.reconstruction, cfg.flux, 1) ? 1 : 0;
        L.grid = make_grid(cfg.dimension, n, s->g, lo, n, cfg.precision, L.shape);
        L.member_elems = (long long)s->nv * L.grid.plane;
        L.first = first;
        first += cfgs[l].members;
        for (int d = 0; d < 3; ++d) {
            // Grid.cpp:24-41: (top - origin) / n, and 1 for a direction with one cell
            L.dx[d] = (cfgs[l].upper[d] - cfgs[l].lower[d]) / double(n[d]);
            if (d > 0 && n[d] == 1) {
                L.dx[d] = 1;
            }
        }
        const size_t bytes = size_t(L.member_elems) * cfgs[l].members * s->elem;
        for (int b = 0; b < 3; ++b) {
            if (b == 2 && cfg.integrator == ALS_INT_FORWARD_EULER) {
                continue;
            }
            ALS_CUDA(cudaMalloc(&L.buf[b], bytes));
            ALS_CUDA(cudaMemset(L.buf[b], 0, bytes));
        }
        s->levels.push_back(L);
    }
    s->members = first;
    s->order.resize(nlevels);
    std::iota(s->order.begin(), s->order.end(), 0);
    ALS_CUDA(cudaMalloc((void**)&s->state, sizeof(als::StepState) * s->members));
    ALS_CUDA(cudaMalloc((void**)&s->counter, 2 * sizeof(unsigned long long)));
    ALS_CUDA(cudaMemset(s->counter, 0, 2 * sizeof(unsigned long long)));
    ALS_CUDA(cudaMallocHost((void**)&s->host_state, sizeof(als::StepState) * s->members));
    int rc = reset_members(s.get(), 0, s->members);
    if (rc != ALS_OK) {
        return rc;
    }
    *out = s.release();
    return ALS_OK;
}

int als_solver_create(const als_solver_config* cfg, int device, als_solver** out) {
    return als_solver_create_levels(cfg, 1, device, out);
}

int als_solver_decompose(als_solver* s, const int* procs) {
    if (!s || !procs) {
        return fail(ALS_E_INVALID, "null argument");
    }
    if (s->levels.size() != 1) {
        return fail(ALS_E_INVALID, "a split grid is a solver of one level");
    }
    if (s->cfg.integrator != ALS_INT_RK2 && s->cfg.integrator != ALS_INT_RK3) {
        return fail(ALS_E_UNSUPPORTED, "split grids advance with rungekutta2 or rungekutta3");
    }
    long long count = 1;
    for (int d = 0; d < 3; ++d) {
        if (procs[d] < 1 || (d >= s->cfg.dimension && procs[d] != 1)) {
            return fail(ALS_E_INVALID, "one or more subdomains per active direction, one per inactive");
        }
        count *= procs[d];
    }
    if (count != s->members) {
        return fail(ALS_E_INVALID, "the solver needs one member per subdomain");
    }
    drop_graph(s);
    s->subdomains = 1;
    for (int d = 0; d < 3; ++d) {
        s->procs[d] = procs[d];
    }
    // a state set before the split has its ghosts filled by the boundary
    // condition, not from the neighbouring subdomains: a new state is due
    s->needs_state = true;
    return ALS_OK;
}

int als_solver_destroy(als_solver* s) {
    delete s;
    return ALS_OK;
}

int als_solver_geometry(const als_solver* s, long long* plane, int* ghosts) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    if (plane) {
        *plane = s->levels[0].grid.plane;
    }
    if (ghosts) {
        *ghosts = s->g;
    }
    return ALS_OK;
}

int als_solver_level(const als_solver* s, int level, int* first_member, int* members,
    long long* plane) {
    if (!s || level < 0 || level >= int(s->levels.size())) {
        return fail(ALS_E_INVALID, "invalid level");
    }
    const SolverLevel& L = s->levels[level];
    if (first_member) {
        *first_member = L.first;
    }
    if (members) {
        *members = L.cfg.members;
    }
    if (plane) {
        *plane = L.grid.plane;
    }
    return ALS_OK;
}

// A split grid's subdomains share member 0's clock and read each other's
// cells as ghosts, so its state is set whole, in one call.
static int check_split_state(const als_solver* s, int first_member, int count) {
    if (s->subdomains && (first_member != 0 || count != s->members)) {
        return fail(ALS_E_INVALID, "a split grid takes the state of all its subdomains in one call");
    }
    return ALS_OK;
}

int als_solver_set_state(als_solver* s, const double* host, int first_member, int count) {
    const int l = s ? range_level(s, first_member, count) : -1;
    if (!s || !host || l < 0) {
        return fail(ALS_E_INVALID, "invalid set_state arguments (members must lie in one level)");
    }
    int split_rc = check_split_state(s, first_member, count);
    if (split_rc != ALS_OK) {
        return split_rc;
    }
    DeviceGuard guard(s->device);
    const SolverLevel& L = s->levels[l];
    const int local = first_member - L.first;
    const size_t n = size_t(L.member_elems) * count;
    s->cur = 0;
    if (s->cfg.precision == ALS_FP64) {
        ALS_CUDA(cudaMemcpyAsync(static_cast<double*>(L.buf[0]) + (long long)local * L.member_elems,
            host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        // subdomains come with their ghosts (their blocks of the whole padded grid)
        int rc = s->subdomains ? ALS_OK : fill_member_ghosts<double>(s, L, L.buf[0], local, count);
        if (rc != ALS_OK) {
            return rc;
        }
    } else {
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) {
            tmp[i] = float(host[i]);
        }
        ALS_CUDA(cudaMemcpyAsync(static_cast<float*>(L.buf[0]) + (long long)local * L.member_elems,
            tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        int rc = s->subdomains ? ALS_OK : fill_member_ghosts<float>(s, L, L.buf[0], local, count);
        if (rc != ALS_OK) {
            return rc;
        }
        ALS_CUDA(cudaStreamSynchronize(s->stream));
    }
    s->needs_state = false;
    return reset_members(s, first_member, count);
}

int als_solver_set_state_device(als_solver* s, const void* dev, int first_member, int count) {
    const int l = s ? range_level(s, first_member, count) : -1;
    if (!s || !dev || l < 0) {
        return fail(ALS_E_INVALID, "invalid set_state_device arguments (members must lie in one level)");
    }
    int split_rc = check_split_state(s, first_member, count);
    if (split_rc != ALS_OK) {
        return split_rc;
    }
    DeviceGuard guard(s->device);
    const SolverLevel& L = s->levels[l];
    const int local = first_member - L.first;
    s->cur = 0;
    const size_t bytes = size_t(L.member_elems) * count * s->elem;
    ALS_CUDA(cudaMemcpyAsync(static_cast<char*>(L.buf[0]) + size_t(local) * L.member_elems * s->elem,
        dev, bytes, cudaMemcpyDeviceToDevice, s->stream));
    int rc = s->subdomains ? ALS_OK
        : (s->cfg.precision == ALS_FP64 ? fill_member_ghosts<double>(s, L, L.buf[0], local, count)
                                        : fill_member_ghosts<float>(s, L, L.buf[0], local, count));
    if (rc != ALS_OK) {
        return rc;
    }
    s->needs_state = false;
    return reset_members(s, first_member, count);
}

// Device address of member m's current state (RK2: by its own step parity).
static const char* member_state_address(als_solver* s, int m) {
    const SolverLevel& L = s->levels[s->level_of(m)];
    const void* base = L.buf[0];
    if (s->cfg.integrator == ALS_INT_RK2 && (s->host_state[m].steps & 1)) {
        base = L.buf[2];
    }
    return static_cast<const char*>(base) + size_t(m - L.first) * L.member_elems * s->elem;
}

int als_solver_get_state(als_solver* s, double* host, int first_member, int count) {
    const int l = s ? range_level(s, first_member, count) : -1;
    if (!s || !host || l < 0) {
        return fail(ALS_E_INVALID, "invalid get_state arguments (members must lie in one level)");
    }
    DeviceGuard guard(s->device);
    int rc = refresh_host_state(s);
    if (rc != ALS_OK) {
        return rc;
    }
    const size_t n = size_t(s->levels[l].member_elems);
    std::vector<float> tmp(s->cfg.precision == ALS_FP64 ? 0 : n);
    for (int m = first_member; m < first_member + count; ++m) {
        const char* src = member_state_address(s, m);
        double* dst = host + size_t(m - first_member) * n;
        if (s->cfg.precision == ALS_FP64) {
            ALS_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
            ALS_CUDA(cudaStreamSynchronize(s->stream));
        } else {
            ALS_CUDA(cudaMemcpyAsync(tmp.data(), src, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
            ALS_CUDA(cudaStreamSynchronize(s->stream));
            for (size_t i = 0; i < n; ++i) {
                dst[i] = double(tmp[i]);
            }
        }
    }
    return ALS_OK;
}

int als_solver_write_netcdf(als_solver* s, int member, const char* basename, int snapshot) {
    const int l = s ? range_level(s, member, 1) : -1;
    if (!s || l < 0 || !basename || snapshot < 0) {
        return fail(ALS_E_INVALID, "invalid write_netcdf arguments");
    }
    const SolverLevel& L = s->levels[l];
    const int dim = s->cfg.dimension;
    std::vector<double> padded(size_t(L.member_elems));
    int rc = als_solver_get_state(s, padded.data(), member, 1);
    if (rc != ALS_OK) {
        return rc;
    }
    als_member_info info;
    rc = als_solver_info(s, member, &info);
    if (rc != ALS_OK) {
        return rc;
    }
    // Volume::copyInternalCells (HostMemory.cpp:239-258): interior, x fastest
    const int* n = L.grid.n;
    const int* N = L.grid.N;
    const int G[3] = {s->g, dim > 1 ? s->g : 0, dim > 2 ? s->g : 0};
    const size_t cells = size_t(n[0]) * n[1] * n[2];
    std::vector<std::vector<double>> interior(size_t(s->nv), std::vector<double>(cells));
    for (int v = 0; v < s->nv; ++v) {
        const double* plane = padded.data() + size_t(v) * size_t(L.grid.plane);
        size_t k = 0;
        for (int z = 0; z < n[2]; ++z) {
            for (int y = 0; y < n[1]; ++y) {
                for (int x = 0; x < n[0]; ++x) {
                    interior[size_t(v)][k++] =
                        plane[(size_t(z + G[2]) * N[1] + size_t(y + G[1])) * N[0] + size_t(x + G[0])];
                }
            }
        }
    }
    // Euler<d>::conservedVariables (alsfvm/src/equation/euler/Euler.cpp:20-75)
    static const char* const names1[] = {"rho", "mx", "E"};
    static const char* const names2[] = {"rho", "mx", "my", "E"};
    static const char* const names3[] = {"rho", "mx", "my", "mz", "E"};
    const char* const* names = dim == 1 ? names1 : (dim == 2 ? names2 : names3);
    std::vector<const double*> ptrs;
    for (const auto& v : interior) {
        ptrs.push_back(v.data());
    }
    const std::string steps = std::to_string(info.steps);
    const std::string prec = s->cfg.precision == ALS_FP64 ? "fp64" : "fp32";
    const char* anames[] = {"alsvinn_b200.software", "alsvinn_b200.steps", "alsvinn_b200.precision"};
    const char* avalues[] = {"alsvinn_b200", steps.c_str(), prec.c_str()};
    // io_utils.cpp:34-40 and NetCDFWriter.cpp:139-146: <base>_<snapshot>.nc
    const std::string path = std::string(basename) + "_" + std::to_string(snapshot) + ".nc";
    int nn[3] = {n[0], n[1], n[2]};
    return als_write_netcdf(path.c_str(), dim, nn, s->nv, names, ptrs.data(), info.t, 3, anames,
        avalues);
}

int als_solver_state_pointer(als_solver* s, void** dev) {
    if (!s || !dev) {
        return fail(ALS_E_INVALID, "null argument");
    }
    *dev = s->current(s->levels[0]);
    return ALS_OK;
}

int als_solver_advance(als_solver* s, long long steps) {
    if (!s || steps < 0) {
        return fail(ALS_E_INVALID, "invalid advance arguments");
    }
    if (s->needs_state) {
        return fail(ALS_E_INVALID, "set the state of the split grid after als_solver_decompose");
    }
    DeviceGuard guard(s->device);
    // whole time steps are captured once into a CUDA graph and replayed; the
    // RK2 ping-pong needs an even number of steps per graph
    const int per_graph = 8;
    if (steps >= per_graph && !s->graph) {
        cudaGraph_t g = nullptr;
        const int cur0 = s->cur;
        ALS_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        int rc = ALS_OK;
        for (int k = 0; k < per_graph && rc == ALS_OK; ++k) {
            rc = enqueue_step(s);
        }
        cudaError_t err = cudaStreamEndCapture(s->stream, &g);
        s->cur = cur0;
        if (rc != ALS_OK) {
            if (g) {
                cudaGraphDestroy(g);
            }
            return rc;
        }
        ALS_CUDA(err);
        err = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        ALS_CUDA(err);
        s->graph_steps = per_graph;
        s->graph_cur = cur0;
    }
    long long left = steps;
    if (s->graph && s->cur != s->graph_cur && left > 0) {
        int rc = enqueue_step(s);
        if (rc != ALS_OK) {
            return rc;
        }
        --left;
    }
    while (s->graph && s->cur == s->graph_cur && left >= s->graph_steps) {
        ALS_CUDA(cudaGraphLaunch(s->graph, s->stream));
        left -= s->graph_steps;
    }
    while (left > 0) {
        int rc = enqueue_step(s);
        if (rc != ALS_OK) {
            return rc;
        }
        --left;
    }
    return ALS_OK;
}

int als_solver_synchronize(als_solver* s) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    DeviceGuard guard(s->device);
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int als_solver_run(als_solver* s) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    DeviceGuard guard(s->device);
    long long chunk = 16;
    double progress_prev = -1.0;
    for (;;) {
        int rc = refresh_host_state(s);
        if (rc != ALS_OK) {
            return rc;
        }
        bool all_done = true;
        bool failed = false;
        double remaining_steps = 0;
        double progress = 0.0;  // sum of member times: must grow while any member is running
        for (int m = 0; m < s->members; ++m) {
            const als::StepState& st = s->host_state[m];
            progress += st.t;
            failed = failed || st.status != 0;
            if (!st.done) {
                all_done = false;
                if (st.dt > 0) {
                    remaining_steps = std::max(remaining_steps, (st.end_time - st.t) / st.dt);
                }
            }
        }
        if (all_done) {
            return failed ? fail(ALS_E_CONSTRAINT, "simulation state does not obey the constraints")
                          : ALS_OK;
        }
        if (progress == progress_prev) {
            return fail(ALS_E_INVALID, "no member advanced (zero or non-finite time step)");
        }
        progress_prev = progress;
        // launch about the remaining number of steps; members that finish
        // early skip the surplus steps on the device
        if (remaining_steps > 0) {
            chunk = (long long)std::min(remaining_steps * 1.05 + 8, 65536.0);
        }
        rc = als_solver_advance(s, chunk);
        if (rc != ALS_OK) {
            return rc;
        }
    }
}

int als_solver_info(als_solver* s, int member, als_member_info* info) {
    if (!s || !info || member < 0 || member >= s->members) {
        return fail(ALS_E_INVALID, "invalid info arguments");
    }
    DeviceGuard guard(s->device);
    int rc = refresh_host_state(s);
    if (rc != ALS_OK) {
        return rc;
    }
    const als::StepState& st = s->host_state[member];
    info->t = st.t;
    info->dt = st.dt;
    info->steps = st.steps;
    info->done = st.done;
    info->status = st.status;
    info->bad_index = st.status ? st.bad_index : -1;
    info->bad_step = st.bad_step;
    return ALS_OK;
}

void* als_solver_stream(als_solver* s) {
    return s ? (void*)s->stream : nullptr;
}

int als_solver_launches_per_step(const als_solver* s) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    if (s->cfg.integrator == ALS_INT_RK3) {
        return 3;
    }
    if (s->cfg.integrator == ALS_INT_RK2) {
        return 2;
    }
    return 1 + int(s->levels.size());
}

int als_solver_profile_step(als_solver* s, float* kernel_ms, int capacity) {
    if (!s || !kernel_ms) {
        return fail(ALS_E_INVALID, "null argument");
    }
    // events sit between the stages: FE counts its per-level updates as one
    const int k = s->cfg.integrator == ALS_INT_RK3 ? 3 : 2;
    if (capacity < k) {
        return fail(ALS_E_INVALID, "capacity below the stages per step");
    }
    DeviceGuard guard(s->device);
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int rc = ALS_OK;
    for (int i = 0; i <= 3 && rc == ALS_OK; ++i) {
        if (cudaEventCreate(&ev[i]) != cudaSuccess) {
            rc = fail(ALS_E_CUDA, "cudaEventCreate failed");
        }
    }
    if (rc == ALS_OK) {
        rc = enqueue_step(s, ev);
    }
    if (rc == ALS_OK && cudaEventSynchronize(ev[k]) != cudaSuccess) {
        rc = fail(ALS_E_CUDA, "cudaEventSynchronize failed");
    }
    for (int i = 0; i < k && rc == ALS_OK; ++i) {
        if (cudaEventElapsedTime(&kernel_ms[i], ev[i], ev[i + 1]) != cudaSuccess) {
            rc = fail(ALS_E_CUDA, "cudaEventElapsedTime failed");
        }
    }
    for (int i = 0; i <= 3; ++i) {
        if (ev[i]) {
            cudaEventDestroy(ev[i]);
        }
    }
    return rc == ALS_OK ? k : rc;
}

int als_solver_set_schedule(als_solver* s, int blocks_per_sm, const int* level_order) {
    if (!s || blocks_per_sm < 0) {
        return fail(ALS_E_INVALID, "invalid schedule");
    }
    std::vector<int> order(s->levels.size());
    if (level_order) {
        std::vector<int> seen(s->levels.size(), 0);
        for (size_t k = 0; k < order.size(); ++k) {
            const int l = level_order[k];
            if (l < 0 || l >= int(order.size()) || seen[l]) {
                return fail(ALS_E_INVALID, "level order must be a permutation of the levels");
            }
            seen[l] = 1;
            order[k] = l;
        }
    } else {
        std::iota(order.begin(), order.end(), 0);
    }
    DeviceGuard guard(s->device);
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    s->blocks_per_sm = blocks_per_sm;
    s->order = order;
    drop_graph(s);
    return ALS_OK;
}

int als_solver_get_schedule(const als_solver* s, int* blocks_per_sm, int* level_order) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    if (blocks_per_sm) {
        *blocks_per_sm = s->blocks_per_sm;
    }
    if (level_order) {
        for (size_t k = 0; k < s->order.size(); ++k) {
            level_order[k] = s->order[k];
        }
    }
    return ALS_OK;
}

int als_solver_set_tiles(als_solver* s, const int* tile_shapes) {
    if (!s || !tile_shapes) {
        return fail(ALS_E_INVALID, "null argument");
    }
    for (size_t l = 0; l < s->levels.size(); ++l) {
        if (!shape_available(s, tile_shapes[l])) {
            return fail(ALS_E_UNSUPPORTED, "tile shape " + std::to_string(tile_shapes[l]) +
                " is not built for this dimension, reconstruction and flux");
        }
    }
    DeviceGuard guard(s->device);
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    set_level_shapes(s, tile_shapes);
    return ALS_OK;
}

int als_solver_get_tiles(const als_solver* s, int* tile_shapes, int* tile_extents) {
    if (!s) {
        return fail(ALS_E_INVALID, "null solver");
    }
    for (size_t l = 0; l < s->levels.size(); ++l) {
        const SolverLevel& L = s->levels[l];
        if (tile_shapes) {
            tile_shapes[l] = L.shape;
        }
        if (tile_extents) {
            for (int d = 0; d < 3; ++d) {
                tile_extents[3 * l + d] = tile_extent(s->cfg.precision, s->cfg.dimension, d, L.shape);
            }
        }
    }
    return ALS_OK;
}

// The schedule autotuner: times `steps` time steps per candidate from the
// same saved state, keeps the fastest, and restores the state and member
// clocks, so tuning changes no result.  First the tile shape of each level
// (coordinate search: one level's shape varied at a time, the others at
// their best so far), then persistent blocks per SM x level order.
int als_solver_tune(als_solver* s, int steps, int* blocks_per_sm, int* level_order,
    int* tile_shapes, double* best_ms_per_step) {
    if (!s || steps < 1) {
        return fail(ALS_E_INVALID, "invalid tune arguments");
    }
    DeviceGuard guard(s->device);
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    // save the state buffer of every level (the flux and stage buffers are
    // rewritten before they are read in every step) and the member clocks;
    // the copies are freed on every return path
    struct Saved {
        std::vector<void*> p;
        ~Saved() {
            for (void* q : p) {
                cudaFree(q);
            }
        }
    } saved;
    for (SolverLevel& L : s->levels) {
        const size_t bytes = size_t(L.member_elems) * L.cfg.members * s->elem;
        void* p = nullptr;
        ALS_CUDA(cudaMalloc(&p, bytes));
        saved.p.push_back(p);
        ALS_CUDA(cudaMemcpyAsync(p, s->current(L), bytes, cudaMemcpyDeviceToDevice, s->stream));
    }
    void* state_copy = nullptr;
    ALS_CUDA(cudaMalloc(&state_copy, sizeof(als::StepState) * s->members));
    saved.p.push_back(state_copy);
    als::StepState* saved_state = static_cast<als::StepState*>(state_copy);
    ALS_CUDA(cudaMemcpyAsync(saved_state, s->state, sizeof(als::StepState) * s->members,
        cudaMemcpyDeviceToDevice, s->stream));
    const int cur0 = s->cur;
    const int bps0 = s->blocks_per_sm;
    const std::vector<int> order0 = s->order;
    std::vector<int> shapes0;
    for (const SolverLevel& L : s->levels) {
        shapes0.push_back(L.shape);
    }

    auto restore = [&]() -> int {
        s->cur = cur0;
        size_t k = 0;
        for (SolverLevel& L : s->levels) {
            const size_t bytes = size_t(L.member_elems) * L.cfg.members * s->elem;
            ALS_CUDA(cudaMemcpyAsync(s->current(L), saved.p[k++], bytes, cudaMemcpyDeviceToDevice,
                s->stream));
        }
        ALS_CUDA(cudaMemcpyAsync(s->state, saved_state, sizeof(als::StepState) * s->members,
            cudaMemcpyDeviceToDevice, s->stream));
        return ALS_OK;
    };

    // candidate level orders: as given, finest first, coarsest first
    std::vector<std::vector<int>> orders;
    orders.push_back(order0);
    std::vector<int> by_cells(s->levels.size());
    std::iota(by_cells.begin(), by_cells.end(), 0);
    std::stable_sort(by_cells.begin(), by_cells.end(), [s](int a, int b) {
        return s->levels[a].grid.plane > s->levels[b].grid.plane;
    });
    orders.push_back(by_cells);
    std::reverse(by_cells.begin(), by_cells.end());
    orders.push_back(by_cells);
    std::sort(orders.begin(), orders.end());
    orders.erase(std::unique(orders.begin(), orders.end()), orders.end());
    // 0: one block per work item; k > 0: persistent, k resident blocks per SM
    const int bps_candidates[] = {0, 1, 2, 3, 4};

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ALS_CUDA(cudaEventCreate(&e0));
    ALS_CUDA(cudaEventCreate(&e1));
    int rc = ALS_OK;
    // ms per step of the current shapes, order and blocks per SM (1e300 after an error)
    auto time_steps = [&]() -> double {
        if (rc != ALS_OK) {
            return 1e300;
        }
        rc = restore();
        // one untimed step, then the timed ones
        for (int k = 0; k < 1 + steps && rc == ALS_OK; ++k) {
            if (k == 1 && cudaEventRecord(e0, s->stream) != cudaSuccess) {
                rc = fail(ALS_E_CUDA, "cudaEventRecord failed");
            }
            if (rc == ALS_OK) {
                rc = enqueue_step(s);
            }
        }
        if (rc == ALS_OK && (cudaEventRecord(e1, s->stream) != cudaSuccess ||
                                cudaEventSynchronize(e1) != cudaSuccess)) {
            rc = fail(ALS_E_CUDA, "timing failed");
        }
        float ms = 0;
        if (rc == ALS_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = fail(ALS_E_CUDA, "cudaEventElapsedTime failed");
        }
        return rc == ALS_OK ? double(ms) / steps : 1e300;
    };
    std::vector<int> best_shapes = shapes0;
    s->order = order0;
    s->blocks_per_sm = bps0;
    double best = time_steps();
    for (size_t l = 0; l < s->levels.size() && rc == ALS_OK; ++l) {
        for (int shape = 0; shape < als::kMaxShapes && rc == ALS_OK; ++shape) {
            if (shape == best_shapes[l] || !shape_available(s, shape)) {
                continue;
            }
            std::vector<int> trial = best_shapes;
            trial[l] = shape;
            set_level_shapes(s, trial.data());
            const double ms = time_steps();
            if (ms < best) {
                best = ms;
                best_shapes = trial;
            }
        }
    }
    set_level_shapes(s, best_shapes.data());
    int best_bps = bps0;
    std::vector<int> best_order = order0;
    for (const std::vector<int>& ord : orders) {
        for (int bps : bps_candidates) {
            if (rc != ALS_OK) {
                break;
            }
            if (ord == order0 && bps == bps0) {
                continue;
            }
            s->order = ord;
            s->blocks_per_sm = bps;
            const double ms = time_steps();
            if (ms < best) {
                best = ms;
                best_bps = bps;
                best_order = ord;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->order = best_order;
    s->blocks_per_sm = best_bps;
    int rc2 = restore();
    cudaStreamSynchronize(s->stream);
    drop_graph(s);
    if (rc != ALS_OK) {
        return rc;
    }
    if (rc2 != ALS_OK) {
        return rc2;
    }
    if (blocks_per_sm) {
        *blocks_per_sm = best_bps;
    }
    if (level_order) {
        for (size_t k = 0; k < best_order.size(); ++k) {
            level_order[k] = best_order[k];
        }
    }
    if (tile_shapes) {
        for (size_t k = 0; k < best_shapes.size(); ++k) {
            tile_shapes[k] = best_shapes[k];
        }
    }
    if (best_ms_per_step) {
        *best_ms_per_step = best;
    }
    return ALS_OK;
}

// FP64 sums of every conserved variable over the interior box [lo, hi)
// (interior cell coordinates, NULL = whole interior) of members
// [first, first+count) of one level: out[k*nvar + v].
int als_solver_region_sums(als_solver* s, int first_member, int count, const int* lo,
    const int* hi, double* out) {
    const int l = s ? range_level(s, first_member, count) : -1;
    if (!s || !out || l < 0) {
        return fail(ALS_E_INVALID, "invalid region_sums arguments (members must lie in one level)");
    }
    const SolverLevel& L = s->levels[l];
    int plo[3], phi[3];
    for (int d = 0; d < 3; ++d) {
        const bool active = d < s->cfg.dimension;
        const int n = L.grid.n[d];
        const int a = lo && active ? lo[d] : 0;
        const int b = hi && active ? hi[d] : n;
        if (active && (a < 0 || b > n || a >= b)) {
            return fail(ALS_E_INVALID, "region must lie inside the interior");
        }
        plo[d] = active ? a + s->g : 0;
        phi[d] = active ? b + s->g : 1;
    }
    DeviceGuard guard(s->device);
    int rc = refresh_host_state(s);
    if (rc != ALS_OK) {
        return rc;
    }
    double* dev = nullptr;
    ALS_CUDA(als::scratch_alloc((void**)&dev, sizeof(double) * s->nv * count, s->stream));
    for (int m = first_member; m < first_member + count; ++m) {
        const void* base = member_state_address(s, m);
        cudaError_t err;
        if (s->cfg.precision == ALS_FP64) {
            als::region_sums<double><<<1, 256, 0, s->stream>>>(static_cast<const double*>(base),
                L.grid.plane, 0, s->nv, L.grid.N[0], L.grid.N[1], plo[0], plo[1], plo[2], phi[0],
                phi[1], phi[2], dev + (m - first_member) * s->nv);
        } else {
            als::region_sums<float><<<1, 256, 0, s->stream>>>(static_cast<const float*>(base),
                L.grid.plane, 0, s->nv, L.grid.N[0], L.grid.N[1], plo[0], plo[1], plo[2], phi[0],
                phi[1], phi[2], dev + (m - first_member) * s->nv);
        }
        err = cudaGetLastError();
        if (err != cudaSuccess) {
            als::scratch_free(dev, s->stream);
            return fail(ALS_E_CUDA, std::string("region_sums: ") + cudaGetErrorString(err));
        }
    }
    ALS_CUDA(cudaMemcpyAsync(out, dev, sizeof(double) * s->nv * count, cudaMemcpyDeviceToHost, s->stream));
    ALS_CUDA(als::scratch_free(dev, s->stream));
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

} // extern "C"

// -------------------------------------------------------------- statistics

struct als_stats {
    int device = 0;
    long long count = 0;          // elements per state
    long long n = 0;              // states accumulated
    double* mean = nullptr;
    double* m2 = nullptr;
    ~als_stats() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (mean) {
            cudaFree(mean);
        }
        if (m2) {
            cudaFree(m2);
        }
        cudaSetDevice(prev);
    }
};

namespace {

template<class R>
int stats_merge_states(als_stats* st, const R* states, int members, long long member_stride,
    cudaStream_t s) {
    // chunks of at most 64 states keep each chunk's two passes in L2
    for (int first = 0; first < members; first += 64) {
        const int k = std::min(64, members - first);
        als::welford_merge<R><<<grid_blocks(st->count, 256), 256, 0, s>>>(
            states + (long long)first * member_stride, st->count, k, member_stride, st->mean, st->m2,
            st->n);
        ALS_CUDA(cudaGetLastError());
        st->n += k;
    }
    return ALS_OK;
}

} // namespace

extern "C" {

int als_stats_create(long long count, int device, als_stats** out) {
    if (!out || count < 1) {
        return fail(ALS_E_INVALID, "invalid stats arguments");
    }
    *out = nullptr;
    std::unique_ptr<als_stats> st(new (std::nothrow) als_stats());
    if (!st) {
        return fail(ALS_E_NOMEM, "out of host memory");
    }
    st->device = device;
    st->count = count;
    DeviceGuard guard(device);
    ALS_CUDA(cudaMalloc((void**)&st->mean, sizeof(double) * count));
    ALS_CUDA(cudaMalloc((void**)&st->m2, sizeof(double) * count));
    ALS_CUDA(cudaMemset(st->mean, 0, sizeof(double) * count));
    ALS_CUDA(cudaMemset(st->m2, 0, sizeof(double) * count));
    *out = st.release();
    return ALS_OK;
}

int als_stats_destroy(als_stats* st) {
    delete st;
    return ALS_OK;
}

int als_stats_add(als_stats* st, const void* states, int precision, int members,
    long long member_stride, void* stream) {
    if (!st || !states || members < 1 || member_stride < st->count ||
        (precision != ALS_FP64 && precision != ALS_FP32)) {
        return fail(ALS_E_INVALID, "invalid stats_add arguments");
    }
    DeviceGuard guard(st->device);
    return precision == ALS_FP64
        ? stats_merge_states(st, static_cast<const double*>(states), members, member_stride, (cudaStream_t)stream)
        : stats_merge_states(st, static_cast<const float*>(states), members, member_stride, (cudaStream_t)stream);
}

int als_stats_add_solver(als_stats* st, als_solver* s, int level) {
    if (!st || !s || level < 0 || level >= int(s->levels.size())) {
        return fail(ALS_E_INVALID, "invalid stats_add_solver arguments");
    }
    const SolverLevel& L = s->levels[level];
    if (L.member_elems != st->count) {
        return fail(ALS_E_INVALID, "statistics size differs from the level's state size");
    }
    DeviceGuard guard(s->device);
    int rc = refresh_host_state(s);
    if (rc != ALS_OK) {
        return rc;
    }
    // RK2 members may sit in either buffer: add them one by one then
    if (s->cfg.integrator == ALS_INT_RK2) {
        for (int m = L.first; m < L.first + L.cfg.members; ++m) {
            rc = als_stats_add(st, member_state_address(s, m), s->cfg.precision, 1, L.member_elems,
                s->stream);
            if (rc != ALS_OK) {
                return rc;
            }
        }
    } else {
        rc = als_stats_add(st, L.buf[0], s->cfg.precision, L.cfg.members, L.member_elems, s->stream);
        if (rc != ALS_OK) {
            return rc;
        }
    }
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int als_stats_merge(als_stats* st, long long n, const double* mean, const double* m2, void* stream) {
    if (!st || n < 0 || (n > 0 && (!mean || !m2))) {
        return fail(ALS_E_INVALID, "invalid stats_merge arguments");
    }
    if (n == 0) {
        return ALS_OK;
    }
    DeviceGuard guard(st->device);
    als::welford_combine<<<grid_blocks(st->count, 256), 256, 0, (cudaStream_t)stream>>>(
        st->mean, st->m2, st->n, mean, m2, n, st->count);
    ALS_CUDA(cudaGetLastError());
    st->n += n;
    return ALS_OK;
}

int als_stats_moments(als_stats* st, long long* n, double** mean, double** m2) {
    if (!st) {
        return fail(ALS_E_INVALID, "null stats");
    }
    if (n) {
        *n = st->n;
    }
    if (mean) {
        *mean = st->mean;
    }
    if (m2) {
        *m2 = st->m2;
    }
    return ALS_OK;
}

int als_stats_result(als_stats* st, double* mean, double* variance, void* stream) {
    if (!st || st->n < 1) {
        return fail(ALS_E_INVALID, "no states accumulated");
    }
    DeviceGuard guard(st->device);
    als::welford_finish<<<grid_blocks(st->count, 256), 256, 0, (cudaStream_t)stream>>>(
        st->mean, st->m2, st->n, st->count, mean, variance);
    ALS_CUDA(cudaGetLastError());
    ALS_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return ALS_OK;
}

} // extern "C"

// ------------------------------------------- allocation-free flux evaluation
//
// als_compute_flux allocates its three wave-speed accumulators once per
// host thread and device (cudaMalloc on first use) and keeps them.  Some
// hosts of NumericalFlux::computeFlux cannot let a library allocate device
// memory at all: a runtime that plans every byte of device
// memory up front (a memory pool owned by another framework, a fixed-budget
// embedded or real-time deployment), or one that forbids allocation calls
// while it drives the flux evaluation many times per time step.  For them,
// als_compute_flux_static keeps those accumulators in the fixed array below
// and allocates nothing.

namespace {

// at most this many states per call; 3 accumulators each: 24 KiB
constexpr int kStaticFluxMembers = 1024;
// every GPU that loads the library holds this array until the process exits
static __device__ __align__(256) unsigned long long g_static_flux_wave_speeds[3 * kStaticFluxMembers];

std::mutex g_static_flux_mutex;
void* g_static_flux_address[256] = {};
// one caller at a time per device uses the array (clear, kernel, read-back)
std::mutex g_static_flux_calls[256];

// Device address of the array on the current device, looked up once per
// device (cudaGetSymbolAddress; the name itself is a host-side stand-in),
// and the device's ordinal.
int static_flux_scratch(void** address, int* device_out) {
    int device = 0;
    ALS_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= 256) {
        return fail(ALS_E_UNSUPPORTED, "device ordinal out of range for the static scratch table");
    }
    std::lock_guard<std::mutex> lock(g_static_flux_mutex);
    if (!g_static_flux_address[device]) {
        void* p = nullptr;
        ALS_CUDA(cudaGetSymbolAddress(&p, g_static_flux_wave_speeds));
        g_static_flux_address[device] = p;
    }
    *address = g_static_flux_address[device];
    *device_out = device;
    return ALS_OK;
}

} // namespace

extern "C" int als_compute_flux_static(const als_grid* grid, int flux, int reconstruction,
    const double* in, double* out, int members, double* wave_speed, void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!valid_choice(flux, reconstruction) || !in || !out || !wave_speed) {
        return fail(ALS_E_INVALID, "invalid flux arguments");
    }
    rc = check_supported(flux, reconstruction);
    if (rc != ALS_OK) {
        return rc;
    }
    if (members < 1 || members > kStaticFluxMembers) {
        return fail(ALS_E_INVALID, "als_compute_flux_static takes 1 to 1024 states per call");
    }
    if (grid->ghosts < als_ghost_cells(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "planes have fewer ghost cells than the flux needs");
    }
    void* scratch = nullptr;
    int device = 0;
    rc = static_flux_scratch(&scratch, &device);
    if (rc != ALS_OK) {
        return rc;
    }
    std::lock_guard<std::mutex> turn(g_static_flux_calls[device]);
    int lo[3] = {0, 0, 0};
    int n[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = d < grid->dimension ? grid->n[d] : 1;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int nvar = grid->dimension + 2;
    als::StageParams P;
    std::memset(&P, 0, sizeof(P));
    als::GridDesc gd = make_grid(grid->dimension, n, grid->ghosts, lo, n);
    const void* planes_in[als::kMaxVars];
    void* planes_out[als::kMaxVars];
    for (int v = 0; v < nvar; ++v) {
        planes_in[v] = in + v * gd.plane;
        planes_out[v] = out + v * gd.plane;
    }
    P.level[0] = plane_level(gd, nvar, planes_in, planes_in, planes_out);
    P.level[0].member_stride = (long long)nvar * gd.plane;
    P.level[0].members = members;
    P.level[0].ws_out = static_cast<unsigned long long*>(scratch);
    P.nlevels = 1;
    P.bc = ALS_BC_NEUMANN;
    P.write_ghosts = 0;
    P.gamma = grid->gamma;
    finish_params(P);
    // the array keeps the previous call's maxima: clear the slots used
    const size_t bytes = sizeof(unsigned long long) * 3 * size_t(members);
    ALS_CUDA(cudaMemsetAsync(scratch, 0, bytes, s));
    ALS_CUDA(launch_stage(ALS_FP64, grid->dimension, reconstruction, flux, als::KIND_FLUX0, P,
        0, s));
    // a non-negative double and its bit pattern read as an unsigned integer
    // are the same 8 bytes, so the maxima are copied straight into doubles
    ALS_CUDA(cudaMemcpyAsync(wave_speed, scratch, bytes, cudaMemcpyDeviceToHost, s));
    ALS_CUDA(cudaStreamSynchronize(s));
    return ALS_OK;
}
