// C ABI of the hot path (include/als_b200.h): plug-in level calls that
// mirror one virtual call of the reference interfaces each, and the fused
// solver that runs whole time steps on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "als_b200.h"
#include "aux_kernels.cuh"
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
    return flux >= ALS_FLUX_HLL && flux <= ALS_FLUX_CENTRAL && recon >= ALS_RECON_NONE &&
        recon <= ALS_RECON_ENO4;
}

cudaError_t launch_stage(int precision, int dim, int recon, int flux, int kind,
    const als::StageParams& P, int members, cudaStream_t s) {
    if (precision == ALS_FP64) {
        switch (dim) {
        case 1: return als::launch_stage_f64_1d(recon, flux, kind, P, members, s);
        case 2: return als::launch_stage_f64_2d(recon, flux, kind, P, members, s);
        default: return als::launch_stage_f64_3d(recon, flux, kind, P, members, s);
        }
    }
    switch (dim) {
    case 1: return als::launch_stage_f32_1d(recon, flux, kind, P, members, s);
    case 2: return als::launch_stage_f32_2d(recon, flux, kind, P, members, s);
    default: return als::launch_stage_f32_3d(recon, flux, kind, P, members, s);
    }
}

// Tile extent along d of the kernels built for (precision, dim), as reported
// by the unit that holds them.
int tile_extent(int precision, int dim, int d) {
    if (d >= dim) {
        return 1;
    }
    int tile[3] = {1, 1, 1};
    if (precision == ALS_FP64) {
        dim == 1 ? als::stage_tile_f64_1d(tile) : (dim == 2 ? als::stage_tile_f64_2d(tile) : als::stage_tile_f64_3d(tile));
    } else {
        dim == 1 ? als::stage_tile_f32_1d(tile) : (dim == 2 ? als::stage_tile_f32_2d(tile) : als::stage_tile_f32_3d(tile));
    }
    return tile[d];
}

// Geometry of a padded grid and the tiles covering the region [lo, hi).
als::GridDesc make_grid(int dim, const int* n, int g, const int* lo, const int* hi,
    int precision = ALS_FP64) {
    als::GridDesc gd;
    for (int d = 0; d < 3; ++d) {
        gd.n[d] = d < dim ? n[d] : 1;
        gd.N[d] = gd.n[d] + (d < dim ? 2 * g : 0);
        gd.lo[d] = d < dim ? lo[d] : 0;
        gd.hi[d] = d < dim ? hi[d] : 1;
        const int t = tile_extent(precision, dim, d);
        gd.tiles[d] = std::max(1, (gd.hi[d] - gd.lo[d] + t - 1) / t);
    }
    gd.plane = (long long)gd.N[0] * gd.N[1] * gd.N[2];
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

} // namespace

extern "C" {

const char* als_last_error(void) {
    return g_error.c_str();
}

int als_version(void) {
    return 1;
}

int als_ghost_cells(int flux, int reconstruction) {
    if (!valid_choice(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "unknown flux or reconstruction");
    }
    // every in-scope flux uses the two-point stencil {0, 1} (numflux_util.hpp:52-60)
    return std::max(1, als::recon_ghosts(reconstruction));
}

int als_fill_ghosts(const als_grid* grid, int boundary, double* planes, int nvar, int members,
    void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!planes || nvar < 1 || members < 1 || (boundary != ALS_BC_NEUMANN && boundary != ALS_BC_PERIODIC)) {
        return fail(ALS_E_INVALID, "invalid ghost-fill arguments");
    }
    int lo[3] = {0, 0, 0};
    als::GridDesc gd = make_grid(grid->dimension, grid->n, grid->ghosts, lo, grid->n);
    dim3 blocks(grid_blocks(gd.plane, 256), members);
    als::fill_ghosts<double><<<blocks, 256, 0, (cudaStream_t)stream>>>(planes, nvar, gd.plane,
        (long long)nvar * gd.plane, grid->dimension, gd.n[0], gd.n[1], gd.n[2], grid->ghosts,
        boundary);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int als_compute_flux(const als_grid* grid, int flux, int reconstruction, const double* in,
    double* out, const int* start, const int* end, double* wave_speed, void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (!valid_choice(flux, reconstruction) || !in || !out || !wave_speed) {
        return fail(ALS_E_INVALID, "invalid flux arguments");
    }
    if (grid->ghosts < als_ghost_cells(flux, reconstruction)) {
        return fail(ALS_E_INVALID, "planes have fewer ghost cells than the reconstruction needs");
    }
    if (grid->ghosts != als_ghost_cells(flux, reconstruction)) {
        return fail(ALS_E_UNSUPPORTED, "planes must have exactly the ghost width of the reconstruction");
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
    P.in = in;
    P.un = in;
    P.out = out;
    P.grid = make_grid(grid->dimension, grid->n, grid->ghosts, lo, hi);
    P.sample_stride = 0;
    P.bc = ALS_BC_NEUMANN;
    P.write_ghosts = 0;
    P.gamma = grid->gamma;
    unsigned long long* ws_dev = nullptr;
    ALS_CUDA(cudaMallocAsync((void**)&ws_dev, 3 * sizeof(unsigned long long), s));
    ALS_CUDA(cudaMemsetAsync(ws_dev, 0, 3 * sizeof(unsigned long long), s));
    P.ws_out = ws_dev;
    cudaError_t err = launch_stage(ALS_FP64, grid->dimension, reconstruction, flux,
        als::KIND_FLUX0, P, 1, s);
    unsigned long long host[3] = {0, 0, 0};
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(host, ws_dev, sizeof(host), cudaMemcpyDeviceToHost, s);
    }
    cudaFreeAsync(ws_dev, s);
    if (err == cudaSuccess) {
        err = cudaStreamSynchronize(s);
    }
    if (err != cudaSuccess) {
        return fail(ALS_E_CUDA, std::string("compute_flux: ") + cudaGetErrorString(err));
    }
    for (int d = 0; d < 3; ++d) {
        double w;
        std::memcpy(&w, &host[d], sizeof(w));
        wave_speed[d] = w;
    }
    return ALS_OK;
}

int als_reconstruct(const als_grid* grid, int reconstruction, int direction, const double* in,
    double* left, double* right, void* stream) {
    int rc = check_grid(grid);
    if (rc != ALS_OK) {
        return rc;
    }
    if (direction < 0 || direction >= grid->dimension || !in || !left || !right ||
        reconstruction < ALS_RECON_NONE || reconstruction > ALS_RECON_ENO4) {
        return fail(ALS_E_INVALID, "invalid reconstruction arguments");
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
    if (plane > INT_MAX) {
        return fail(ALS_E_UNSUPPORTED, "plane too large for the plug-in reconstruction");
    }
    const int blocks = grid_blocks(plane, 256);
    cudaStream_t s = (cudaStream_t)stream;
    const int dim = grid->dimension;
    if (reconstruction == ALS_RECON_NONE) {
        // NoReconstruction copies every cell, ghosts included (NoReconstruction.cpp:51-61)
        const size_t bytes = sizeof(double) * size_t(dim + 2) * size_t(plane);
        ALS_CUDA(cudaMemcpyAsync(left, in, bytes, cudaMemcpyDeviceToDevice, s));
        ALS_CUDA(cudaMemcpyAsync(right, in, bytes, cudaMemcpyDeviceToDevice, s));
        return ALS_OK;
    }
#define ALS_RECON_CASE(NV, RC)                                                               \
    als::reconstruct_dir<double, NV, RC><<<blocks, 256, 0, s>>>(in, left, right, plane, dim,  \
        N[0], N[1], N[2], G, direction)
#define ALS_RECON_NV(NV)                                                                     \
    switch (reconstruction) {                                                                \
    case ALS_RECON_NONE: ALS_RECON_CASE(NV, als::RECON_NONE); break;                         \
    case ALS_RECON_WENO2: ALS_RECON_CASE(NV, als::RECON_WENO2); break;                       \
    case ALS_RECON_ENO2: ALS_RECON_CASE(NV, als::RECON_ENO2); break;                         \
    case ALS_RECON_ENO3: ALS_RECON_CASE(NV, als::RECON_ENO3); break;                         \
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
    if (integrator < ALS_INT_FORWARD_EULER || integrator > ALS_INT_RK3 || substep < 0 ||
        substep >= substeps || !out || !us || (substep > 0 && !u0)) {
        return fail(ALS_E_INVALID, "invalid combine arguments");
    }
    als::combine<double><<<grid_blocks((long long)count, 256), 256, 0, (cudaStream_t)stream>>>(
        out, us, u0, (long long)count, c, integrator, substep);
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

struct als_solver {
    als_solver_config cfg;
    int device = 0;
    int g = 0;
    int nv = 0;
    size_t elem = 8;
    als::GridDesc grid;
    long long member_elems = 0;   // nv * plane
    void* buf[3] = {nullptr, nullptr, nullptr};  // state A, flux L, state B
    int cur = 0;                  // RK2 ping-pong: index (0 -> buf[0], 1 -> buf[2]) of U^n
    als::StepState* state = nullptr;
    als::StepState* host_state = nullptr;  // pinned mirror
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    int graph_cur = 0;            // ping-pong position the graph was captured at
    double dx[3];

    ~als_solver() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (graph) {
            cudaGraphExecDestroy(graph);
        }
        for (void* p : buf) {
            if (p) {
                cudaFree(p);
            }
        }
        if (state) {
            cudaFree(state);
        }
        if (host_state) {
            cudaFreeHost(host_state);
        }
        if (stream) {
            cudaStreamDestroy(stream);
        }
        cudaSetDevice(prev);
    }

    void* current() const {
        return cfg.integrator == ALS_INT_RK2 && cur == 1 ? buf[2] : buf[0];
    }
    void* other() const {
        return cfg.integrator == ALS_INT_RK2 && cur == 1 ? buf[0] : buf[2];
    }
};

namespace {

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

als::StageParams solver_params(const als_solver* s) {
    als::StageParams P;
    std::memset(&P, 0, sizeof(P));
    P.grid = s->grid;
    P.sample_stride = s->member_elems;
    P.bc = s->cfg.boundary;
    P.write_ghosts = 1;
    P.gamma = s->cfg.gamma;
    P.state = s->state;
    P.member0 = 0;
    return P;
}

// Enqueues one time step.  FE: FLUX0 + fe_update.  RK2: FLUX0 + RK2_1 into the
// other buffer (ping-pong).  RK3: FLUX0 + RK3_1 + RK3_2 in place.
// With `ev` (launches+1 events), records ev[0] before the first kernel and
// ev[k] after kernel k.
int enqueue_step(als_solver* s, cudaEvent_t* ev = nullptr) {
    const int prec = s->cfg.precision;
    const int dim = s->cfg.dimension;
    const int recon = s->cfg.reconstruction;
    const int flux = s->cfg.flux;
    const int members = s->cfg.members;
    als::StageParams P = solver_params(s);
    void* un = s->current();
    P.in = un;
    P.un = un;
    P.out = s->buf[1];
    if (ev) {
        ALS_CUDA(cudaEventRecord(ev[0], s->stream));
    }
    ALS_CUDA(launch_stage(prec, dim, recon, flux, als::KIND_FLUX0, P, members, s->stream));
    if (ev) {
        ALS_CUDA(cudaEventRecord(ev[1], s->stream));
    }
    if (s->cfg.integrator == ALS_INT_FORWARD_EULER) {
        dim3 blocks(grid_blocks(s->grid.plane, 256), members);
        if (prec == ALS_FP64) {
            if (dim == 1) {
                als::fe_update<double, 3><<<blocks, 256, 0, s->stream>>>((const double*)s->buf[1], (double*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            } else if (dim == 2) {
                als::fe_update<double, 4><<<blocks, 256, 0, s->stream>>>((const double*)s->buf[1], (double*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            } else {
                als::fe_update<double, 5><<<blocks, 256, 0, s->stream>>>((const double*)s->buf[1], (double*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            }
        } else {
            if (dim == 1) {
                als::fe_update<float, 3><<<blocks, 256, 0, s->stream>>>((const float*)s->buf[1], (float*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            } else if (dim == 2) {
                als::fe_update<float, 4><<<blocks, 256, 0, s->stream>>>((const float*)s->buf[1], (float*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            } else {
                als::fe_update<float, 5><<<blocks, 256, 0, s->stream>>>((const float*)s->buf[1], (float*)un, s->grid.plane, s->member_elems, s->state, 0, s->cfg.gamma);
            }
        }
        ALS_CUDA(cudaGetLastError());
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
    } else if (s->cfg.integrator == ALS_INT_RK2) {
        P.in = s->buf[1];
        P.un = un;
        P.out = s->other();
        ALS_CUDA(launch_stage(prec, dim, recon, flux, als::KIND_RK2_1, P, members, s->stream));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
        s->cur ^= 1;
    } else {
        P.in = s->buf[1];
        P.un = un;
        P.out = s->buf[2];
        ALS_CUDA(launch_stage(prec, dim, recon, flux, als::KIND_RK3_1, P, members, s->stream));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[2], s->stream));
        }
        P.in = s->buf[2];
        P.un = un;
        P.out = un;
        ALS_CUDA(launch_stage(prec, dim, recon, flux, als::KIND_RK3_2, P, members, s->stream));
        if (ev) {
            ALS_CUDA(cudaEventRecord(ev[3], s->stream));
        }
    }
    return ALS_OK;
}

template<class R>
int fill_member_ghosts(als_solver* s, void* base, int first, int count) {
    dim3 blocks(grid_blocks(s->grid.plane, 256), count);
    als::fill_ghosts<R><<<blocks, 256, 0, s->stream>>>(
        static_cast<R*>(base) + (long long)first * s->member_elems, s->nv, s->grid.plane,
        s->member_elems, s->cfg.dimension, s->grid.n[0], s->grid.n[1], s->grid.n[2], s->g,
        s->cfg.boundary);
    ALS_CUDA(cudaGetLastError());
    return ALS_OK;
}

int reset_members(als_solver* s, int first, int count) {
    for (int m = first; m < first + count; ++m) {
        als::StepState& st = s->host_state[m];
        std::memset(&st, 0, sizeof(st));
        st.t = 0;
        st.dt = 0;
        st.end_time = s->cfg.end_time;
        st.cfl = s->cfg.cfl;
        st.max_steps = s->cfg.max_steps > 0 ? s->cfg.max_steps : LLONG_MAX;
        st.done = (0 >= s->cfg.end_time) ? 1 : 0;
        st.bad_index = -1;  // as unsigned: the largest value, lowered by atomicMin
        st.bad_step = -1;
        for (int d = 0; d < 3; ++d) {
            st.dx[d] = s->dx[d];
        }
    }
    ALS_CUDA(cudaMemcpyAsync(s->state + first, s->host_state + first,
        sizeof(als::StepState) * count, cudaMemcpyHostToDevice, s->stream));
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

int refresh_host_state(als_solver* s) {
    ALS_CUDA(cudaMemcpyAsync(s->host_state, s->state, sizeof(als::StepState) * s->cfg.members,
        cudaMemcpyDeviceToHost, s->stream));
    ALS_CUDA(cudaStreamSynchronize(s->stream));
    return ALS_OK;
}

} // namespace

extern "C" {

int als_solver_create(const als_solver_config* cfg, int device, als_solver** out) {
    if (!cfg || !out) {
        return fail(ALS_E_INVALID, "null argument");
    }
    *out = nullptr;
    if (cfg->dimension < 1 || cfg->dimension > 3 || !valid_choice(cfg->flux, cfg->reconstruction) ||
        cfg->integrator < ALS_INT_FORWARD_EULER || cfg->integrator > ALS_INT_RK3 ||
        (cfg->boundary != ALS_BC_NEUMANN && cfg->boundary != ALS_BC_PERIODIC) ||
        (cfg->precision != ALS_FP64 && cfg->precision != ALS_FP32) || cfg->members < 1 ||
        !(cfg->gamma > 1) || !(cfg->cfl > 0)) {
        return fail(ALS_E_INVALID, "invalid solver configuration");
    }
    const int g = als_ghost_cells(cfg->flux, cfg->reconstruction);
    for (int d = 0; d < cfg->dimension; ++d) {
        // ConservedSystem splits the update into an interior and 2*dim side
        // regions of width g (ConservedSystem.cpp:59-96); with fewer than 2g
        // cells those regions reach into the ghost layer, which this solver
        // does not reproduce.
        if (cfg->n[d] < 2 * g) {
            return fail(ALS_E_INVALID, "every active direction needs at least 2*ghosts interior cells");
        }
    }
    std::unique_ptr<als_solver> s(new (std::nothrow) als_solver());
    if (!s) {
        return fail(ALS_E_NOMEM, "out of host memory");
    }
    s->cfg = *cfg;
    s->device = device;
    s->g = g;
    s->nv = cfg->dimension + 2;
    s->elem = cfg->precision == ALS_FP64 ? 8 : 4;
    int lo[3] = {0, 0, 0};
    int n[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = d < cfg->dimension ? cfg->n[d] : 1;
    }
    s->grid = make_grid(cfg->dimension, n, g, lo, n, cfg->precision);
    s->member_elems = (long long)s->nv * s->grid.plane;
    for (int d = 0; d < 3; ++d) {
        // Grid.cpp:24-41: (top - origin) / n, and 1 for a direction with one cell
        s->dx[d] = (cfg->upper[d] - cfg->lower[d]) / double(n[d]);
        if (d > 0 && n[d] == 1) {
            s->dx[d] = 1;
        }
    }
    DeviceGuard guard(device);
    ALS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    const size_t bytes = size_t(s->member_elems) * cfg->members * s->elem;
    for (int b = 0; b < 3; ++b) {
        if (b == 2 && cfg->integrator == ALS_INT_FORWARD_EULER) {
            continue;
        }
        ALS_CUDA(cudaMalloc(&s->buf[b], bytes));
        ALS_CUDA(cudaMemset(s->buf[b], 0, bytes));
    }
    ALS_CUDA(cudaMalloc((void**)&s->state, sizeof(als::StepState) * cfg->members));
    ALS_CUDA(cudaMallocHost((void**)&s->host_state, sizeof(als::StepState) * cfg->members));
    int rc = reset_members(s.get(), 0, cfg->members);
    if (rc != ALS_OK) {
        return rc;
    }
    *out = s.release();
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
        *plane = s->grid.plane;
    }
    if (ghosts) {
        *ghosts = s->g;
    }
    return ALS_OK;
}

int als_solver_set_state(als_solver* s, const double* host, int first_member, int count) {
    if (!s || !host || first_member < 0 || count < 1 || first_member + count > s->cfg.members) {
        return fail(ALS_E_INVALID, "invalid set_state arguments");
    }
    DeviceGuard guard(s->device);
    const size_t n = size_t(s->member_elems) * count;
    s->cur = 0;
    if (s->cfg.precision == ALS_FP64) {
        ALS_CUDA(cudaMemcpyAsync(static_cast<double*>(s->buf[0]) + (long long)first_member * s->member_elems,
            host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        int rc = fill_member_ghosts<double>(s, s->buf[0], first_member, count);
        if (rc != ALS_OK) {
            return rc;
        }
    } else {
        std::vector<float> tmp(n);
        for (size_t i = 0; i < n; ++i) {
            tmp[i] = float(host[i]);
        }
        ALS_CUDA(cudaMemcpyAsync(static_cast<float*>(s->buf[0]) + (long long)first_member * s->member_elems,
            tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
        int rc = fill_member_ghosts<float>(s, s->buf[0], first_member, count);
        if (rc != ALS_OK) {
            return rc;
        }
        ALS_CUDA(cudaStreamSynchronize(s->stream));
    }
    return reset_members(s, first_member, count);
}

int als_solver_set_state_device(als_solver* s, const void* dev, int first_member, int count) {
    if (!s || !dev || first_member < 0 || count < 1 || first_member + count > s->cfg.members) {
        return fail(ALS_E_INVALID, "invalid set_state_device arguments");
    }
    DeviceGuard guard(s->device);
    s->cur = 0;
    const size_t bytes = size_t(s->member_elems) * count * s->elem;
    ALS_CUDA(cudaMemcpyAsync(static_cast<char*>(s->buf[0]) + size_t(first_member) * s->member_elems * s->elem,
        dev, bytes, cudaMemcpyDeviceToDevice, s->stream));
    int rc = s->cfg.precision == ALS_FP64 ? fill_member_ghosts<double>(s, s->buf[0], first_member, count)
                                          : fill_member_ghosts<float>(s, s->buf[0], first_member, count);
    if (rc != ALS_OK) {
        return rc;
    }
    return reset_members(s, first_member, count);
}

int als_solver_get_state(als_solver* s, double* host, int first_member, int count) {
    if (!s || !host || first_member < 0 || count < 1 || first_member + count > s->cfg.members) {
        return fail(ALS_E_INVALID, "invalid get_state arguments");
    }
    DeviceGuard guard(s->device);
    if (s->cfg.integrator == ALS_INT_RK2) {
        // RK2 alternates between two buffers; a member's state sits in the
        // buffer given by the parity of its own completed steps
        int rc = refresh_host_state(s);
        if (rc != ALS_OK) {
            return rc;
        }
    }
    const size_t n = size_t(s->member_elems);
    std::vector<float> tmp(s->cfg.precision == ALS_FP64 ? 0 : n);
    for (int m = first_member; m < first_member + count; ++m) {
        const void* base = s->buf[0];
        if (s->cfg.integrator == ALS_INT_RK2 && (s->host_state[m].steps & 1)) {
            base = s->buf[2];
        }
        const char* src = static_cast<const char*>(base) + size_t(m) * n * s->elem;
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

int als_solver_state_pointer(als_solver* s, void** dev) {
    if (!s || !dev) {
        return fail(ALS_E_INVALID, "null argument");
    }
    *dev = s->current();
    return ALS_OK;
}

int als_solver_advance(als_solver* s, long long steps) {
    if (!s || steps < 0) {
        return fail(ALS_E_INVALID, "invalid advance arguments");
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
        for (int m = 0; m < s->cfg.members; ++m) {
            const als::StepState& st = s->host_state[m];
            progress += st.t;
        }
        for (int m = 0; m < s->cfg.members; ++m) {
            const als::StepState& st = s->host_state[m];
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
    if (!s || !info || member < 0 || member >= s->cfg.members) {
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
    return s->cfg.integrator == ALS_INT_RK3 ? 3 : 2;
}

int als_solver_profile_step(als_solver* s, float* kernel_ms, int capacity) {
    if (!s || !kernel_ms) {
        return fail(ALS_E_INVALID, "null argument");
    }
    const int k = als_solver_launches_per_step(s);
    if (capacity < k) {
        return fail(ALS_E_INVALID, "capacity below the launches per step");
    }
    DeviceGuard guard(s->device);
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int rc = ALS_OK;
    for (int i = 0; i <= k && rc == ALS_OK; ++i) {
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
    for (int i = 0; i <= k; ++i) {
        if (ev[i]) {
            cudaEventDestroy(ev[i]);
        }
    }
    return rc == ALS_OK ? k : rc;
}

} // extern "C"

// ------------------------------------------- allocation-free flux evaluation
//
// als_compute_flux reserves three wave-speed accumulators per call with
// cudaMallocAsync.  Some hosts of NumericalFlux::computeFlux cannot let a
// library allocate device memory: a runtime that plans every byte of device
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

// Device address of the array on the current device, looked up once per
// device (cudaGetSymbolAddress; the name itself is a host-side stand-in).
int static_flux_scratch(void** address) {
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
    if (members < 1 || members > kStaticFluxMembers) {
        return fail(ALS_E_INVALID, "als_compute_flux_static takes 1 to 1024 states per call");
    }
    if (grid->ghosts != als_ghost_cells(flux, reconstruction)) {
        return fail(ALS_E_UNSUPPORTED, "planes must have exactly the ghost width of the reconstruction");
    }
    void* scratch = nullptr;
    rc = static_flux_scratch(&scratch);
    if (rc != ALS_OK) {
        return rc;
    }
    int lo[3] = {0, 0, 0};
    int n[3];
    for (int d = 0; d < 3; ++d) {
        n[d] = d < grid->dimension ? grid->n[d] : 1;
    }
    cudaStream_t s = (cudaStream_t)stream;
    als::StageParams P;
    std::memset(&P, 0, sizeof(P));
    P.in = in;
    P.un = in;
    P.out = out;
    P.grid = make_grid(grid->dimension, n, grid->ghosts, lo, n);
    P.sample_stride = (long long)(grid->dimension + 2) * P.grid.plane;
    P.bc = ALS_BC_NEUMANN;
    P.write_ghosts = 0;
    P.gamma = grid->gamma;
    P.ws_out = static_cast<unsigned long long*>(scratch);
    // the array keeps the previous call's maxima: clear the slots used
    const size_t bytes = sizeof(unsigned long long) * 3 * size_t(members);
    ALS_CUDA(cudaMemsetAsync(scratch, 0, bytes, s));
    ALS_CUDA(launch_stage(ALS_FP64, grid->dimension, reconstruction, flux, als::KIND_FLUX0, P,
        members, s));
    // a non-negative double and its bit pattern read as an unsigned integer
    // are the same 8 bytes, so the maxima are copied straight into doubles
    ALS_CUDA(cudaMemcpyAsync(wave_speed, scratch, bytes, cudaMemcpyDeviceToHost, s));
    ALS_CUDA(cudaStreamSynchronize(s));
    return ALS_OK;
}
