/*
 * als_b200.h -- C ABI of the B200 cell-update hot path of alsfvm.
 *
 * Plain C types only: device pointers are `void*`/`double*` obtained from
 * cudaMalloc (or any allocator of device memory), streams are passed as
 * `void*` (a cudaStream_t; NULL = legacy default stream).  Every function
 * returns ALS_OK (0) or a negative ALS_E* code; als_last_error() gives a
 * readable message for the calling thread.  No C++ exception crosses the
 * ABI.
 *
 * Data layout (alsfvm::volume::Volume, alsfvm/src/volume/Volume.cpp:44-60,
 * alsfvm/include/alsfvm/memory/View.hpp): one contiguous plane per conserved
 * variable, (nx+2g)(ny+2g)(nz+2g) cells each with x fastest, no pitch;
 * inactive directions have extent 1 and no ghost cells.  Variable order
 * rho, mx, [my, [mz,]] E (alsfvm/src/equation/euler/Euler.cpp:20-75).
 * An ensemble of M members stores its members one after another.
 */
#ifndef ALS_B200_H
#define ALS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ codes */
#define ALS_OK 0
#define ALS_E_INVALID (-1)          /* bad argument */
#define ALS_E_CUDA (-2)             /* a CUDA call failed */
#define ALS_E_CONSTRAINT (-3)       /* Simulator::checkConstraints would throw */
#define ALS_E_UNSUPPORTED (-4)      /* combination not built */
#define ALS_E_NOMEM (-5)

/* names as in the reference's XML (<flux>, <reconstruction>, <integrator>, <boundary>) */
#define ALS_FLUX_HLL 0              /* "hll",     numflux/euler/HLL.hpp */
#define ALS_FLUX_HLL3 1             /* "hll3",    numflux/euler/HLL3.hpp */
#define ALS_FLUX_CENTRAL 2          /* "central", numflux/Central.hpp */
/* TeCNO fluxes, with reconstruction "none" (ALS_E_UNSUPPORTED otherwise): */
#define ALS_FLUX_TECNO1 3           /* "tecno1",  numflux/euler/Tecno1.hpp (entropy conservative) */
#define ALS_FLUX_TECNO4 4           /* "tecno4",  numflux/TecnoCombined4.hpp (stencil -1..2, 3 ghost cells) */
#define ALS_FLUX_TECNO6 5           /* "tecno6",  numflux/TecnoCombined6.hpp (stencil -2..3, 5 ghost cells) */
#define ALS_RECON_NONE 0            /* "none",  reconstruction/NoReconstruction.cpp */
#define ALS_RECON_WENO2 1           /* "weno2", reconstruction/WENO2.hpp */
#define ALS_RECON_ENO2 2            /* "eno2",  reconstruction/ENOCPU.cpp */
#define ALS_RECON_ENO3 3            /* "eno3" */
#define ALS_RECON_ENO4 4            /* "eno4" */
#define ALS_RECON_MC 5              /* "mc", reconstruction/MC.hpp */
#define ALS_RECON_MM 6              /* "mm", reconstruction/MM.hpp */
#define ALS_RECON_WENOF2 7          /* "wenof2", reconstruction/WENOF2.hpp (WENO2 in primitive variables, bounded) */
#define ALS_RECON_WENO3 8           /* "weno3", reconstruction/WENOCPU.cpp (order 3, three ghost cells) */
#define ALS_INT_FORWARD_EULER 0     /* "forwardeuler", integrator/ForwardEuler.cpp */
#define ALS_INT_RK2 1               /* "rungekutta2",  integrator/RungeKutta2.cpp */
#define ALS_INT_RK3 2               /* "rungekutta3",  integrator/RungeKutta3.cpp */
#define ALS_INT_RK4 3               /* "rungekutta4",  integrator/RungeKutta4.cpp (plug-in path only) */
#define ALS_BC_NEUMANN 0            /* "neumann",  boundary/Neumann.hpp */
#define ALS_BC_PERIODIC 1           /* "periodic", boundary/Periodic.hpp */
#define ALS_FP64 0
#define ALS_FP32 1

const char* als_last_error(void);
int als_version(void);
/* Scratch memory of the entry points that need temporary device memory
 * (functionals, structure functions, region sums) comes from one retaining
 * pool per device: it keeps the largest amount any call needed until the
 * process exits, hidden from other allocators.  This hands the unused part
 * of `device`'s pool back until at most `keep_bytes` stay reserved.  It has
 * no counterpart in the reference (its volumes allocate per object). */
int als_scratch_trim(int device, unsigned long long keep_bytes);

/* Ghost width of a flux/reconstruction pair: max(stencil-1, reconstruction
 * ghosts).  Replaces NumericalFlux::getNumberOfGhostCells,
 * alsfvm/src/numflux/NumericalFluxCPU.cpp:227-231 (and
 * Reconstruction::getNumberOfGhostCells, reconstruction/Reconstruction.hpp:56). */
int als_ghost_cells(int flux, int reconstruction);

/* ------------------------------------------------ plug-in level calls
 * Each call works on caller-owned device planes, is stream ordered, and
 * has the meaning of one virtual call of the reference interface it cites.
 */
typedef struct {
    int dimension;      /* 1, 2 or 3 */
    int n[3];           /* interior cells (1 for inactive directions) */
    int ghosts;         /* ghost width of the planes */
    double gamma;
} als_grid;

/* Planes are passed as arrays of `nvar` device pointers, one per conserved
 * variable, like the reference Volume's one Memory per variable
 * (alsfvm/src/volume/Volume.cpp:44-60); the planes need not be adjacent. */

/* Boundary::applyBoundaryConditions(Volume&, const Grid&)
 * (alsfvm/include/alsfvm/boundary/Boundary.hpp:30-31; BoundaryCPU.cpp:30-106).
 * Fills the ghost cells of `nvar` planes.  Requires n >= ghosts in every
 * active direction. */
int als_fill_ghosts(const als_grid* grid, int boundary, double* const* planes, int nvar,
    void* stream);

/* NumericalFlux::computeFlux(const Volume&, rvec3& waveSpeed, bool, Volume& out,
 * const ivec3& start, const ivec3& end)
 * (alsfvm/include/alsfvm/numflux/NumericalFlux.hpp:44-52; NumericalFluxCPU.cpp:171-221).
 * `out` receives the net flux of the interior cells in the region
 * [start, n+end) (start/end as in the reference: offsets from the interior
 * bounds, end <= 0); other cells are left untouched.  `wave_speed` (host,
 * 3 doubles) receives the maximal face wave speed per direction; the call
 * synchronises `stream` to read it back, like the reference's CUDA path.
 * With `wave_speed` null (the reference's computeWaveSpeed == false) the
 * flux is only enqueued on `stream`: no wave speeds, no synchronisation.
 * The wave-speed accumulators are three words of device memory that each
 * host thread allocates once per device and reuses (a call that reads them
 * back has finished with them when it returns); that first call on a thread
 * and device allocates, so make it before any stream capture. */
int als_compute_flux(const als_grid* grid, int flux, int reconstruction, const double* const* in,
    double* const* out, const int* start, const int* end, double* wave_speed, void* stream);

/* Allocation-free variant of als_compute_flux; it has no counterpart in the
 * reference.  For callers that cannot let a library allocate device memory:
 * a runtime that owns and pre-plans all device memory (another framework's
 * pool, a fixed-budget deployment) or one that forbids allocation while it
 * drives the flux evaluation many times per time step.  It evaluates the
 * net flux of `members` (1..1024) consecutive states (each nvar adjacent
 * padded planes, the whole interior, no region arguments) into `out`, and writes
 * their maximal face wave speeds to `wave_speed` (host, 3 per state).  The
 * wave-speed accumulators live in a fixed 24 KiB device array inside the
 * library that every GPU loading it keeps until the process exits; no
 * cudaMalloc, cudaFree or allocating routine is called.  The first call on a
 * device looks the array's address up (cudaGetSymbolAddress) in the
 * runtime's primary context of that device, which later calls on that
 * device use: make that first call before any stream capture, and call it
 * only with the primary context current.  Calls share the array and the call
 * clears what it uses; calls on one device from several threads take
 * turns (a lock held from the clearing of the array to the read-back), and
 * the call synchronises `stream` before it returns.  More than 1024 states
 * is rejected with ALS_E_INVALID. */
int als_compute_flux_static(const als_grid* grid, int flux, int reconstruction, const double* in,
    double* out, int members, double* wave_speed, void* stream);

/* Reconstruction::performReconstruction(const Volume& in, size_t direction,
 * size_t indicatorVariable=0, Volume& left, Volume& right)
 * (alsfvm/include/alsfvm/reconstruction/Reconstruction.hpp:46-58;
 * ReconstructionCPU.cpp:37-97, ENOCPU.cpp:41-187).  The indicator is rho. */
int als_reconstruct(const als_grid* grid, int reconstruction, int direction,
    const double* const* in, double* const* left, double* const* right, void* stream);

/* Stage combination of Integrator::performSubstep
 * (alsfvm/include/alsfvm/integrator/Integrator.hpp:59-80; ForwardEuler.cpp:32-51,
 * RungeKutta2.cpp:37-67, RungeKutta3.cpp:49-86, RungeKutta4.cpp:66-78) over
 * `count` elements: on entry out = L(U_substep); us = U_substep, u0 = U_0;
 * c = dt/dx.  RK4's substep 3 takes als_integrator_combine_rk4. */
int als_integrator_combine(int integrator, int substep, double* out, const double* us,
    const double* u0, size_t count, double c, void* stream);

/* RK4's last stage (RungeKutta4.cpp:80-87, Volume::addLinearCombination):
 * out = (c/6) L(U_3) + U_1/3 + 2 U_2/3 + U_3/3 - U_0/3, on entry out = L(U_3). */
int als_integrator_combine_rk4(double* out, const double* u0, const double* u1, const double* u2,
    const double* u3, size_t count, double c, void* stream);

/* Integrator::computeTimestep + adjustTimestep with an end-time clamp
 * (alsfvm/src/integrator/Integrator.cpp:20-46, alsfvm/src/io/FixedIntervalWriter.cpp:45-53):
 * dt = min(cfl / sum_d ws_d/dx_d, end_time - t).  Host-only arithmetic. */
double als_compute_timestep(const double* wave_speed, const double* cell_lengths, double cfl,
    double t, double end_time);

/* ----------------------------------------------------- fused solver
 * Owns the state of one simulation or of an ensemble of `members`
 * simulations of the same grid, and advances whole time steps with no host
 * round trip: the time step, the CFL dt and the end-time test live on the
 * device.  Replaces Simulator::incrementSolution + checkConstraints
 * (alsfvm/src/simulator/Simulator.cpp:180-214) and, for ensembles, the
 * serial sample loop of alsuq::run::Runner::run (alsuq/src/run/Runner.cpp:42-78).
 */
typedef struct {
    int dimension;
    int n[3];
    double lower[3];    /* domain corners; cell lengths as Grid.cpp:24-41 */
    double upper[3];
    int flux;
    int reconstruction;
    int integrator;
    int boundary;
    double gamma;
    double cfl;
    double end_time;
    long long max_steps; /* <= 0: unlimited */
    int precision;      /* ALS_FP64, or ALS_FP32 for ensemble members */
    int members;        /* ensemble size, >= 1 */
} als_solver_config;

typedef struct {
    double t;
    double dt;          /* dt of the last completed step */
    long long steps;
    int done;
    int status;         /* 0 ok, 1 constraint violation */
    long long bad_index;  /* padded cell index of the first violation, or -1 */
    long long bad_step;   /* step at which it was detected, or -1 */
} als_member_info;

typedef struct als_solver als_solver;

int als_solver_create(const als_solver_config* cfg, int device, als_solver** out);
/* A solver over 1..4 grid levels (e.g. the levels of a multilevel Monte
 * Carlo batch) advanced together: every stage is one persistent launch over
 * the tiles of every member of every level.  Levels may differ only in n,
 * lower, upper and members; members are numbered level after level. */
int als_solver_create_levels(const als_solver_config* levels, int nlevels, int device,
    als_solver** out);
/* First member index, member count and padded plane size of a level. */
int als_solver_level(const als_solver* s, int level, int* first_member, int* members,
    long long* plane);
int als_solver_destroy(als_solver* s);
/* Makes the members of a one-level RK2/RK3 solver the subdomains of one
 * grid split over procs[0] x procs[1] x procs[2] ranks, as the reference's
 * MPI path splits it (alsfvm/src/mpi/domain/CartesianDecomposition.cpp:40-135,
 * rank = x + px (y + py z)); the level's n, lower and upper are one
 * subdomain's, and inactive directions take 1.  The subdomains then advance
 * as one simulation: one time step from the largest wave speed over all of
 * them (CartesianCellExchanger.cpp:37-44), and each stage kernel writes
 * every updated cell's images into the ghost layers of the neighbouring
 * subdomains, in place of the reference's exchange of ghost slabs after
 * each stage (CartesianCellExchanger.cpp:51-100); physical sides take the
 * boundary condition.  Results equal the undivided grid's bit for bit.
 * als_solver_set_state then takes each subdomain's padded block as given,
 * ghosts included (its block of the whole grid with the whole grid's ghosts
 * filled).  Every member reports the shared time, step and status;
 * bad_index is member * padded plane + the cell's index in its block.
 * ALS_E_UNSUPPORTED for forward Euler; ALS_E_INVALID unless the solver has
 * one level of exactly procs[0] * procs[1] * procs[2] members. */
int als_solver_decompose(als_solver* s, const int* procs);
/* padded cells per plane (level 0) and the ghost width the solver uses */
int als_solver_geometry(const als_solver* s, long long* plane, int* ghosts);
/* Uploads member states (host, FP64, padded planes; ghost cells are filled
 * by the solver), resets time and step counters of those members.  The
 * members of one call must belong to one level.  Set every member before
 * advancing (RK2 keeps one ping-pong parity for all members). */
int als_solver_set_state(als_solver* s, const double* host, int first_member, int count);
/* Same from device memory already in the solver's precision. */
int als_solver_set_state_device(als_solver* s, const void* dev, int first_member, int count);
/* Downloads member states as FP64 into `host` (padded planes). */
int als_solver_get_state(als_solver* s, double* host, int first_member, int count);
/* Device pointer of the current state of member 0 (layout as above, members consecutive). */
int als_solver_state_pointer(als_solver* s, void** dev);
/* Enqueues `steps` time steps on the solver's stream (no synchronisation);
 * members that are done skip them. */
int als_solver_advance(als_solver* s, long long steps);
/* Advances until every member is done (t >= end_time, max_steps, or a
 * constraint violation); returns ALS_E_CONSTRAINT if any member failed. */
int als_solver_run(als_solver* s);
int als_solver_info(als_solver* s, int member, als_member_info* info);
int als_solver_synchronize(als_solver* s);
/* the stream the solver enqueues on (a cudaStream_t) */
void* als_solver_stream(als_solver* s);
/* Kernel launches a single time step issues (for launch accounting). */
int als_solver_launches_per_step(const als_solver* s);
/* Runs one time step with CUDA events around each kernel (the reference's
 * ALSVINN_TIME_CUDA_BLOCK, alsutils/include/alsutils/timer/CudaTimer.hpp:42-47);
 * kernel_ms[k] receives the duration of kernel k.  Synchronises; returns the
 * number of kernels. */
int als_solver_profile_step(als_solver* s, float* kernel_ms, int capacity);
/* Schedule of the stage launches: blocks_per_sm = 0 launches one block per
 * work item (level, member, tile); k > 0 makes every stage one persistent
 * launch of k resident blocks per SM (capped by what fits) that take work
 * items from a counter.  level_order is the order of the levels in the
 * work list (a permutation, NULL = as created). */
int als_solver_set_schedule(als_solver* s, int blocks_per_sm, const int* level_order);
int als_solver_get_schedule(const als_solver* s, int* blocks_per_sm, int* level_order);
/* Tile shape of each level's stage kernels: 0 is every dimension's default
 * (1-D 256, 2-D 32x16, 3-D 8x8x4 cells); 2-D WENO2 with HLL, HLL3 or
 * Central also has shape 1 (16x16 cells, 288 threads).  Levels of
 * different shapes take one launch per shape and stage.  The shape changes
 * no result.  set returns ALS_E_UNSUPPORTED for a shape not built for the
 * configuration; get fills tile_shapes[level] and tile_extents[3*level + d]
 * (either may be NULL). */
int als_solver_set_tiles(als_solver* s, const int* tile_shapes);
int als_solver_get_tiles(const als_solver* s, int* tile_shapes, int* tile_extents);
/* Autotuner: times `steps` steps per candidate from the same saved state,
 * keeps the fastest and restores the state and member clocks, so results
 * are unchanged.  It searches the tile shape of each level first (one level
 * varied at a time, the others at their best so far), then blocks per SM in
 * {0 (one per item), 1, 2, 3, 4} x level order in {as created, finest
 * first, coarsest first}.  Returns the choice (any out pointer may be NULL)
 * and its ms per step.  This replaces the reference's serial sample loop
 * (alsuq/src/run/Runner.cpp:42-78), which has no schedule to choose. */
int als_solver_tune(als_solver* s, int steps, int* blocks_per_sm, int* level_order,
    int* tile_shapes, double* best_ms_per_step);
/* FP64 sums of every conserved variable over the interior box [lo, hi)
 * (interior cell coordinates; NULL = whole interior) of members
 * [first_member, first_member+count) of one level: out[k*nvar + v].  The
 * conservation check of FP32 members and the observables use it. */
int als_solver_region_sums(als_solver* s, int first_member, int count, const int* lo,
    const int* hi, double* out);

/* ------------------------------------------------ ensemble statistics
 * FP64 mean and variance of an ensemble, accumulated with Welford/Chan
 * updates (mean and M2 per element, merged chunk by chunk), whatever the
 * members' precision.  Replaces alsuq::stats::MeanVariance
 * (alsuq/src/stats/MeanVariance.cpp:30-67, raw sums S1, S2 and
 * var = S2/M - (S1/M)^2) and StatisticsHelper::combineStatistics
 * (alsuq/src/stats/StatisticsHelper.cpp:35-79).  The variance is the biased
 * one (divided by M), like the reference. */
typedef struct als_stats als_stats;
int als_stats_create(long long count, int device, als_stats** out);
int als_stats_destroy(als_stats* st);
/* Adds `members` states (each `count` elements, `member_stride` apart) in
 * ALS_FP64 or ALS_FP32 from device memory. */
int als_stats_add(als_stats* st, const void* states, int precision, int members,
    long long member_stride, void* stream);
/* Adds the current state of every member of a solver level. */
int als_stats_add_solver(als_stats* st, als_solver* s, int level);
/* Chan merge of another accumulator's (n, mean, M2) (device arrays), e.g.
 * from another GPU. */
int als_stats_merge(als_stats* st, long long n, const double* mean, const double* m2, void* stream);
/* n and device pointers of the running mean and M2. */
int als_stats_moments(als_stats* st, long long* n, double** mean, double** m2);
/* Writes mean and variance (device arrays of `count` doubles; either may be NULL). */
int als_stats_result(als_stats* st, double* mean, double* variance, void* stream);

/* ------------------------------------------------------------- output
 * Snapshot files with the layout of alsfvm::io::NetCDFWriter
 * (alsfvm/src/io/NetCDFWriter.cpp:32-146) in the classic NetCDF format
 * (version 2, 64-bit offsets; the reference writes NetCDF-4 through
 * libnetcdf, which readers open alike): dimensions t = 1, x, y, z; a double
 * variable "time"; one double variable per conserved variable with
 * dimensions (x, y, z) holding the interior cells in the order
 * Volume::copyInternalCells gives them (x fastest); global text attributes.
 * `interior` holds nvar host arrays of n[0]*n[1]*n[2] doubles (1 for
 * inactive directions). */
int als_write_netcdf(const char* path, int dimension, const int* n, int nvar,
    const char* const* names, const double* const* interior, double time, int nattr,
    const char* const* attr_names, const char* const* attr_values);
/* The current state of one member, its time and the reference's variable
 * names (rho, mx, [my, [mz,]] E) into <basename>_<snapshot>.nc
 * (alsfvm/src/io/io_utils.cpp:34-40). */
int als_solver_write_netcdf(als_solver* s, int member, const char* basename, int snapshot);

/* ------------------------------------------------- structure functions
 * Structure-function statistics of `members` states (device memory, FP64
 * or FP32, `member_stride` elements apart, dimension+2 padded planes each)
 * into out (device, FP64): out[(member*nvar + var)*H + h].
 *   ALS_STRUCTURE_CUBE  - alsuq/src/stats/StructureCube.cpp:39-75 and
 *     alsfvm/src/functional/StructureCube.cpp via
 *     alsfvm/include/alsfvm/functional/structure_common.hpp:39-160:
 *     sum over cells and over the cube surface at distance h = 1..H-1 of
 *     |u - u_h|^p / (nx*ny*nz); out[.., 0] = 0.
 *   ALS_STRUCTURE_BASIC - alsuq/src/stats/StructureBasic.cpp:74-118: the
 *     point h cells along `direction`, h = 0..H-1.
 * Points outside the interior wrap (ALS_BC_PERIODIC) or clamp
 * (ALS_BC_NEUMANN) as in ValueAtBoundary.hpp:20-110.  H <= 512.  Sums are
 * FP64 in a fixed order; they equal the reference's sequential sums to
 * rounding.  Stream-ordered. */
#define ALS_STRUCTURE_CUBE 0
#define ALS_STRUCTURE_BASIC 1
int als_structure_functions(const als_grid* grid, int boundary, int kind, int direction, int H,
    double p, const void* states, int precision, long long member_stride, int members,
    double* out, void* stream);

/* ------------------------------------------------------- functionals
 * Functional::operator()(out, U, weight, grid) (alsfvm/src/functional/,
 * Functional.hpp:41-60): out += weight * f(U), batched over `members`
 * states (`states` + m * member_stride elements, nvar padded planes of
 * `precision` each; ghosts as `grid`).  Results are FP64, per member
 * nvar blocks of als_functional_size elements (out + m * out_member_stride):
 *   IDENTITY            interior cells, x fastest        (Identity.cpp:25-48)
 *   MOMENT              padded cells, U^degree          (Moment.cpp:27-37)
 *   LOG_ENTROPY         1 value, in the energy block     (LogEntropy.cpp:30-80)
 *   LEGENDRE            1 value per variable, 2-D        (Legendre.cpp:36-98)
 *   LEGENDRE_POINTWISE  interior cells, 2-D              (LegendrePointWise.cpp:32-87)
 *   BV                  1 value per variable, 1-D/2-D    (BoundedVariation.cpp:24-52)
 *   BV_DIRECTION        1 value per variable: sum |u(x) - u(x - e_d)|^degree
 *                       (alsuq BoundedVariationDirection.cpp:35-70,
 *                       HostMemory::getTotalVariation(direction, ...))
 *   STRUCTURE_2PT       number_of_h^2 values per variable (h1 fastest):
 *                       sum (u(x+h1 e) - u)^2 (u(x+h2 e) - u) / cells, shifts
 *                       clamped at the last cell (alsuq StructureTwoPoints.cpp:48-92)
 * Cell midpoints and volumes follow Grid.cpp:24-41 (a direction with one
 * cell has length 1).  Sums over cells are reduced in a fixed order
 * (deterministic; equal to the reference's sequential sums to rounding).
 * The Legendre polynomials are boost::math::legendre_p's recurrence in FP64
 * (the reference's Boost evaluates it in long double: values agree to a few
 * units of 2^-52), a negative degree l taken as -l - 1; an argument outside
 * [-1, 1], Boost's domain error in the reference, is evaluated here.
 * Stream-ordered. */
#define ALS_FUNCTIONAL_IDENTITY 0            /* "identity" */
#define ALS_FUNCTIONAL_MOMENT 1              /* "moment" */
#define ALS_FUNCTIONAL_LOG_ENTROPY 2         /* "log_entropy" */
#define ALS_FUNCTIONAL_LEGENDRE 3            /* "legendre" */
#define ALS_FUNCTIONAL_LEGENDRE_POINTWISE 4  /* "legendre_pointwise" */
#define ALS_FUNCTIONAL_BV 5                  /* "bv" */
#define ALS_FUNCTIONAL_BV_DIRECTION 6        /* alsuq statistic "bv_direction" */
#define ALS_FUNCTIONAL_STRUCTURE_2PT 7       /* alsuq statistic "structure_2pt" */
typedef struct {
    int degree;                        /* moment, legendre_pointwise, bv (the power p) */
    int degree_k, degree_n, degree_m;  /* legendre: x, y and value degrees */
    double min_value, max_value;       /* legendre*: value scaled to (u - min)/(max - min) */
    double gamma;                      /* log_entropy */
    double lower[3], upper[3];         /* domain corners (Grid origin and top) */
    int direction;                     /* bv_direction, structure_2pt (its direction1) */
    int number_of_h;                   /* structure_2pt */
} als_functional_params;
/* elements per variable; STRUCTURE_2PT needs params (its number_of_h) */
int als_functional_size2(const als_grid* grid, int kind, const als_functional_params* params,
    long long* elements_per_variable);
int als_functional_size(const als_grid* grid, int kind, long long* elements_per_variable);
int als_functional(const als_grid* grid, int kind, const als_functional_params* params,
    const void* states, int precision, long long member_stride, int members, double* out,
    long long out_member_stride, double weight, void* stream);

/* ------------------------------------------------------- TeCNO diffusion
 * DiffusionOperator for the Euler equations: TecnoDiffusionCPU with the Roe
 * or Rusanov diffusion matrix over a TeCNO reconstruction of the scaled
 * entropy variables (alsfvm/src/diffusion/TecnoDiffusionCPU.cpp:23-170,
 * DiffusionFactory.cpp:41-95, reconstruction/tecno/).  FP64. */
#define ALS_DIFFUSION_TECNOROE 0        /* "tecnoroe",     diffusion/RoeMatrix.hpp */
#define ALS_DIFFUSION_TECNORUSANOV 1    /* "tecnorusanov", diffusion/RusanovMatrix.hpp */
#define ALS_TECNO_RECON_NONE 0          /* "none", reconstruction/tecno/NoReconstruction */
#define ALS_TECNO_RECON_ENO2 2          /* "eno2", reconstruction/tecno/ENOCPU<2> */
#define ALS_TECNO_RECON_ENO3 3          /* "eno3" */
#define ALS_TECNO_RECON_ENO4 4          /* "eno4" */
typedef struct als_diffusion als_diffusion;

/* Ghost cells the operator needs (1 for none, the order for ENO); replaces
 * TecnoDiffusionCPU::getNumberOfGhostCells (TecnoDiffusionCPU.cpp:172-176).
 * A simulation's planes carry max(this, als_ghost_cells(flux, recon))
 * (ConservedSystem.cpp:109-114). */
int als_diffusion_ghost_cells(int reconstruction);

/* One operator for planes of `grid` (grid->ghosts >= the operator's ghost
 * cells) on the current device.  It owns work arrays that persist between
 * calls like the reference's work volumes, whose entries the reference
 * partly reads before writing; results depend on earlier calls in the same
 * way.  Replaces DiffusionFactory::createDiffusionOperator. */
int als_diffusion_create(const als_grid* grid, int kind, int reconstruction, als_diffusion** out);

/* out += the diffusion of `conserved` (nvar device planes each, ghosts
 * filled), on every cell the reference updates (ghost cells included,
 * which a later boundary fill overwrites).  Replaces
 * DiffusionOperator::applyDiffusion(output, conservedVolume).  Stream-ordered;
 * calls on one operator must not overlap. */
int als_diffusion_apply(als_diffusion* h, const double* const* conserved, double* const* out,
    void* stream);
int als_diffusion_destroy(als_diffusion* h);

/* ------------------------------------------------------- UQ sampling
 * Parameter draws of samples [first_sample, first_sample+count) for a
 * parameter of length `dimension`: out[k*dimension + c].  Same numbers as
 * alsuq's STLMersenne generator with a Uniform(lower, upper) distribution
 * (alsuq/src/generator/STLMersenne.cpp:38-85, alsuq/src/distribution/Uniform.cpp:27-34,
 * alsuq/src/samples/SampleGenerator.cpp:29-56).  Host-only. */
int als_uniform_draws(long long dimension, long long first_sample, long long count,
    double lower, double upper, double* out);

#ifdef __cplusplus
}
#endif
#endif
