/*
 * CPU restatement of alsfvm's cell-update hot path, written in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU path is compared
 * against; it is never linked into, loaded by or called from the product
 * library.  Only tests/, the smoke check and bench.py's CPU-baseline leg
 * may use it.  It is pinned bit-for-bit against the reference's own CPU
 * sources (oracle/_ref/libalsref.so, built by `make -C oracle ref`) by
 * tests/test_oracle_pin.py and against committed fixtures in tests/golden/.
 *
 * Data layout (same as alsfvm::volume::Volume, alsfvm/src/volume/Volume.cpp:44-60):
 * one contiguous plane of doubles per conserved variable, each plane
 * (nx+2g)*(ny+2g)*(nz+2g) cells with x fastest, inactive dimensions have
 * extent 1 and no ghost cells.  Variable order rho, mx, [my, [mz,]] E
 * (alsfvm/src/equation/euler/Euler.cpp:20-75).
 */
#ifndef ALS_ORACLE_H
#define ALS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_FLUX_HLL = 0, ORC_FLUX_HLL3 = 1, ORC_FLUX_CENTRAL = 2, ORC_FLUX_TECNO1 = 3,
       ORC_FLUX_TECNO4 = 4, ORC_FLUX_TECNO6 = 5 };
enum { ORC_RECON_NONE = 0, ORC_RECON_WENO2 = 1, ORC_RECON_ENO2 = 2,
       ORC_RECON_ENO3 = 3, ORC_RECON_ENO4 = 4, ORC_RECON_MC = 5, ORC_RECON_MM = 6,
       ORC_RECON_WENOF2 = 7, ORC_RECON_WENO3 = 8 };
enum { ORC_INT_FE = 0, ORC_INT_RK2 = 1, ORC_INT_RK3 = 2, ORC_INT_RK4 = 3 };
enum { ORC_BC_NEUMANN = 0, ORC_BC_PERIODIC = 1 };

typedef struct {
    int dim;          /* 1, 2 or 3 */
    int n[3];         /* interior cells per direction (1 for inactive) */
    int g;            /* ghost width */
    double gamma;
    int flux, recon, integrator, bc;
    double dx[3];     /* cell lengths; 1 for inactive directions */
    int diffusion;    /* -1 none, 0 tecnoroe, 1 tecnorusanov (orc_set_diffusion) */
    int diffusion_recon;
} orc_config;

/* Ghost width max(stencil-1, reconstruction ghosts), NumericalFluxCPU.cpp:227-231. */
int orc_ghost_cells(int flux, int recon);

/* Fills cfg->g, cell lengths from the domain [lower, upper], Grid.cpp:24-41. */
int orc_configure(orc_config* cfg, int dim, const int* n, const double* lower,
    const double* upper, int flux, int recon, int integrator, int bc, double gamma);

long orc_plane_size(const orc_config* cfg);

/* Ghost-cell fill, BoundaryCPU.cpp:30-106 with Neumann.hpp:24-35 / Periodic.hpp:24-42. */
void orc_fill_ghosts(const orc_config* cfg, double* planes, int nvar);

/* Reconstruction along direction `dir` for every cell the reference
 * reconstructs (ReconstructionCPU.cpp:37-97, ENOCPU.cpp:41-187). */
void orc_reconstruct(const orc_config* cfg, int dir, const double* in,
    double* left, double* right);

/* Net flux of every interior cell (ghost cells untouched) and the maximal
 * face wave speed per direction (NumericalFluxCPU.cpp:32-221). */
void orc_net_flux(const orc_config* cfg, const double* in, double* out, double ws[3]);

/* The Simulator time loop with an end-time clamp (Simulator.cpp:191-214,
 * Integrator.cpp:20-46, FixedIntervalWriter.cpp:45-53).  `planes` holds the
 * initial state (ghosts are filled first) and receives the final state.
 * Returns 0, 1 on a constraint violation, -1 on bad arguments. */
int orc_simulate(const orc_config* cfg, double cfl, double end_time, long max_steps,
    double* planes, double* dts, long dts_capacity, long* steps_out, double* t_out);

/* MeanVariance with raw moments (MeanVariance.cpp:30-67): mean = S1/M,
 * var = S2/M - mean^2, over `samples` states of `count` doubles each. */
void orc_meanvar(long count, long samples, const double* states, double* mean, double* var);

/* Structure functions of each of `nvar` padded planes (ghost width g on the
 * active sides).  Cube (alsfvm/include/alsfvm/functional/structure_common.hpp:39-160,
 * used by alsuq/src/stats/StructureCube.cpp:39-75 and
 * alsfvm/src/functional/StructureCube.cpp): out[v*H + h] = sum over cells and
 * over the points of the cube surface at distance h (h = 1..H-1) of
 * |u - u_h|^p / (nx*ny*nz), FastPower for p = 1..5, pow otherwise.
 * Basic (alsuq/src/stats/StructureBasic.cpp:74-118): the single point
 * h steps along `direction`, h = 0..H-1, pow always.  Points outside the
 * interior wrap (periodic) or clamp (Neumann), ValueAtBoundary.hpp:20-110. */
void orc_structure_cube(int dim, const int* n, int g, int bc, int nvar, int H, double p,
    const double* planes, double* out);
void orc_structure_basic(int dim, const int* n, int g, int bc, int nvar, int direction, int H,
    double p, const double* planes, double* out);

/* Constraint check of CPUCellComputer::obeysConstraints (CPUCellComputer.cpp:80-128)
 * over all cells; returns 1 when every cell obeys. */
int orc_obeys_constraints(const orc_config* cfg, const double* planes);

/* Functionals (alsfvm/src/functional/): out += weight * f(U) for one state,
 * sums in the reference's sequential order.  Output per variable:
 * orc_functional_size elements (interior cells, padded cells or 1).
 * Returns 0, -1 for a functional the reference does not define on the grid,
 * -2 when a Legendre argument left [-1, 1] (boost::math::legendre_p's
 * domain error, an exception in the reference). */
enum { ORC_FUNCTIONAL_IDENTITY = 0, ORC_FUNCTIONAL_MOMENT = 1, ORC_FUNCTIONAL_LOG_ENTROPY = 2,
       ORC_FUNCTIONAL_LEGENDRE = 3, ORC_FUNCTIONAL_LEGENDRE_POINTWISE = 4, ORC_FUNCTIONAL_BV = 5,
       ORC_FUNCTIONAL_BV_DIRECTION = 6, ORC_FUNCTIONAL_STRUCTURE_2PT = 7 };
typedef struct {
    int degree, degree_k, degree_n, degree_m;
    double min_value, max_value, gamma;
    double lower[3], upper[3];
    int direction, number_of_h;
} orc_functional_params;
long orc_functional_size(int dim, const int* n, int g, int kind, int number_of_h);
int orc_functional(int dim, const int* n, int g, int kind, const orc_functional_params* p,
    const double* planes, double* out, double weight);

/* TeCNO diffusion, TecnoDiffusionCPU::applyDiffusion (TecnoDiffusionCPU.cpp:
 * 23-170): kind 0 tecnoroe (RoeMatrix), 1 tecnorusanov (RusanovMatrix);
 * recon 0 none, 2/3/4 ENO of that order (reconstruction/tecno/).  Adds the
 * diffusion to `out` (every cell the reference touches, ghosts included).
 * `state` holds the operator's persistent work arrays: four volumes
 * (scaled entropy variables left/right, their reconstructions left/right;
 * 4 * nvar planes), which the caller fills with 42 once, as HostMemory does
 * (HostMemory.cpp:36-37), then the ENO's three difference planes, filled
 * with 0 (ENOCPU.cpp:27-33, 196-203).  The caller keeps them between calls:
 * the reference reads entries its passes do not write (the last cells along
 * each direction), so results depend on what earlier calls, directions and
 * variables left there. */
int orc_diffusion_ghost_cells(int recon);

/* Adds a TeCNO diffusion operator to the system of orc_simulate
 * (ConservedSystem.cpp:102) and widens cfg->g to
 * max(flux ghosts, diffusion ghosts) (ConservedSystem.cpp:109-114). */
int orc_set_diffusion(orc_config* cfg, int kind, int recon);
void orc_diffusion_apply(const orc_config* cfg, int kind, int recon, double* state,
    const double* U, double* out);

#ifdef __cplusplus
}
#endif
#endif
