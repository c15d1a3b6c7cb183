// Structures shared by the host driver and the stage kernels.
#pragma once

#include <cstdint>

namespace als {

enum Kind {
    KIND_FLUX0 = 0,   // out = L(U^n) (unscaled net flux), face wave speeds reduced
    KIND_RK2_1 = 1,   // U1 = c*L + U^n on load; out = ((c*L(U1) + U1) + U^n) * 0.5
    KIND_RK3_1 = 2,   // U1 = c*L + U^n on load; out = ((c*L(U1) + U1) * 1/3 + U^n) * 3/4
    KIND_RK3_2 = 3,   // out(in place over U^n) = ((c*L(U2) + U2) * 2 + U^n) * 1/3
};

enum Boundary { BC_NEUMANN = 0, BC_PERIODIC = 1 };

constexpr int kMaxVars = 5;
constexpr int kMaxLevels = 4;

// Per-simulation time-stepping state kept on the device, so a whole time
// step runs without a host round trip.  One per ensemble member.
struct alignas(64) StepState {
    double t;                       // current time
    double dt;                      // dt of the step in flight
    double end_time;                // T
    double cfl;
    unsigned long long ws[3];       // max face wave speed per direction (bit pattern of a non-negative double)
    long long steps;                // completed time steps
    long long max_steps;
    int done;                       // 1 once t >= T, max_steps reached or a constraint failed
    int status;                     // 0 ok, 1 constraint violation
    unsigned int arrive;            // tiles of the last stage that finished (last-tile bookkeeping)
    unsigned int pad0;
    long long bad_index;            // first padded cell index that violated a constraint
    long long bad_step;             // step number at which it happened
    double dx[3];                   // cell lengths (1 for inactive directions)
    double pad1[3];
};

// Geometry of one grid (one multilevel level, or the single grid).
struct GridDesc {
    int n[3];          // interior cells (1 for inactive directions)
    int N[3];          // padded extents
    int tiles[3];      // tiles covering the region [lo, hi)
    int lo[3], hi[3];  // region of interior cells to update (interior coordinates)
    long long plane;   // padded cells per plane
    int ghosts;        // ghost width of the planes (>= the stencil's)
};

// One grid level of a launch: its geometry, its planes (one pointer per
// conserved variable, member 0; member m is m*member_stride elements
// further), its members and their states.
struct LevelDesc {
    GridDesc grid;
    const void* in[kMaxVars];   // stencil input: U^n (FLUX0), L (RK*_1), U2 (RK3_2)
    const void* un[kMaxVars];   // U^n (RK*_1 and RK3_2); may alias `out` for RK3_2
    void* out[kMaxVars];
    long long member_stride;
    StepState* state;           // member 0's state, or null for plug-in calls
    unsigned long long* ws_out; // FLUX0 without state: 3 maxima per member
    int members;
    int tiles_per_member;
    long long work_begin;       // first work item of this level in the launch
    // Subdomains of one grid split over procs[0] x procs[1] x procs[2]
    // members (member = x + procs[0] (y + procs[1] z)): they share state 0
    // (one dt, one wave-speed maximum), and each updated cell also writes
    // its images into the neighbouring members' ghost cells.  0: members
    // are independent simulations.
    int subdomains;
    int procs[3];
};

// A launch walks a list of work items (level, member, tile): levels one
// after another, members one after another, tiles of a member together.
struct StageParams {
    LevelDesc level[kMaxLevels];
    int nlevels;
    long long total_work;
    int bc;                  // BC_NEUMANN / BC_PERIODIC
    int write_ghosts;        // 1: also write the boundary images of every updated cell
    double gamma;
    double c_fixed;          // dt/dx for stages when a level has no state
    unsigned long long* counter; // persistent mode: [next item, blocks done], zero between launches; null: one item per block
};

} // namespace als
