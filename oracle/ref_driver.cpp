// Test oracle driver around the reference's own CPU implementation.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// unmodified reference sources (see oracle/Makefile) into oracle/_ref/libalsref.so.
// Only tests/, the smoke check and bench.py's CPU-baseline leg may load it,
// and only as the checker or the timed CPU baseline, never as the product.
//
// What it reproduces (reference file:line):
//  * Simulator::incrementSolution            alsfvm/src/simulator/Simulator.cpp:191-214
//  * Simulator::atEnd / checkConstraints      alsfvm/src/simulator/Simulator.cpp:77-79,180-189
//  * FixedIntervalWriter::adjustTimestep with one save at T
//                                             alsfvm/src/io/FixedIntervalWriter.cpp:45-53
//  * MeanVariance compute/combine/finalize    alsuq/src/stats/MeanVariance.cpp:30-67,
//                                             alsuq/src/stats/StatisticsHelper.cpp:35-79
//  * STLMersenne sample draws                 alsuq/src/generator/STLMersenne.cpp:38-85
//  * Statistics by name, combined, finalized and written as the UQ runner
//    does it                                  alsuq/src/run/Runner.cpp:80-87
//  * Functionals by name, output allocated as TimeIntegrationFunctional does
//                                             alsfvm/src/functional/TimeIntegrationFunctional.cpp:64-72
// All arithmetic is done by the reference's own classes; this file only wires
// them together and copies planes in and out.
#include "alsfvm/types.hpp"
#include "alsfvm/grid/Grid.hpp"
#include "alsfvm/boundary/BoundaryCPU.hpp"
#include "alsfvm/boundary/Neumann.hpp"
#include "alsfvm/boundary/Periodic.hpp"
#include "alsfvm/numflux/NumericalFluxCPU.hpp"
#include "alsfvm/numflux/euler/HLL.hpp"
#include "alsfvm/numflux/euler/HLL3.hpp"
#include "alsfvm/numflux/Central.hpp"
#include "alsfvm/numflux/TecnoCombined4.hpp"
#include "alsfvm/numflux/TecnoCombined6.hpp"
#include "alsfvm/numflux/euler/Tecno1.hpp"
#include "alsfvm/reconstruction/ReconstructionCPU.hpp"
#include "alsfvm/reconstruction/WENO2.hpp"
#include "alsfvm/reconstruction/MC.hpp"
#include "alsfvm/reconstruction/MM.hpp"
#include "alsfvm/reconstruction/WENOF2.hpp"
#include "alsfvm/reconstruction/WENOCPU.hpp"
#include "alsfvm/reconstruction/ENOCPU.hpp"
#include "alsfvm/reconstruction/NoReconstruction.hpp"
#include "alsfvm/integrator/ForwardEuler.hpp"
#include "alsfvm/integrator/RungeKutta2.hpp"
#include "alsfvm/integrator/RungeKutta3.hpp"
#include "alsfvm/integrator/RungeKutta4.hpp"
#include "alsfvm/integrator/TimestepAdjuster.hpp"
#include "alsfvm/simulator/ConservedSystem.hpp"
#include "alsfvm/simulator/SimulatorParameters.hpp"
#include "alsfvm/simulator/TimestepInformation.hpp"
#include "alsfvm/diffusion/NoDiffusion.hpp"
#include "alsfvm/diffusion/TecnoDiffusionCPU.hpp"
#include "alsfvm/diffusion/RoeMatrix.hpp"
#include "alsfvm/diffusion/RusanovMatrix.hpp"
#include "alsfvm/reconstruction/tecno/ENOCPU.hpp"
#include "alsfvm/reconstruction/tecno/NoReconstruction.hpp"
#include "alsfvm/volume/VolumeFactory.hpp"
#include "alsfvm/memory/MemoryFactory.hpp"
#include "alsfvm/equation/euler/EulerParameters.hpp"
#include "alsfvm/equation/CPUCellComputer.hpp"
#include "alsfvm/DeviceConfiguration.hpp"
#include "alsuq/generator/STLMersenne.hpp"
#include "alsfvm/functional/structure_common.hpp"
#include "alsfvm/functional/FunctionalFactory.hpp"
#include "alsfvm/io/Writer.hpp"
#include "alsuq/stats/StatisticsFactory.hpp"
#include "alsuq/stats/StatisticsParameters.hpp"
#include "alsuq/stats/stats_util.hpp"
#ifdef ALSREF_WITH_B200
#include "adapter/NumericalFluxB200.hpp"
#include "adapter/B200Adapters.hpp"
#include "adapter/StatisticsB200.hpp"
#endif

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace alsfvm;

namespace {

std::string g_last_error;
double g_last_loop_seconds = 0;

struct Setup {
    int dim;
    ivec3 n;
    rvec3 lower, upper;
    std::string flux, recon, integrator, bc;
    double gamma, cfl;
};

// Stops the step that would pass the end time, like a FixedIntervalWriter
// whose only save is at T (FixedIntervalWriter.cpp:45-53).
class EndTimeClamp : public integrator::TimestepAdjuster {
public:
    explicit EndTimeClamp(real endTime) : endTime(endTime) {}
    real adjustTimestep(real dt,
        const simulator::TimestepInformation& info) const override {
        return std::min(dt, endTime - info.getCurrentTime());
    }
private:
    real endTime;
};

struct Objects {
    std::shared_ptr<DeviceConfiguration> device;
    std::shared_ptr<memory::MemoryFactory> memoryFactory;
    std::shared_ptr<simulator::SimulatorParameters> params;
    std::shared_ptr<grid::Grid> grid;
    std::shared_ptr<reconstruction::Reconstruction> recon;
    std::shared_ptr<numflux::NumericalFlux> flux;
    std::shared_ptr<integrator::System> system;
    std::shared_ptr<diffusion::DiffusionOperator> diffusion;
    std::shared_ptr<integrator::Integrator> integ;
    std::shared_ptr<boundary::Boundary> boundary;
    std::shared_ptr<volume::VolumeFactory> volumeFactory;
    size_t ghosts = 0;
    std::string eqName;
};

// Diffusion operator of the next builds: "none" or "tecnoroe" /
// "tecnorusanov" over the TeCNO reconstruction g_diffusion_recon
// ("none", "eno2", "eno3", "eno4"), as DiffusionFactory.cpp:41-95 builds them.
std::string g_diffusion = "none";
std::string g_diffusion_recon = "none";

#ifdef ALSREF_WITH_B200
extern std::string g_flux_platform;
#endif

template<int d>
std::shared_ptr<diffusion::DiffusionOperator> makeDiffusion(const Setup& s, Objects& o) {
    typedef equation::euler::Euler<d> Eq;
    if (g_diffusion == "none") {
        return std::make_shared<diffusion::NoDiffusion>();
    }
#ifdef ALSREF_WITH_B200
    if (g_flux_platform == "b200-all") {
        const int kind = g_diffusion == "tecnoroe" ? ALS_DIFFUSION_TECNOROE : ALS_DIFFUSION_TECNORUSANOV;
        const int rec = g_diffusion_recon == "none" ? ALS_TECNO_RECON_NONE
            : (g_diffusion_recon == "eno2" ? ALS_TECNO_RECON_ENO2
            : (g_diffusion_recon == "eno3" ? ALS_TECNO_RECON_ENO3 : ALS_TECNO_RECON_ENO4));
        return std::make_shared<b200::DiffusionB200>(d, kind, rec, s.gamma);
    }
#endif
    std::shared_ptr<reconstruction::tecno::TecnoReconstruction> rec;
    if (g_diffusion_recon == "none") {
        rec = std::make_shared<reconstruction::tecno::NoReconstruction>();
    } else if (g_diffusion_recon == "eno2") {
        rec = std::make_shared<reconstruction::tecno::ENOCPU<2>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else if (g_diffusion_recon == "eno3") {
        rec = std::make_shared<reconstruction::tecno::ENOCPU<3>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else if (g_diffusion_recon == "eno4") {
        rec = std::make_shared<reconstruction::tecno::ENOCPU<4>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else {
        THROW("unknown diffusion reconstruction " << g_diffusion_recon);
    }
    if (g_diffusion == "tecnoroe") {
        return std::make_shared<diffusion::TecnoDiffusionCPU<Eq, diffusion::RoeMatrix>>(
            *o.volumeFactory, rec, *o.params);
    } else if (g_diffusion == "tecnorusanov") {
        return std::make_shared<diffusion::TecnoDiffusionCPU<Eq, diffusion::RusanovMatrix>>(
            *o.volumeFactory, rec, *o.params);
    }
    THROW("unknown diffusion " << g_diffusion);
}

#ifdef ALSREF_WITH_B200
// Flux platform of the next builds: "cpu" (the reference's NumericalFluxCPU)
// or "b200" (numflux::NumericalFluxB200 over the B200 library).
std::string g_flux_platform = "cpu";

int b200_code(const std::string& name, const char* const* names, int count) {
    for (int i = 0; i < count; ++i) {
        if (name == names[i]) {
            return i;
        }
    }
    THROW("no B200 code for " << name);
}
#endif

template<int d>
std::shared_ptr<reconstruction::Reconstruction> makeRecon(const Setup& s, Objects& o) {
    typedef equation::euler::Euler<d> Eq;
#ifdef ALSREF_WITH_B200
    if (g_flux_platform == "b200-parts") {
        // the reference's NumericalFluxCPU over the B200 reconstruction
        static const char* const recons[] = {"none", "weno2", "eno2", "eno3", "eno4", "mc", "mm",
            "wenof2", "weno3"};
        return std::make_shared<b200::ReconstructionB200>(d, b200_code(s.recon, recons, 9), s.gamma);
    }
#endif
    if (s.recon == "weno2") {
        return std::make_shared<reconstruction::ReconstructionCPU<reconstruction::WENO2<Eq>, Eq>>(*o.params);
    } else if (s.recon == "eno2") {
        return std::make_shared<reconstruction::ENOCPU<2>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else if (s.recon == "eno3") {
        return std::make_shared<reconstruction::ENOCPU<3>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else if (s.recon == "eno4") {
        return std::make_shared<reconstruction::ENOCPU<4>>(o.memoryFactory, s.n.x, s.n.y, s.n.z);
    } else if (s.recon == "mc") {
        return std::make_shared<reconstruction::ReconstructionCPU<reconstruction::MC<Eq>, Eq>>(*o.params);
    } else if (s.recon == "weno3") {
        return std::make_shared<reconstruction::WENOCPU<3>>();
    } else if (s.recon == "wenof2") {
        return std::make_shared<reconstruction::ReconstructionCPU<reconstruction::WENOF2<Eq>, Eq>>(*o.params);
    } else if (s.recon == "mm") {
        return std::make_shared<reconstruction::ReconstructionCPU<reconstruction::MM<Eq>, Eq>>(*o.params);
    } else if (s.recon == "none") {
        return std::make_shared<reconstruction::NoReconstruction>();
    }
    THROW("unknown reconstruction " << s.recon);
}


template<int d>
std::shared_ptr<numflux::NumericalFlux> makeFlux(const Setup& s, Objects& o) {
    typedef equation::euler::Euler<d> Eq;
#ifdef ALSREF_WITH_B200
    if (g_flux_platform == "b200" || g_flux_platform == "b200-all") {
        // names in the order of the ALS_FLUX_* / ALS_RECON_* codes
        static const char* const fluxes[] = {"hll", "hll3", "central", "tecno1", "tecno4",
            "tecno6"};
        static const char* const recons[] = {"none", "weno2", "eno2", "eno3", "eno4", "mc", "mm",
            "wenof2", "weno3"};
        return std::make_shared<numflux::NumericalFluxB200>(*o.grid, b200_code(s.flux, fluxes, 6),
            b200_code(s.recon, recons, 9), s.gamma);
    }
#endif
    if (s.flux == "hll") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::euler::HLL<d>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    } else if (s.flux == "hll3") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::euler::HLL3<d>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    } else if (s.flux == "central") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::Central<Eq>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    } else if (s.flux == "tecno1") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::euler::Tecno1<d>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    } else if (s.flux == "tecno4") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::TecnoCombined4<Eq, numflux::euler::Tecno1<d>>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    } else if (s.flux == "tecno6") {
        return std::make_shared<numflux::NumericalFluxCPU<numflux::TecnoCombined6<Eq, numflux::euler::Tecno1<d>>, Eq, d>>(*o.grid, o.recon, o.params, o.device);
    }
    THROW("unknown flux " << s.flux);
}

Objects build(const Setup& s) {
    Objects o;
    o.device = std::make_shared<DeviceConfiguration>("cpu");
    o.memoryFactory = std::make_shared<memory::MemoryFactory>(o.device);
    o.eqName = "euler" + std::to_string(s.dim);
    auto eulerParams = std::make_shared<equation::euler::EulerParameters>();
    eulerParams->setGamma(s.gamma);
    o.params = std::make_shared<simulator::SimulatorParameters>(o.eqName, "cpu");
    o.params->setEquationParameters(eulerParams);
    o.params->setCFLNumber(s.cfl);

    boundary::Type t;
    if (s.bc == "neumann") {
        t = boundary::Type::NEUMANN;
    } else if (s.bc == "periodic") {
        t = boundary::Type::PERIODIC;
    } else {
        THROW("unknown boundary " << s.bc);
    }
    std::array<boundary::Type, 6> bcs = {t, t, t, t, t, t};
    o.grid = std::make_shared<grid::Grid>(s.lower, s.upper, s.n, bcs);

    o.volumeFactory = std::make_shared<volume::VolumeFactory>(o.eqName, o.memoryFactory);
    switch (s.dim) {
    case 1: o.recon = makeRecon<1>(s, o); o.flux = makeFlux<1>(s, o); o.diffusion = makeDiffusion<1>(s, o); break;
    case 2: o.recon = makeRecon<2>(s, o); o.flux = makeFlux<2>(s, o); o.diffusion = makeDiffusion<2>(s, o); break;
    case 3: o.recon = makeRecon<3>(s, o); o.flux = makeFlux<3>(s, o); o.diffusion = makeDiffusion<3>(s, o); break;
    default: THROW("dimension must be 1, 2 or 3");
    }
    o.system = std::make_shared<simulator::ConservedSystem>(o.flux, o.diffusion);
    if (s.integrator == "forwardeuler") {
        o.integ = std::make_shared<integrator::ForwardEuler>(o.system);
    } else if (s.integrator == "rungekutta2") {
        o.integ = std::make_shared<integrator::RungeKutta2>(o.system);
    } else if (s.integrator == "rungekutta3") {
        o.integ = std::make_shared<integrator::RungeKutta3>(o.system);
    } else if (s.integrator == "rungekutta4") {
        o.integ = std::make_shared<integrator::RungeKutta4>(o.system);
    } else {
        THROW("unknown integrator " << s.integrator);
    }
    o.ghosts = o.system->getNumberOfGhostCells();
    if (t == boundary::Type::NEUMANN) {
        o.boundary = std::make_shared<boundary::BoundaryCPU<boundary::Neumann>>(o.ghosts);
    } else {
        o.boundary = std::make_shared<boundary::BoundaryCPU<boundary::Periodic>>(o.ghosts);
    }
#ifdef ALSREF_WITH_B200
    if (g_flux_platform == "b200-parts" || g_flux_platform == "b200-all") {
        // the boundary and the integrator as B200 adapters too
        o.boundary = std::make_shared<b200::BoundaryB200>(
            t == boundary::Type::NEUMANN ? ALS_BC_NEUMANN : ALS_BC_PERIODIC, int(o.ghosts));
        static const char* const integs[] = {"forwardeuler", "rungekutta2", "rungekutta3",
            "rungekutta4"};
        o.integ = std::make_shared<b200::IntegratorB200>(b200_code(s.integrator, integs, 4),
            o.system);
    }
#endif
    return o;
}

Setup makeSetup(int dim, const int* n, const double* lower, const double* upper,
    const char* flux, const char* recon, const char* integ, const char* bc,
    double gamma, double cfl) {
    Setup s;
    s.dim = dim;
    s.n = ivec3(n[0], dim > 1 ? n[1] : 1, dim > 2 ? n[2] : 1);
    s.lower = rvec3(lower[0], lower[1], lower[2]);
    s.upper = rvec3(upper[0], upper[1], upper[2]);
    s.flux = flux ? flux : "";
    s.recon = recon ? recon : "";
    s.integrator = integ ? integ : "rungekutta3";
    s.bc = bc ? bc : "";
    s.gamma = gamma;
    s.cfl = cfl;
    return s;
}

size_t paddedCells(const volume::Volume& v) {
    return v.getTotalNumberOfXCells() * v.getTotalNumberOfYCells() *
        v.getTotalNumberOfZCells();
}

void copyIn(volume::Volume& v, const double* planes) {
    const size_t cells = paddedCells(v);
    for (size_t var = 0; var < v.getNumberOfVariables(); ++var) {
        std::memcpy(v.getScalarMemoryArea(var)->getPointer(), planes + var * cells,
            cells * sizeof(double));
    }
}

void copyOut(const volume::Volume& v, double* planes) {
    const size_t cells = paddedCells(v);
    for (size_t var = 0; var < v.getNumberOfVariables(); ++var) {
        std::memcpy(planes + var * cells, v.getScalarMemoryArea(var)->getPointer(),
            cells * sizeof(double));
    }
}

// An io::Writer that copies the volume it is given (a statistic's result)
// into caller memory.
class CaptureWriter : public io::Writer {
public:
    explicit CaptureWriter(double* out) : out(out) {}
    void write(const volume::Volume& conservedVariables, const grid::Grid&,
        const simulator::TimestepInformation&) override {
        copyOut(conservedVariables, out);
        ++writes;
    }
    double* out;
    int writes = 0;
};

} // namespace

#ifdef ALSREF_WITH_B200
// The B200 statistics registered by name, as a maintainer would in their
// statistics source file.
REGISTER_STATISTICS(b200, meanvar, alsuq::stats::MeanVarianceB200)
#endif

extern "C" {

const char* alsref_last_error() {
    return g_last_error.c_str();
}

// Wall time of the step loop of the last alsref_simulate call (set-up,
// initial boundary fill and copies excluded): the timed CPU baseline.
double alsref_last_loop_seconds() {
    return g_last_loop_seconds;
}

// Ghost width the reference picks for a flux/reconstruction pair
// (NumericalFluxCPU.cpp:227-231).
int alsref_ghost_cells(int dim, const char* flux, const char* recon) {
    try {
        int n[3] = {16, 16, 16};
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, flux, recon, "forwardeuler", "neumann", 1.4, 0.5);
        auto o = build(s);
        return int(o.ghosts);
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// The reference time loop.  `planes` holds nvar padded planes of initial
// conserved data (ghost cells are ignored on input and filled by the
// boundary, Simulator.cpp:161).  On return it holds the final padded state.
// dts[k] receives the dt of step k (up to dts_capacity entries).
// Returns 0, or 1 when the constraint check failed, or -1 on error.
int alsref_simulate(int dim, const int* n, const double* lower, const double* upper,
    const char* flux, const char* recon, const char* integ, const char* bc,
    double gamma, double cfl, double end_time, long max_steps,
    double* planes, double* dts, long dts_capacity,
    long* steps_out, double* t_out) {
    try {
        auto s = makeSetup(dim, n, lower, upper, flux, recon, integ, bc, gamma, cfl);
        auto o = build(s);
        std::shared_ptr<integrator::TimestepAdjuster> clamp =
            std::make_shared<EndTimeClamp>(end_time);
        o.integ->addTimestepAdjuster(clamp);

        std::vector<std::shared_ptr<volume::Volume>> volumes;
        for (size_t i = 0; i < o.integ->getNumberOfSubsteps() + 1; ++i) {
            volumes.push_back(o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, o.ghosts));
        }
        copyIn(*volumes[0], planes);
        o.boundary->applyBoundaryConditions(*volumes[0], *o.grid);

        std::shared_ptr<equation::CellComputer> cellComputer;
        switch (dim) {
        case 1: cellComputer = std::make_shared<equation::CPUCellComputer<equation::euler::Euler<1>>>(*o.params); break;
        case 2: cellComputer = std::make_shared<equation::CPUCellComputer<equation::euler::Euler<2>>>(*o.params); break;
        default: cellComputer = std::make_shared<equation::CPUCellComputer<equation::euler::Euler<3>>>(*o.params); break;
        }

        simulator::TimestepInformation info;
        int status = 0;
        long steps = 0;
        const auto loop_start = std::chrono::steady_clock::now();
        while (info.getCurrentTime() < end_time && steps < max_steps) {
            real dt = 0;
            for (size_t substep = 0; substep < o.integ->getNumberOfSubsteps(); ++substep) {
                auto& next = volumes[substep + 1];
                dt = o.integ->performSubstep(volumes, o.grid->getCellLengths(), dt,
                        s.cfl, *next, substep, info);
                o.boundary->applyBoundaryConditions(*next, *o.grid);
            }
            volumes[0].swap(volumes.back());
            info.incrementTime(dt);
            if (steps < dts_capacity && dts) {
                dts[steps] = dt;
            }
            ++steps;
            if (!cellComputer->obeysConstraints(*volumes[0])) {
                status = 1;
                break;
            }
        }
        g_last_loop_seconds = std::chrono::duration<double>(
            std::chrono::steady_clock::now() - loop_start).count();
        copyOut(*volumes[0], planes);
        if (steps_out) {
            *steps_out = steps;
        }
        if (t_out) {
            *t_out = info.getCurrentTime();
        }
        return status;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// One spatial-operator evaluation: ConservedSystem::operator()
// (ConservedSystem.cpp:31-103) on a state whose ghost cells are filled by the
// boundary first.  out_planes receives the net flux (interior cells; ghost
// cells are left zero), ws the per-direction maximal wave speeds.
int alsref_compute_flux(int dim, const int* n, const double* lower, const double* upper,
    const char* flux, const char* recon, const char* bc, double gamma,
    double* in_planes, double* out_planes, double* ws) {
    try {
        auto s = makeSetup(dim, n, lower, upper, flux, recon, "forwardeuler", bc, gamma, 0.5);
        auto o = build(s);
        auto in = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, o.ghosts);
        auto out = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, o.ghosts);
        copyIn(*in, in_planes);
        o.boundary->applyBoundaryConditions(*in, *o.grid);
        out->makeZero();
        rvec3 waveSpeed(0, 0, 0);
        (*o.system)(*in, waveSpeed, true, *out);
        copyOut(*in, in_planes);
        copyOut(*out, out_planes);
        ws[0] = waveSpeed.x;
        ws[1] = waveSpeed.y;
        ws[2] = waveSpeed.z;
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Reconstruction::performReconstruction along `direction` on a state whose
// ghost cells are taken as given (no boundary applied).
int alsref_reconstruct(int dim, const int* n, const char* recon, double gamma,
    int direction, const double* in_planes, double* left, double* right) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", recon, "forwardeuler", "neumann", gamma, 0.5);
        auto o = build(s);
        const size_t g = o.recon->getNumberOfGhostCells();
        auto in = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, g);
        auto l = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, g);
        auto r = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, g);
        copyIn(*in, in_planes);
        l->makeZero();
        r->makeZero();
        o.recon->performReconstruction(*in, direction, 0, *l, *r);
        copyOut(*l, left);
        copyOut(*r, right);
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Boundary::applyBoundaryConditions on nvar padded planes with ghost width g.
int alsref_apply_boundary(int dim, const int* n, int ghosts, const char* bc,
    double* planes) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", bc, 1.4, 0.5);
        auto o = build(s);
        auto v = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        copyIn(*v, planes);
        std::shared_ptr<boundary::Boundary> b;
        if (s.bc == "neumann") {
            b = std::make_shared<boundary::BoundaryCPU<boundary::Neumann>>(ghosts);
        } else {
            b = std::make_shared<boundary::BoundaryCPU<boundary::Periodic>>(ghosts);
        }
        b->applyBoundaryConditions(*v, *o.grid);
        copyOut(*v, planes);
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// MeanVariance over `samples` padded states of one volume shape
// (MeanVariance.cpp:30-67 with StatisticsHelper.cpp:74 `/= samples`).
int alsref_meanvar(int dim, const int* n, int ghosts, long samples,
    const double* states, double* mean_out, double* var_out) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", "neumann", 1.4, 0.5);
        auto o = build(s);
        auto u = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        auto mean = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        auto var = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        mean->makeZero();
        var->makeZero();
        const size_t stride = paddedCells(*u) * u->getNumberOfVariables();
        for (long k = 0; k < samples; ++k) {
            copyIn(*u, states + k * stride);
            *mean += *u;
            var->addPower(*u, 2);
        }
        for (size_t v = 0; v < u->getNumberOfVariables(); ++v) {
            *mean->getScalarMemoryArea(v) /= real(samples);
            *var->getScalarMemoryArea(v) /= real(samples);
        }
        var->subtractPower(*mean, 2.);
        copyOut(*mean, mean_out);
        copyOut(*var, var_out);
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Parameter draws of samples [first, first+count) for a parameter of length
// `dimension` (STLMersenne.cpp:38-85): out[k*dimension + c].
// The generator is a process-wide singleton in the reference, so this must
// be called with increasing sample numbers within one process.
int alsref_stlmersenne(long dimension, long first, long count, double* out) {
    try {
        alsuq::generator::STLMersenne gen(dimension);
        for (long k = 0; k < count; ++k) {
            for (long c = 0; c < dimension; ++c) {
                out[k * dimension + c] = gen.generate(c, first + k);
            }
        }
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Structure-function cube of every variable of one padded state, through the
// reference's own dispatchComputeStructureCubeCPU (structure_common.hpp:122-160)
// into a (numberOfH x 1 x 1) volume made as StatisticsHelper::findOrCreateSnapshot
// makes it (StatisticsHelper.cpp:127-160): out[var*numberOfH + h].
int alsref_structure_cube(int dim, const int* n, int ghosts, const char* bc, int numberOfH,
    double p, const double* planes, double* out) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", bc, 1.4, 0.5);
        auto o = build(s);
        auto in = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        copyIn(*in, planes);
        auto res = in->makeInstance(size_t(numberOfH), 1, 1, "default");
        res->makeZero();
        if (s.bc == "periodic") {
            functional::dispatchComputeStructureCubeCPU<boundary::PERIODIC>(*res, *in, numberOfH, p);
        } else {
            functional::dispatchComputeStructureCubeCPU<boundary::NEUMANN>(*res, *in, numberOfH, p);
        }
        for (size_t var = 0; var < res->getNumberOfVariables(); ++var) {
            std::memcpy(out + var * numberOfH, res->getScalarMemoryArea(var)->getPointer(),
                size_t(numberOfH) * sizeof(double));
        }
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Selects the diffusion operator of the following builds (see g_diffusion).
int alsref_set_diffusion(const char* kind, const char* recon) {
    const std::string k(kind ? kind : ""), r(recon ? recon : "");
    if ((k != "none" && k != "tecnoroe" && k != "tecnorusanov") ||
        (r != "none" && r != "eno2" && r != "eno3" && r != "eno4")) {
        g_last_error = "unknown diffusion " + k + " / " + r;
        return -1;
    }
    g_diffusion = k;
    g_diffusion_recon = r;
    return 0;
}

// DiffusionOperator::applyDiffusion of one operator object, called `calls`
// times: call k adds the diffusion of state k to output k (both nvar padded
// planes of the ghost width the reference picks, flux hll + reconstruction
// none + this diffusion).  The operator keeps its work volumes between
// calls, as in a time loop.  *ghosts receives that width.
int alsref_apply_diffusion(int dim, const int* n, const char* kind, const char* recon,
    double gamma, int calls, const double* states, double* outs, int* ghosts) {
    const std::string k0 = g_diffusion, r0 = g_diffusion_recon;
    try {
        if (alsref_set_diffusion(kind, recon) != 0) {
            return -1;
        }
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", "neumann", gamma, 0.5);
        auto o = build(s);
        g_diffusion = k0;
        g_diffusion_recon = r0;
        *ghosts = int(o.ghosts);
        auto u = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, o.ghosts);
        auto out = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, o.ghosts);
        const size_t size = paddedCells(*u) * u->getNumberOfVariables();
        for (int c = 0; c < calls; ++c) {
            copyIn(*u, states + size_t(c) * size);
            copyIn(*out, outs + size_t(c) * size);
            o.diffusion->applyDiffusion(*out, *u);
            copyOut(*out, outs + size_t(c) * size);
        }
        return 0;
    } catch (std::exception& e) {
        g_diffusion = k0;
        g_diffusion_recon = r0;
        g_last_error = e.what();
        return -1;
    }
}

// The statistics `name` of `platform` from the reference's
// StatisticsFactory ("cpu": the reference's own classes; "b200": the
// adapters registered above, only in the B200 build) over `samples` padded
// states at time `time` on one rank: each sample is written to it
// (Statistics::write -> computeStatistics), then combineStatistics,
// finalizeStatistics and writeStatistics run in the order of
// Runner.cpp:80-87.  first_out / second_out receive the first two
// statistics it names (mean and variance for meanvar), nvar padded planes
// each.
int alsref_statistics(const char* platform, const char* name, int dim, const int* n,
    int ghosts, long samples, const double* states, double time, double* first_out,
    double* second_out) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", "periodic", 1.4, 0.5);
        auto o = build(s);
        auto u = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        boost::property_tree::ptree tree;
        alsuq::stats::StatisticsParameters params(tree);
        params.setNumberOfSamples(size_t(samples));
        params.setMpiConfiguration(std::make_shared<alsutils::mpi::Configuration>(MPI_COMM_WORLD,
                "cpu"));
        params.setPlatform("cpu");
        alsuq::stats::StatisticsFactory factory;
        auto stats = factory.makeStatistics(platform, name, params);
        auto names = stats->getStatisticsNames();
        std::vector<std::shared_ptr<CaptureWriter>> captures;
        double* outs[2] = {first_out, second_out};
        for (size_t k = 0; k < names.size() && k < 2; ++k) {
            captures.push_back(std::make_shared<CaptureWriter>(outs[k]));
            std::shared_ptr<io::Writer> w = captures.back();
            stats->addWriter(names[k], w);
        }
        const size_t stride = paddedCells(*u) * u->getNumberOfVariables();
        const simulator::TimestepInformation info(time, 0);
        for (long k = 0; k < samples; ++k) {
            copyIn(*u, states + size_t(k) * stride);
            stats->write(*u, *o.grid, info);
        }
        stats->combineStatistics();
        stats->finalizeStatistics();
        stats->writeStatistics(*o.grid);
        for (auto& c : captures) {
            if (c->writes != 1) {
                THROW("statistic written " << c->writes << " times");
            }
        }
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// Number of doubles per variable of the functional `name`'s output for a
// grid of n cells with `ghosts` ghost cells (functional size and ghost
// widths as TimeIntegrationFunctional.cpp:64-72 allocates them).
// The parameters every functional of the factory reads (Moment and
// BoundedVariation "degree", LogEntropy "gamma", Legendre "minValue",
// "maxValue", "degree_k", "degree_n", "degree_m", LegendrePointWise
// "minValue", "maxValue", "degree").
functional::Functional::Parameters functionalParameters(int degree, double gamma,
    const int* legendre_degrees, double min_value, double max_value) {
    functional::Functional::Parameters p(std::map<std::string, std::string>{});
    p.addIntegerParameter("degree", degree);
    p.addDoubleParameter("gamma", gamma);
    p.addIntegerParameter("degree_k", legendre_degrees ? legendre_degrees[0] : 0);
    p.addIntegerParameter("degree_n", legendre_degrees ? legendre_degrees[1] : 0);
    p.addIntegerParameter("degree_m", legendre_degrees ? legendre_degrees[2] : 0);
    p.addDoubleParameter("minValue", min_value);
    p.addDoubleParameter("maxValue", max_value);
    return p;
}

long alsref_functional_size(int dim, const int* n, int ghosts, const char* name, int degree,
    double gamma) {
    try {
        double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        auto s = makeSetup(dim, n, lo, hi, "hll", "none", "forwardeuler", "periodic", gamma, 0.5);
        auto o = build(s);
        auto u = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        auto p = functionalParameters(degree, gamma, nullptr, 0.0, 1.0);
        auto f = functional::FunctionalFactory().makeFunctional("cpu", name, p);
        const ivec3 size = f->getFunctionalSize(*o.grid);
        const ivec3 g = f->getGhostCellSizes(*o.grid, *u);
        auto out = o.volumeFactory->createConservedVolume(size.x, size.y, size.z, g.x);
        return long(paddedCells(*out));
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// The functional `name` of the reference's FunctionalFactory ("cpu"), with
// parameters degree, gamma, the Legendre degrees (k, n, m) and the value
// range [min_value, max_value], on the grid [lower, upper] of n cells:
// out += weight * f(state) for one padded state.  `out` holds the output
// volume's nvar planes (alsref_functional_size doubles each).
int alsref_functional(int dim, const int* n, const double* lower, const double* upper,
    int ghosts, const char* name, int degree, double gamma, const int* legendre_degrees,
    double min_value, double max_value, double weight, const double* planes, double* out) {
    try {
        auto s = makeSetup(dim, n, lower, upper, "hll", "none", "forwardeuler", "periodic",
            gamma, 0.5);
        auto o = build(s);
        auto u = o.volumeFactory->createConservedVolume(s.n.x, s.n.y, s.n.z, ghosts);
        copyIn(*u, planes);
        auto p = functionalParameters(degree, gamma, legendre_degrees, min_value, max_value);
        auto f = functional::FunctionalFactory().makeFunctional("cpu", name, p);
        const ivec3 size = f->getFunctionalSize(*o.grid);
        const ivec3 g = f->getGhostCellSizes(*o.grid, *u);
        auto res = o.volumeFactory->createConservedVolume(size.x, size.y, size.z, g.x);
        copyIn(*res, out);
        (*f)(*res, *u, weight, *o.grid);
        copyOut(*res, out);
        return 0;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

#ifdef ALSREF_WITH_B200
// Selects the classes of the following builds: "cpu" (the reference's),
// "b200" (NumericalFluxB200), "b200-parts" (the reference's NumericalFluxCPU
// over ReconstructionB200, with BoundaryB200 and IntegratorB200) or
// "b200-all" (NumericalFluxB200, BoundaryB200, IntegratorB200).
int alsref_set_flux_platform(const char* platform) {
    const std::string p(platform ? platform : "");
    if (p != "cpu" && p != "b200" && p != "b200-parts" && p != "b200-all") {
        g_last_error = "unknown flux platform " + p;
        return -1;
    }
    g_flux_platform = p;
    return 0;
}
#endif

} // extern "C"
