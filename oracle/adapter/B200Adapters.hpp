// boundary::Boundary, reconstruction::Reconstruction, integrator::Integrator
// and diffusion::DiffusionOperator backed by the B200 library: the other
// adapter classes a maintainer adds to alsfvm's factories beside
// numflux::NumericalFluxB200, compiled against the reference's headers:
//   alsfvm/include/alsfvm/boundary/Boundary.hpp:25-35
//   alsfvm/include/alsfvm/reconstruction/Reconstruction.hpp:40-58
//   alsfvm/include/alsfvm/integrator/Integrator.hpp:52-100
//   alsfvm/include/alsfvm/diffusion/DiffusionOperator.hpp:25-47
//
// TEST INFRASTRUCTURE in this repository (built only into
// oracle/_ref/libalsref_b200.so): the reference's time loop drives them and
// tests/test_gpu_dropin.py compares whole simulations with the reference's
// own classes.  Host volumes are staged through device buffers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "alsfvm/boundary/Boundary.hpp"
#include "alsfvm/diffusion/DiffusionOperator.hpp"
#include "alsfvm/grid/Grid.hpp"
#include "alsfvm/integrator/Integrator.hpp"
#include "alsfvm/integrator/System.hpp"
#include "alsfvm/reconstruction/Reconstruction.hpp"
#include "alsutils/error/Exception.hpp"
#include "als_b200.h"

namespace alsfvm {
namespace b200 {

inline void check_cuda(cudaError_t e) {
    if (e != cudaSuccess) {
        THROW("CUDA: " << cudaGetErrorString(e));
    }
}

inline void check_als(int rc, const char* what) {
    if (rc != ALS_OK) {
        THROW(what << ": " << als_last_error());
    }
}

inline size_t padded_cells(const volume::Volume& v) {
    return v.getTotalNumberOfXCells() * v.getTotalNumberOfYCells() * v.getTotalNumberOfZCells();
}

// Device copies of the planes of a few volumes (one slot per volume).
class Staging {
public:
    ~Staging() {
        for (double* p : planes) {
            cudaFree(p);
        }
    }

    // device plane pointers of `slot` for `v`, copying the host data in when `load`
    std::vector<double*> put(int slot, const volume::Volume& v, bool load) {
        const size_t nvar = v.getNumberOfVariables();
        const size_t cells = padded_cells(v);
        std::vector<double*> out(nvar);
        const bool host = v.getScalarMemoryArea(0)->isOnHost();
        for (size_t k = 0; k < nvar; ++k) {
            if (!host) {
                out[k] = const_cast<double*>(v.getScalarMemoryArea(k)->getPointer());
                continue;
            }
            out[k] = plane(slot * 8 + int(k), cells);
            if (load) {
                check_cuda(cudaMemcpy(out[k], v.getScalarMemoryArea(k)->getPointer(),
                    cells * sizeof(double), cudaMemcpyHostToDevice));
            }
        }
        return out;
    }

    // copies the device planes of `slot` back into a host volume
    void get(int slot, volume::Volume& v) {
        if (!v.getScalarMemoryArea(0)->isOnHost()) {
            return;
        }
        const size_t cells = padded_cells(v);
        for (size_t k = 0; k < v.getNumberOfVariables(); ++k) {
            check_cuda(cudaMemcpy(v.getScalarMemoryArea(k)->getPointer(), plane(slot * 8 + int(k), cells),
                cells * sizeof(double), cudaMemcpyDeviceToHost));
        }
    }

private:
    double* plane(int index, size_t cells) {
        if (index >= int(planes.size())) {
            planes.resize(size_t(index) + 1, nullptr);
            sizes.resize(size_t(index) + 1, 0);
        }
        if (sizes[size_t(index)] != cells) {
            cudaFree(planes[size_t(index)]);
            check_cuda(cudaMalloc(&planes[size_t(index)], cells * sizeof(double)));
            sizes[size_t(index)] = cells;
        }
        return planes[size_t(index)];
    }

    std::vector<double*> planes;
    std::vector<size_t> sizes;
};

inline als_grid make_grid(const volume::Volume& v, int dimension, int ghosts, real gamma) {
    als_grid g;
    g.dimension = dimension;
    g.n[0] = int(v.getNumberOfXCells());
    g.n[1] = int(v.getNumberOfYCells());
    g.n[2] = int(v.getNumberOfZCells());
    g.ghosts = ghosts;
    g.gamma = gamma;
    return g;
}

class BoundaryB200 : public boundary::Boundary {
public:
    BoundaryB200(int boundaryCode, int ghosts) : code(boundaryCode), ghosts(ghosts) {}

    void applyBoundaryConditions(volume::Volume& volume, const grid::Grid& grid) override {
        std::vector<double*> p = stage.put(0, volume, true);
        const als_grid g = make_grid(volume, grid.getActiveDimension(), ghosts, 1.4);
        check_als(als_fill_ghosts(&g, code, p.data(), int(p.size()), nullptr), "als_fill_ghosts");
        stage.get(0, volume);
    }

private:
    int code;
    int ghosts;
    Staging stage;
};

class ReconstructionB200 : public reconstruction::Reconstruction {
public:
    ReconstructionB200(int dimension, int reconstructionCode, real gamma)
        : dimension(dimension), code(reconstructionCode), gamma(gamma) {}

    // The library reconstructs the reference's whole range; a region
    // [start, end) of the caller is contained in it with identical values.
    void performReconstruction(const volume::Volume& in, size_t direction, size_t indicatorVariable,
        volume::Volume& leftOut, volume::Volume& rightOut, const ivec3& start,
        const ivec3& end) override {
        (void)indicatorVariable;   // rho, as in the reference's Euler reconstructions
        (void)start;
        (void)end;
        std::vector<double*> pin = stage.put(0, in, true);
        std::vector<double*> pl = stage.put(1, leftOut, true);
        std::vector<double*> pr = stage.put(2, rightOut, true);
        const als_grid g = make_grid(in, dimension, int(getNumberOfGhostCells()), gamma);
        std::vector<const double*> cin(pin.begin(), pin.end());
        check_als(als_reconstruct(&g, code, int(direction), cin.data(), pl.data(), pr.data(),
            nullptr), "als_reconstruct");
        stage.get(1, leftOut);
        stage.get(2, rightOut);
    }

    size_t getNumberOfGhostCells() override {
        return size_t(als_ghost_cells(ALS_FLUX_HLL, code));
    }

private:
    int dimension;
    int code;
    real gamma;
    Staging stage;
};

// The system evaluates L(U) (ConservedSystem with any flux); the stage
// combination and its scaling run in the library (als_integrator_combine),
// dt is the Integrator's own computeTimestep (with every adjuster added).
class IntegratorB200 : public integrator::Integrator {
public:
    IntegratorB200(int integratorCode, alsfvm::shared_ptr<integrator::System> system)
        : code(integratorCode), system(system) {}

    size_t getNumberOfSubsteps() const override {
        return size_t(code + 1);
    }

    real performSubstep(std::vector<alsfvm::shared_ptr<volume::Volume>>& inputConserved,
        rvec3 spatialCellSizes, real dt, real cfl, volume::Volume& output, size_t substep,
        const simulator::TimestepInformation& timestepInformation) override {
        rvec3 waveSpeeds(0, 0, 0);
        (*system)(*inputConserved[substep], waveSpeeds, true, output);
        if (substep == 0) {
            dt = computeTimestep(waveSpeeds, spatialCellSizes, cfl, timestepInformation);
        }
        std::vector<double*> o = stage.put(0, output, true);
        std::vector<double*> us = stage.put(1, *inputConserved[substep], true);
        std::vector<double*> u0 = stage.put(2, *inputConserved[0], true);
        const size_t cells = padded_cells(output);
        if (code == ALS_INT_RK4 && substep == 3) {
            // out = (c/6) L + U1/3 + 2 U2/3 + U3/3 - U0/3 (RungeKutta4.cpp:80-87)
            std::vector<double*> u1 = stage.put(3, *inputConserved[1], true);
            std::vector<double*> u2 = stage.put(4, *inputConserved[2], true);
            for (size_t k = 0; k < o.size(); ++k) {
                check_als(als_integrator_combine_rk4(o[k], u0[k], u1[k], u2[k], us[k], cells,
                    dt / spatialCellSizes.x, nullptr), "als_integrator_combine_rk4");
            }
        } else {
            for (size_t k = 0; k < o.size(); ++k) {
                check_als(als_integrator_combine(code, int(substep), o[k], us[k], u0[k], cells,
                    dt / spatialCellSizes.x, nullptr), "als_integrator_combine");
            }
        }
        check_cuda(cudaDeviceSynchronize());
        stage.get(0, output);
        return dt;
    }

private:
    int code;
    alsfvm::shared_ptr<integrator::System> system;
    Staging stage;
};

// diffusion::DiffusionOperator (DiffusionOperator.hpp:25-47) backed by an
// als_diffusion operator, created on the first call for the volume's shape.
class DiffusionB200 : public diffusion::DiffusionOperator {
public:
    DiffusionB200(int dimension, int kind, int reconstruction, real gamma)
        : dimension(dimension), kind(kind), reconstruction(reconstruction), gamma(gamma) {}

    ~DiffusionB200() override {
        als_diffusion_destroy(op);
    }

    void applyDiffusion(volume::Volume& outputVolume, const volume::Volume& conservedVolume) override {
        if (!op) {
            als_grid g;
            g.dimension = dimension;
            g.n[0] = int(conservedVolume.getNumberOfXCells());
            g.n[1] = int(conservedVolume.getNumberOfYCells());
            g.n[2] = int(conservedVolume.getNumberOfZCells());
            g.ghosts = int(conservedVolume.getNumberOfXGhostCells());
            g.gamma = gamma;
            check_als(als_diffusion_create(&g, kind, reconstruction, &op), "als_diffusion_create");
        }
        std::vector<double*> u = stage.put(0, conservedVolume, true);
        std::vector<double*> o = stage.put(1, outputVolume, true);
        std::vector<const double*> cu(u.begin(), u.end());
        check_als(als_diffusion_apply(op, cu.data(), o.data(), nullptr), "als_diffusion_apply");
        check_cuda(cudaDeviceSynchronize());
        stage.get(1, outputVolume);
    }

    size_t getNumberOfGhostCells() const override {
        return size_t(als_diffusion_ghost_cells(reconstruction));
    }

private:
    int dimension;
    int kind;
    int reconstruction;
    real gamma;
    als_diffusion* op = nullptr;
    Staging stage;
};

} // namespace b200
} // namespace alsfvm
