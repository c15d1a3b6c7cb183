// numflux::NumericalFlux backed by the B200 library: the class a maintainer
// adds to alsfvm's flux factory to select this path as a platform, compiled
// here against the reference's own headers
// (alsfvm/include/alsfvm/numflux/NumericalFlux.hpp:25-52).
//
// TEST INFRASTRUCTURE in this repository: it is built only into
// oracle/_ref/libalsref_b200.so, where the reference's unmodified time
// integrators and ConservedSystem drive it, so that a whole simulation with
// this flux can be compared bit for bit with the reference's CPU flux.
//
// Volumes on the host (the reference's "cpu" memory) are staged through
// device buffers; the region [start, end) and the output outside it behave
// as in NumericalFluxCPU::computeFlux (NumericalFluxCPU.cpp:171-221): the
// output is zeroed and filled inside the region only, and waveSpeed gets the
// region's maximal face speed per active direction.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "alsfvm/numflux/NumericalFlux.hpp"
#include "alsfvm/grid/Grid.hpp"
#include "alsutils/error/Exception.hpp"
#include "als_b200.h"

namespace alsfvm {
namespace numflux {

class NumericalFluxB200 : public NumericalFlux {
public:
    NumericalFluxB200(const grid::Grid& grid, int flux, int reconstruction, real gamma)
        : dimension(grid.getActiveDimension()), n(grid.getDimensions()), flux(flux),
          reconstruction(reconstruction), gamma(gamma) {
    }

    ~NumericalFluxB200() override {
        for (double* p : device) {
            cudaFree(p);
        }
    }

    void computeFlux(const volume::Volume& U, rvec3& waveSpeed, bool computeWaveSpeed,
        volume::Volume& out, const ivec3& start, const ivec3& end) override {
        const size_t nvar = U.getNumberOfVariables();
        const size_t plane = U.getTotalNumberOfXCells() * U.getTotalNumberOfYCells() *
            U.getTotalNumberOfZCells();
        const bool host = U.getScalarMemoryArea(0)->isOnHost();
        std::vector<const double*> in(nvar);
        std::vector<double*> o(nvar);
        if (host) {
            stage(nvar, plane);
            for (size_t v = 0; v < nvar; ++v) {
                check(cudaMemcpy(device[v], U.getScalarMemoryArea(v)->getPointer(),
                    plane * sizeof(double), cudaMemcpyHostToDevice));
                check(cudaMemcpy(device[nvar + v], out.getScalarMemoryArea(v)->getPointer(),
                    plane * sizeof(double), cudaMemcpyHostToDevice));
                in[v] = device[v];
                o[v] = device[nvar + v];
            }
        } else {
            for (size_t v = 0; v < nvar; ++v) {
                in[v] = U.getScalarMemoryArea(v)->getPointer();
                o[v] = out.getScalarMemoryArea(v)->getPointer();
            }
        }
        als_grid g;
        g.dimension = dimension;
        g.n[0] = n.x;
        g.n[1] = n.y;
        g.n[2] = n.z;
        // the volume's ghost width: at least the flux's, wider when a
        // diffusion operator needs more (ConservedSystem.cpp:109-114)
        g.ghosts = int(U.getNumberOfXGhostCells());
        g.gamma = gamma;
        const int s[3] = {start.x, start.y, start.z};
        const int e[3] = {end.x, end.y, end.z};
        double ws[3] = {0, 0, 0};
        // computeWaveSpeed == false: no wave speeds, so no synchronisation
        const int rc = als_compute_flux(&g, flux, reconstruction, in.data(), o.data(), s, e,
            computeWaveSpeed ? ws : nullptr, nullptr);
        if (rc != ALS_OK) {
            THROW("als_compute_flux: " << als_last_error());
        }
        if (host) {
            for (size_t v = 0; v < nvar; ++v) {
                check(cudaMemcpy(out.getScalarMemoryArea(v)->getPointer(), device[nvar + v],
                    plane * sizeof(double), cudaMemcpyDeviceToHost));
            }
        }
        if (!computeWaveSpeed) {
            return;
        }
        waveSpeed.x = ws[0];
        if (dimension > 1) {
            waveSpeed.y = ws[1];
        }
        if (dimension > 2) {
            waveSpeed.z = ws[2];
        }
    }

    size_t getNumberOfGhostCells() override {
        return size_t(als_ghost_cells(flux, reconstruction));
    }

private:
    static void check(cudaError_t e) {
        if (e != cudaSuccess) {
            THROW("CUDA: " << cudaGetErrorString(e));
        }
    }

    void stage(size_t nvar, size_t plane) {
        if (device.size() == 2 * nvar && staged == plane) {
            return;
        }
        for (double* p : device) {
            cudaFree(p);
        }
        device.assign(2 * nvar, nullptr);
        for (double*& p : device) {
            check(cudaMalloc(&p, plane * sizeof(double)));
        }
        staged = plane;
    }

    int dimension;
    ivec3 n;
    int flux;
    int reconstruction;
    real gamma;
    std::vector<double*> device;
    size_t staged = 0;
};

} // namespace numflux
} // namespace alsfvm
