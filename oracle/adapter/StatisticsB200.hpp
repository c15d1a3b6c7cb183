// alsuq::stats::Statistics "meanvar" backed by the B200 library's FP64
// Welford accumulator (als_stats_*): the statistics class a maintainer
// registers beside the reference's MeanVariance
// (alsuq/include/alsuq/stats/MeanVariance.hpp:23-35,
//  alsuq/src/stats/MeanVariance.cpp:30-67) with
//   REGISTER_STATISTICS(b200, meanvar, alsuq::stats::MeanVarianceB200)
// (alsuq/include/alsuq/stats/stats_util.hpp:18-25), compiled here against
// the reference's own headers.
//
// TEST INFRASTRUCTURE in this repository: it is built only into
// oracle/_ref/libalsref_b200.so, where the reference's StatisticsFactory
// creates it by name and tests/test_gpu_dropin.py feeds it and the
// reference's own MeanVariance the same samples.
//
// Against the reference, step by step:
//  * computeStatistics adds the sample (every variable, the whole padded
//    volume, as Volume::operator+= and addPower do) to the accumulator of
//    its snapshot time; the snapshot volumes "mean" and "variance" come from
//    StatisticsHelper::findOrCreateSnapshot as in MeanVariance.cpp:33-43.
//    Host volumes are staged through one device buffer.
//  * combineStatistics gathers every rank's (n, mean, M2) and merges them in
//    rank order (Chan), so every rank holds the same bits; the reference
//    sum-reduces S1 and S2 to rank 0 and divides by the configured sample
//    count (StatisticsHelper.cpp:35-79).
//  * finalizeStatistics writes the mean and the biased variance M2/n into
//    the snapshot volumes; the reference forms S2/M - (S1/M)^2
//    (MeanVariance.cpp:55-67).  The quantities are the same; the Welford
//    form avoids the cancellation of the raw-moment difference, so the
//    variance agrees to rounding, not bit for bit.
//  * writeStatistics is StatisticsHelper's (writers added by name).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <vector>

#include "alsuq/stats/StatisticsHelper.hpp"
#include "alsuq/mpi/utils.hpp"
#include "alsutils/error/Exception.hpp"
#include "als_b200.h"

namespace alsuq {
namespace stats {

class MeanVarianceB200 : public StatisticsHelper {
public:
    explicit MeanVarianceB200(const StatisticsParameters& parameters)
        : StatisticsHelper(parameters), mpiConfig(parameters.getMpiConfiguration()) {}

    ~MeanVarianceB200() override {
        for (auto& a : accumulators) {
            als_stats_destroy(a.second.stats);
        }
        cudaFree(staging);
    }

    std::vector<std::string> getStatisticsNames() const override {
        return {"mean", "variance"};
    }

    void computeStatistics(const alsfvm::volume::Volume& conservedVariables,
        const alsfvm::grid::Grid&,
        const alsfvm::simulator::TimestepInformation& timestepInformation) override {
        findOrCreateSnapshot("mean", timestepInformation, conservedVariables);
        findOrCreateSnapshot("variance", timestepInformation, conservedVariables);
        const size_t nvar = conservedVariables.getNumberOfVariables();
        const size_t cells = conservedVariables.getTotalNumberOfXCells() *
            conservedVariables.getTotalNumberOfYCells() *
            conservedVariables.getTotalNumberOfZCells();
        Accumulator& acc = accumulator(timestepInformation.getCurrentTime(), nvar * cells);
        double* dev = stage(nvar * cells);
        for (size_t v = 0; v < nvar; ++v) {
            auto area = conservedVariables.getScalarMemoryArea(v);
            check_cuda(cudaMemcpy(dev + v * cells, area->getPointer(), cells * sizeof(double),
                area->isOnHost() ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice));
        }
        check(als_stats_add(acc.stats, dev, ALS_FP64, 1, (long long)(nvar * cells), nullptr),
            "als_stats_add");
        check_cuda(cudaDeviceSynchronize());
    }

    void combineStatistics() override {
        const int ranks = mpiConfig ? mpiConfig->getNumberOfProcesses() : 1;
        if (ranks == 1) {
            return;
        }
        for (auto& a : accumulators) {
            Accumulator& acc = a.second;
            long long n = 0;
            double *mean = nullptr, *m2 = nullptr;
            check(als_stats_moments(acc.stats, &n, &mean, &m2), "als_stats_moments");
            const size_t count = acc.count;
            std::vector<double> local(2 * count), all(2 * count * size_t(ranks));
            std::vector<long long> counts(static_cast<size_t>(ranks));
            check_cuda(cudaMemcpy(local.data(), mean, count * sizeof(double), cudaMemcpyDeviceToHost));
            check_cuda(cudaMemcpy(local.data() + count, m2, count * sizeof(double),
                cudaMemcpyDeviceToHost));
            MPI_SAFE_CALL(MPI_Allgather(&n, 1, MPI_LONG_LONG, counts.data(), 1, MPI_LONG_LONG,
                    mpiConfig->getCommunicator()));
            MPI_SAFE_CALL(MPI_Allgather(local.data(), int(2 * count), MPI_DOUBLE, all.data(),
                    int(2 * count), MPI_DOUBLE, mpiConfig->getCommunicator()));
            // a fresh accumulator takes rank 0's moments exactly, then the others in order
            als_stats* merged = nullptr;
            check(als_stats_create((long long)count, device(), &merged), "als_stats_create");
            double* dev = stage(2 * count);
            for (int r = 0; r < ranks; ++r) {
                check_cuda(cudaMemcpy(dev, all.data() + size_t(r) * 2 * count,
                    2 * count * sizeof(double), cudaMemcpyHostToDevice));
                check(als_stats_merge(merged, counts[size_t(r)], dev, dev + count, nullptr),
                    "als_stats_merge");
                check_cuda(cudaDeviceSynchronize());
            }
            als_stats_destroy(acc.stats);
            acc.stats = merged;
        }
    }

    void finalizeStatistics() override {
        for (auto& snapshot : this->snapshots) {
            auto found = accumulators.find(snapshot.first);
            if (found == accumulators.end()) {
                continue;
            }
            Accumulator& acc = found->second;
            double* dev = stage(2 * acc.count);
            check(als_stats_result(acc.stats, dev, dev + acc.count, nullptr), "als_stats_result");
            check_cuda(cudaDeviceSynchronize());
            unstage(dev, *snapshot.second["mean"].getVolumes().getConservedVolume());
            unstage(dev + acc.count,
                *snapshot.second["variance"].getVolumes().getConservedVolume());
        }
    }

private:
    struct Accumulator {
        als_stats* stats = nullptr;
        size_t count = 0;
    };

    static void check_cuda(cudaError_t e) {
        if (e != cudaSuccess) {
            THROW("CUDA: " << cudaGetErrorString(e));
        }
    }

    static void check(int rc, const char* what) {
        if (rc != ALS_OK) {
            THROW(what << ": " << als_last_error());
        }
    }

    static int device() {
        int d = 0;
        check_cuda(cudaGetDevice(&d));
        return d;
    }

    Accumulator& accumulator(real time, size_t count) {
        Accumulator& acc = accumulators[time];
        if (!acc.stats) {
            check(als_stats_create((long long)count, device(), &acc.stats), "als_stats_create");
            acc.count = count;
        } else if (acc.count != count) {
            THROW("sample size " << count << " differs from the snapshot's " << acc.count);
        }
        return acc;
    }

    double* stage(size_t count) {
        if (count > staged) {
            cudaFree(staging);
            staging = nullptr;
            check_cuda(cudaMalloc(&staging, count * sizeof(double)));
            staged = count;
        }
        return staging;
    }

    // copies count = nvar * padded cells doubles into the volume's planes
    static void unstage(const double* dev, alsfvm::volume::Volume& volume) {
        const size_t cells = volume.getTotalNumberOfXCells() * volume.getTotalNumberOfYCells() *
            volume.getTotalNumberOfZCells();
        for (size_t v = 0; v < volume.getNumberOfVariables(); ++v) {
            auto area = volume.getScalarMemoryArea(v);
            check_cuda(cudaMemcpy(area->getPointer(), dev + v * cells, cells * sizeof(double),
                area->isOnHost() ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
        }
    }

    mpi::ConfigurationPtr mpiConfig;
    std::map<real, Accumulator> accumulators;
    double* staging = nullptr;
    size_t staged = 0;
};

} // namespace stats
} // namespace alsuq
