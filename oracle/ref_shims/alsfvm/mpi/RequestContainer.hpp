// Plumbing shim: without MPI there are never outstanding requests.
#pragma once
#include <memory>
#include <vector>
namespace alsfvm {
namespace mpi {
class RequestContainer {
public:
    void waitForAll() {}
};
} // namespace mpi
} // namespace alsfvm
