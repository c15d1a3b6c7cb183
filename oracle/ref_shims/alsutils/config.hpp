// Plumbing shim for building the reference CPU path as a test oracle.
// Replaces the CMake-generated alsutils/config.hpp: no CUDA, no timers.
// ALSVINN_USE_MPI is set as in the reference's default build
// (CMakeLists.txt:60), so alsutils::mpi::Configuration is the real class;
// the MPI it calls is the single-rank stand-in in ref_shims/mpi.h.
#pragma once
#include <vector>
#include <iostream>
#include <sstream>
#include <fstream>
#define ALSVINN_HAS_CONFIG 1
#define ALSVINN_USE_MPI 1
