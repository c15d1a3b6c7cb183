// Plumbing shim for building the reference CPU path as a test oracle.
// Replaces the CMake-generated alsutils/config.hpp: no CUDA, no MPI, no timers.
#pragma once
#include <vector>
#include <iostream>
#include <sstream>
#include <fstream>
#define ALSVINN_HAS_CONFIG 1
