// Parameter draws of the UQ sample loop, host side.
//
// alsuq's default generator is one process-wide, default-seeded
// std::mt19937_64 read through std::uniform_real_distribution<double>(0, 1);
// component c of sample s is draw number s*dimension + c
// (alsuq/src/generator/STLMersenne.cpp:38-85, STLMersenne.hpp:37), scaled
// to [lower, upper] as x*(upper-lower)+lower (alsuq/src/distribution/Uniform.cpp:32-34).
// Using the same standard-library engine and distribution gives the same
// numbers for the same sample indices.
#include <random>

#include "als_b200.h"

extern "C" int als_uniform_draws(long long dimension, long long first_sample, long long count,
    double lower, double upper, double* out) {
    if (dimension < 1 || first_sample < 0 || count < 0 || (count > 0 && !out)) {
        return ALS_E_INVALID;
    }
    std::mt19937_64 engine;
    std::uniform_real_distribution<double> uniform(0.0, 1.0);
    engine.discard((unsigned long long)(first_sample * dimension));
    for (long long k = 0; k < count * dimension; ++k) {
        out[k] = uniform(engine) * (upper - lower) + lower;
    }
    return ALS_OK;
}
