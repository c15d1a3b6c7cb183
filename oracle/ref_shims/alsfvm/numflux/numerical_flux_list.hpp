// Plumbing shim: the reference's flux type list reduced to HLL, HLL3,
// Central, Tecno1, TecnoCombined4 and TecnoCombined6 for Euler 1/2/3 (the
// fluxes the oracle builds).
#pragma once
#include "alsfvm/equation/equation_list.hpp"
#include "alsfvm/numflux/euler/HLL.hpp"
#include "alsfvm/numflux/euler/HLL3.hpp"
#include "alsfvm/numflux/Central.hpp"
#include "alsfvm/numflux/TecnoCombined4.hpp"
#include "alsfvm/numflux/TecnoCombined6.hpp"
#include "alsfvm/numflux/euler/Tecno1.hpp"

// the combined fluxes by name, so that no macro argument holds a comma
namespace alsref_shim {
template<int d>
using TecnoCombined4Euler = ::alsfvm::numflux::TecnoCombined4< ::alsfvm::equation::euler::Euler<d>,
    ::alsfvm::numflux::euler::Tecno1<d> >;
template<int d>
using TecnoCombined6Euler = ::alsfvm::numflux::TecnoCombined6< ::alsfvm::equation::euler::Euler<d>,
    ::alsfvm::numflux::euler::Tecno1<d> >;
}

#define ALSFVM_FLUX_INSTANTIATE_ONE(X, F, E) \
    template class X< F, E, 1>; template class X< F, E, 2>; template class X< F, E, 3>;
#define ALSFVM_FLUX_INSTANTIATE(X) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL<1>, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL<2>, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL<3>, ::alsfvm::equation::euler::Euler<3>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL3<1>, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL3<2>, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::HLL3<3>, ::alsfvm::equation::euler::Euler<3>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::Central< ::alsfvm::equation::euler::Euler<1> >, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::Central< ::alsfvm::equation::euler::Euler<2> >, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::Central< ::alsfvm::equation::euler::Euler<3> >, ::alsfvm::equation::euler::Euler<3>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::Tecno1<1>, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::Tecno1<2>, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsfvm::numflux::euler::Tecno1<3>, ::alsfvm::equation::euler::Euler<3>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined4Euler<1>, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined4Euler<2>, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined4Euler<3>, ::alsfvm::equation::euler::Euler<3>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined6Euler<1>, ::alsfvm::equation::euler::Euler<1>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined6Euler<2>, ::alsfvm::equation::euler::Euler<2>) \
    ALSFVM_FLUX_INSTANTIATE_ONE(X, ::alsref_shim::TecnoCombined6Euler<3>, ::alsfvm::equation::euler::Euler<3>)
