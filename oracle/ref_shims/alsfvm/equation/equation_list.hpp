// Plumbing shim: the reference's boost::fusion type list reduced to the three
// Euler equations that the oracle builds.  No arithmetic lives here.
#pragma once
#include "alsfvm/equation/euler/Euler.hpp"
#include "alsfvm/equation/EquationInformation.hpp"

namespace alsfvm {
namespace equation {
template<class Function>
void for_each_equation(const Function& f) {
    f(EquationInformation<euler::Euler<1>>());
    f(EquationInformation<euler::Euler<2>>());
    f(EquationInformation<euler::Euler<3>>());
}
}
}

#define ALSFVM_EQUATION_INSTANTIATE(X) \
    template class X< ::alsfvm::equation::euler::Euler<1> >; \
    template class X< ::alsfvm::equation::euler::Euler<2> >; \
    template class X< ::alsfvm::equation::euler::Euler<3> >;
