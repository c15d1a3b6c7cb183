// Plumbing shim: token pasting for the registration macros
// (REGISTER_STATISTICS, REGISTER_FUNCTIONAL).
#pragma once
#define BOOST_PP_CAT(a, b) BOOST_PP_CAT_I(a, b)
#define BOOST_PP_CAT_I(a, b) a##b
