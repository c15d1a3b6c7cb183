// Plumbing shim: alsfvm/src/functional/Moment.cpp includes this header but
// calls nothing from it.  (Legendre.cpp, which does, is not built.)
#pragma once
