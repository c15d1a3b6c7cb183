// Plumbing shim: logging is compiled out (the reference uses Boost.Log).
#pragma once
#include <sstream>
#define ALSVINN_LOG(severity, message) { }
