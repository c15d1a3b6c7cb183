// Plumbing shim: replaces the Boost-based stack trace used in THROW messages.
#include <string>
namespace alsutils { namespace debug {
std::string getLongStacktrace() { return std::string("(stack trace not available in the oracle build)"); }
} }
