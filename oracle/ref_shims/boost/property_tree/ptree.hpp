// Plumbing shim: the oracle never parses XML, so ptree is an empty type.
#pragma once
namespace boost { namespace property_tree { struct ptree {}; } }
