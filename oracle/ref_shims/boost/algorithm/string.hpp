// Plumbing shim: the string helpers alsutils/src/parameters/Parameters.cpp
// calls (split on any of a set of characters, join with a separator).
#pragma once
#include <string>
#include <vector>
namespace boost {
namespace algorithm {
struct any_of_chars {
    std::string chars;
    bool operator()(char c) const { return chars.find(c) != std::string::npos; }
};
inline any_of_chars is_any_of(const std::string& chars) {
    return any_of_chars{chars};
}
inline std::vector<std::string>& split(std::vector<std::string>& out, const std::string& in,
    const any_of_chars& sep) {
    out.clear();
    std::string cur;
    for (char c : in) {
        if (sep(c)) {
            out.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    out.push_back(cur);
    return out;
}
inline std::string join(const std::vector<std::string>& parts, const std::string& sep) {
    std::string out;
    for (size_t i = 0; i < parts.size(); ++i) {
        out += (i ? sep : std::string()) + parts[i];
    }
    return out;
}
} // namespace algorithm
using algorithm::is_any_of;
using algorithm::join;
using algorithm::split;
} // namespace boost
