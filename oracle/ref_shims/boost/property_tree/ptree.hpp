// Plumbing shim: the oracle never parses XML.  Parameters objects
// (alsutils/src/parameters/Parameters.cpp) keep their values in a property
// tree, so this is a flat ordered list of (key, value) children with the few
// members that file calls: get<T>, put, add, find / not_found and iteration.
// Values are stored as text with enough digits to read doubles back exactly.
#pragma once
#include <iomanip>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
namespace boost {
namespace property_tree {
struct ptree {
    typedef std::pair<std::string, ptree> value_type;
    typedef std::vector<value_type>::iterator iterator;
    typedef std::vector<value_type>::const_iterator const_iterator;

    std::string data;
    std::vector<value_type> children;

    iterator begin() { return children.begin(); }
    iterator end() { return children.end(); }
    const_iterator begin() const { return children.begin(); }
    const_iterator end() const { return children.end(); }

    const_iterator find(const std::string& key) const {
        for (const_iterator it = children.begin(); it != children.end(); ++it) {
            if (it->first == key) {
                return it;
            }
        }
        return children.end();
    }
    const_iterator not_found() const { return children.end(); }

    template<class T> T get(const std::string& key) const {
        const_iterator it = find(key);
        if (it == end()) {
            throw std::runtime_error("No such node (" + key + ")");
        }
        return convert<T>(it->second.data);
    }

    template<class T> ptree& put(const std::string& key, const T& value) {
        for (auto& child : children) {
            if (child.first == key) {
                child.second.data = text(value);
                return child.second;
            }
        }
        return add(key, value);
    }

    template<class T> ptree& add(const std::string& key, const T& value) {
        ptree child;
        child.data = text(value);
        children.push_back(value_type(key, child));
        return children.back().second;
    }

private:
    template<class T> static std::string text(const T& value) {
        std::ostringstream s;
        s << std::setprecision(std::numeric_limits<double>::max_digits10) << value;
        return s.str();
    }
    template<class T> static T convert(const std::string& s) {
        std::istringstream in(s);
        T value;
        in >> value;
        if (in.fail()) {
            throw std::runtime_error("conversion of data to type failed (" + s + ")");
        }
        return value;
    }
};
template<> inline std::string ptree::convert<std::string>(const std::string& s) {
    return s;
}
} // namespace property_tree
} // namespace boost
