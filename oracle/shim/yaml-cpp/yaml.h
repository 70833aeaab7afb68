// Minimal stand-in for the part of yaml-cpp that the CTBB_ICD reference uses
// (parse_config.cpp:27-111): YAML::LoadFile, Node::operator[](const char*),
// Node::as<T>() for std::string / double / size_t, and
// YAML::RepresentationException thrown when a key is absent, empty or not
// convertible (the reference then prints "NOT FOUND").
//
// Test infrastructure only (oracle build). The parameter files are flat
// `key: value  # comment` mappings, which is all this reader understands.
#pragma once

#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>

namespace YAML {

class Exception : public std::runtime_error {
public:
    explicit Exception(const std::string& m) : std::runtime_error(m) {}
};
class RepresentationException : public Exception {
public:
    explicit RepresentationException(const std::string& m) : Exception(m) {}
};
class BadFile : public Exception {
public:
    explicit BadFile(const std::string& m) : Exception("bad file: " + m) {}
};

namespace detail {
inline std::string trim(const std::string& s) {
    const char* ws = " \t\r\n";
    const std::size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return "";
    const std::size_t e = s.find_last_not_of(ws);
    return s.substr(b, e - b + 1);
}
}  // namespace detail

class Node {
public:
    Node() : defined_(false) {}
    explicit Node(const std::string& scalar) : defined_(true), scalar_(scalar) {}

    Node operator[](const char* key) const {
        std::map<std::string, std::string>::const_iterator it = map_.find(key);
        if (it == map_.end()) return Node();
        return Node(it->second);
    }
    Node operator[](const std::string& key) const { return (*this)[key.c_str()]; }

    template <class T>
    T as() const;

    std::map<std::string, std::string> map_;

private:
    void require() const {
        if (!defined_ || scalar_.empty()) throw RepresentationException("invalid node");
    }
    bool defined_;
    std::string scalar_;
};

template <>
inline std::string Node::as<std::string>() const {
    require();
    return scalar_;
}

template <>
inline double Node::as<double>() const {
    require();
    char* end = 0;
    errno = 0;
    const double v = std::strtod(scalar_.c_str(), &end);
    if (end == scalar_.c_str() || *end != '\0' || errno == ERANGE)
        throw RepresentationException("bad conversion");
    return v;
}

template <>
inline unsigned long Node::as<unsigned long>() const {
    require();
    if (scalar_[0] == '-') throw RepresentationException("bad conversion");
    char* end = 0;
    errno = 0;
    const unsigned long long v = std::strtoull(scalar_.c_str(), &end, 10);
    if (end == scalar_.c_str() || *end != '\0' || errno == ERANGE)
        throw RepresentationException("bad conversion");
    return static_cast<unsigned long>(v);
}

inline Node LoadFile(const std::string& path) {
    std::ifstream f(path.c_str());
    if (!f.good()) throw BadFile(path);
    Node root;
    std::string line;
    while (std::getline(f, line)) {
        // Strip a comment: '#' at line start or preceded by whitespace.
        for (std::size_t i = 0; i < line.size(); ++i) {
            if (line[i] == '#' && (i == 0 || line[i - 1] == ' ' || line[i - 1] == '\t')) {
                line.erase(i);
                break;
            }
        }
        const std::size_t colon = line.find(':');
        if (colon == std::string::npos) continue;
        const std::string key = detail::trim(line.substr(0, colon));
        const std::string val = detail::trim(line.substr(colon + 1));
        if (key.empty()) continue;
        root.map_[key] = val;
    }
    return root;
}

}  // namespace YAML
