// sfh_yaml.hpp -- reader for the subset of YAML that sonicSolver case
// directories use: block mappings by indentation, `key: value`, block
// sequences (`- item`), flow sequences / mappings (`[a, b]`, `{k: v}`),
// quoted and plain scalars, `#` comments, and whole JSON documents (the
// mesh generation file is JSON, which is YAML flow style).  It replaces the
// reference's yaml-cpp / nlohmann_json front end for the files the explicit
// Euler path reads; anything outside the subset is reported with file and
// line, never guessed.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace sfh {

struct Node {
    enum Kind { Null, Scalar, Seq, Map };
    Kind kind = Null;
    std::string text;                                  // Scalar
    std::vector<Node> items;                           // Seq
    std::vector<std::pair<std::string, Node>> fields;  // Map (file order)

    bool is_map() const { return kind == Map; }
    bool is_seq() const { return kind == Seq; }
    bool is_scalar() const { return kind == Scalar; }
    // Child of a mapping, or nullptr.
    const Node* get(const std::string& key) const;
    // Child of a mapping; throws naming the key when absent.
    const Node& at(const std::string& key) const;
    double number() const;     // Scalar parsed as a double (throws otherwise)
    long long integer() const;  // Scalar parsed as an integer
    bool boolean() const;       // true/false/yes/no/on/off
    const std::string& str() const;
};

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Parses a document; `origin` names it in error messages.
Node parse_yaml(const std::string& text, const std::string& origin = "<string>");
Node load_yaml_file(const std::string& path);

}  // namespace sfh
