// sfh_yaml.cpp -- the YAML-subset / JSON reader (see sfh_yaml.hpp).
#include "sfh_yaml.hpp"

#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <regex>
#include <sstream>

namespace sfh {

const Node* Node::get(const std::string& key) const {
    if (kind != Map) return nullptr;
    for (const auto& kv : fields)
        if (kv.first == key) return &kv.second;
    return nullptr;
}

const Node& Node::at(const std::string& key) const {
    const Node* n = get(key);
    if (!n) throw ParseError("missing key '" + key + "'");
    return *n;
}

const std::string& Node::str() const {
    if (kind != Scalar) throw ParseError("expected a scalar value");
    return text;
}

double Node::number() const {
    const std::string& s = str();
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(s.c_str(), &end);
    if (s.empty() || *end != '\0' || errno == ERANGE) throw ParseError("'" + s + "' is not a number");
    return v;
}

long long Node::integer() const {
    const double v = number();
    const long long i = (long long)v;
    if ((double)i != v) throw ParseError("'" + text + "' is not an integer");
    return i;
}

bool Node::boolean() const {
    const std::string& s = str();
    if (s == "true" || s == "True" || s == "yes" || s == "on") return true;
    if (s == "false" || s == "False" || s == "no" || s == "off") return false;
    throw ParseError("'" + s + "' is not a boolean");
}

namespace {

struct Line {
    int indent;
    std::string body;
    int number;
};

bool space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && space(s[a])) ++a;
    while (b > a && space(s[b - 1])) --b;
    return s.substr(a, b - a);
}

// Removes a comment: '#' outside quotes at the start or after whitespace.
std::string strip_comment(const std::string& s) {
    char quote = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (quote) {
            if (c == '\\' && quote == '"' && i + 1 < s.size()) ++i;
            else if (c == quote) quote = 0;
        } else if (c == '"' || c == '\'') {
            quote = c;
        } else if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) {
            return s.substr(0, i);
        }
    }
    return s;
}

Node scalar(std::string s) {
    Node n;
    n.kind = Node::Scalar;
    n.text = std::move(s);
    return n;
}

// Flow-style values: JSON and YAML [..] / {..}.
class Flow {
public:
    Flow(const std::string& s, const std::string& where) : s_(s), where_(where) {}

    Node document() {
        Node v = value();
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    std::string where_;
    size_t i_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        throw ParseError(where_ + ": " + what + " at offset " + std::to_string(i_));
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    Node value() {
        ws();
        if (i_ >= s_.size()) fail("unexpected end");
        const char c = s_[i_];
        if (c == '[') return seq();
        if (c == '{') return map();
        if (c == '"' || c == '\'') return scalar(quoted());
        return plain();
    }
    std::string quoted() {
        const char q = s_[i_++];
        std::string out;
        while (i_ < s_.size()) {
            const char c = s_[i_++];
            if (c == q) {
                if (q == '\'' && i_ < s_.size() && s_[i_] == '\'') {
                    out += '\'';
                    ++i_;
                    continue;
                }
                return out;
            }
            if (q == '"' && c == '\\' && i_ < s_.size()) {
                const char e = s_[i_++];
                out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
            } else {
                out += c;
            }
        }
        fail("unterminated string");
    }
    Node plain() {
        const size_t a = i_;
        while (i_ < s_.size() && s_[i_] != ',' && s_[i_] != ']' && s_[i_] != '}' &&
               !(s_[i_] == ':' && (i_ + 1 >= s_.size() || s_[i_ + 1] == ' ')))
            ++i_;
        const std::string t = trim(s_.substr(a, i_ - a));
        if (t.empty()) fail("empty value");
        if (t == "null" || t == "~") return Node{};
        return scalar(t);
    }
    Node seq() {
        Node n;
        n.kind = Node::Seq;
        ++i_;
        ws();
        if (i_ < s_.size() && s_[i_] == ']') {
            ++i_;
            return n;
        }
        for (;;) {
            n.items.push_back(value());
            ws();
            if (i_ >= s_.size()) fail("unterminated sequence");
            if (s_[i_] == ',') {
                ++i_;
                continue;
            }
            if (s_[i_] == ']') {
                ++i_;
                return n;
            }
            fail("expected ',' or ']'");
        }
    }
    Node map() {
        Node n;
        n.kind = Node::Map;
        ++i_;
        ws();
        if (i_ < s_.size() && s_[i_] == '}') {
            ++i_;
            return n;
        }
        for (;;) {
            ws();
            Node key = value();
            if (key.kind != Node::Scalar) fail("mapping key must be a scalar");
            ws();
            if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
            ++i_;
            Node v = value();
            if (n.get(key.text)) fail("duplicate key '" + key.text + "'");
            n.fields.emplace_back(key.text, std::move(v));
            ws();
            if (i_ >= s_.size()) fail("unterminated mapping");
            if (s_[i_] == ',') {
                ++i_;
                continue;
            }
            if (s_[i_] == '}') {
                ++i_;
                return n;
            }
            fail("expected ',' or '}'");
        }
    }
};

int bracket_balance(const std::string& s) {
    int depth = 0;
    char quote = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (quote) {
            if (c == '\\' && quote == '"') ++i;
            else if (c == quote) quote = 0;
        } else if (c == '"' || c == '\'') {
            quote = c;
        } else if (c == '[' || c == '{') {
            ++depth;
        } else if (c == ']' || c == '}') {
            --depth;
        }
    }
    return depth;
}

// Position of the ':' that separates a block mapping key, or npos.
size_t key_colon(const std::string& s) {
    char quote = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (quote) {
            if (c == quote) quote = 0;
        } else if (c == '"' || c == '\'') {
            quote = c;
        } else if (c == '[' || c == '{') {
            return std::string::npos;
        } else if (c == ':' && (i + 1 == s.size() || s[i + 1] == ' ')) {
            return i;
        }
    }
    return std::string::npos;
}

bool is_item(const std::string& body) { return body == "-" || body.rfind("- ", 0) == 0; }

class Block {
public:
    Block(std::vector<Line> lines, std::string origin) : lines_(std::move(lines)), origin_(std::move(origin)) {}

    Node document() {
        if (lines_.empty()) return Node{};
        Node n = node(lines_[0].indent);
        if (pos_ != lines_.size()) fail(lines_[pos_], "unexpected indentation");
        return n;
    }

private:
    std::vector<Line> lines_;
    std::string origin_;
    size_t pos_ = 0;

    [[noreturn]] void fail(const Line& l, const std::string& what) const {
        throw ParseError(origin_ + ":" + std::to_string(l.number) + ": " + what);
    }

    Node node(int indent) {
        return is_item(lines_[pos_].body) ? sequence(indent) : mapping(indent);
    }

    // The value text after "key:" or "- ": a scalar, or a flow collection
    // that may continue on the following lines.
    Node inline_value(std::string text, const Line& where) {
        if (!text.empty() && (text[0] == '[' || text[0] == '{')) {
            while (bracket_balance(text) > 0) {
                if (pos_ >= lines_.size()) fail(where, "unterminated flow collection");
                text += "\n" + lines_[pos_++].body;
            }
            return Flow(text, origin_ + ":" + std::to_string(where.number)).document();
        }
        if (!text.empty() && (text[0] == '"' || text[0] == '\''))
            return Flow(text, origin_ + ":" + std::to_string(where.number)).document();
        if (text == "null" || text == "~") return Node{};
        return scalar(text);
    }

    Node nested_or_null(int indent, bool allow_same_indent_seq) {
        if (pos_ < lines_.size()) {
            const Line& nx = lines_[pos_];
            if (nx.indent > indent) return node(nx.indent);
            if (allow_same_indent_seq && nx.indent == indent && is_item(nx.body)) return sequence(indent);
        }
        return Node{};
    }

    Node mapping(int indent) {
        Node n;
        n.kind = Node::Map;
        while (pos_ < lines_.size() && lines_[pos_].indent == indent && !is_item(lines_[pos_].body)) {
            const Line l = lines_[pos_++];
            const size_t c = key_colon(l.body);
            if (c == std::string::npos) fail(l, "expected 'key: value'");
            std::string key = trim(l.body.substr(0, c));
            if (!key.empty() && (key[0] == '"' || key[0] == '\'')) key = Flow(key, origin_).document().text;
            const std::string rest = trim(l.body.substr(c + 1));
            if (n.get(key)) fail(l, "duplicate key '" + key + "'");
            n.fields.emplace_back(key, rest.empty() ? nested_or_null(indent, true) : inline_value(rest, l));
        }
        return n;
    }

    Node sequence(int indent) {
        Node n;
        n.kind = Node::Seq;
        while (pos_ < lines_.size() && lines_[pos_].indent == indent && is_item(lines_[pos_].body)) {
            Line l = lines_[pos_++];
            const std::string rest = l.body.size() > 1 ? trim(l.body.substr(1)) : std::string();
            if (rest.empty()) {
                n.items.push_back(nested_or_null(indent, false));
            } else if (key_colon(rest) != std::string::npos) {
                // "- key: value" opens a mapping indented past the dash
                const int inner = indent + int(l.body.find(rest));
                --pos_;
                lines_[pos_].indent = inner;
                lines_[pos_].body = rest;
                n.items.push_back(mapping(inner));
            } else {
                n.items.push_back(inline_value(rest, l));
            }
        }
        return n;
    }
};

}  // namespace

Node parse_yaml(const std::string& text, const std::string& origin) {
    std::vector<Line> lines;
    std::istringstream in(text);
    std::string raw;
    int number = 0;
    while (std::getline(in, raw)) {
        ++number;
        const std::string body = strip_comment(raw);
        const std::string t = trim(body);
        if (t.empty() || t == "---") continue;
        size_t ind = 0;
        while (ind < body.size() && body[ind] == ' ') ++ind;
        if (ind < body.size() && body[ind] == '\t')
            throw ParseError(origin + ":" + std::to_string(number) + ": tab indentation");
        lines.push_back({int(ind), t, number});
    }
    if (lines.empty()) return Node{};
    if (lines[0].body[0] == '{' || lines[0].body[0] == '[') {
        std::string all;
        for (const auto& l : lines) all += l.body + "\n";
        return Flow(all, origin).document();
    }
    return Block(std::move(lines), origin).document();
}

// The two input conveniences of SonicFile, rewritten to plain YAML before
// parsing as the reference does (normalizeSonicSyntax,
// src/infrastructure/io/serialization/SF_serialization.cpp:35-60):
//   `patch: fixedValue: V`  ->  `patch:` / `  fixedValue: V`
//   `[1 0 0]`               ->  `[1, 0, 0]`
std::string normalize_sonic_syntax(const std::string& text) {
    static const std::regex compact(R"(^([ \t]*)([^:#\n][^:\n]*):[ \t]*([A-Za-z][A-Za-z0-9_-]*)[ \t]*:[ \t]*(.*)$)");
    static const std::regex bracket(R"(\[([^\[\],#'"]+)\])");
    std::istringstream in(text);
    std::ostringstream out;
    std::string line;
    while (std::getline(in, line)) {
        std::smatch m;
        if (std::regex_match(line, m, compact))
            line = m[1].str() + m[2].str() + ":\n" + m[1].str() + "  " + m[3].str() + ": " + m[4].str();
        std::string fixed;
        size_t pos = 0;
        for (std::sregex_iterator it(line.begin(), line.end(), bracket), end; it != end; ++it) {
            const std::smatch& b = *it;
            fixed.append(line, pos, (size_t)b.position() - pos);
            std::istringstream words(b[1].str());
            std::vector<std::string> tok;
            for (std::string w; words >> w;) tok.push_back(w);
            if (tok.size() > 1) {
                fixed += "[";
                for (size_t i = 0; i < tok.size(); ++i) fixed += (i ? ", " : "") + tok[i];
                fixed += "]";
            } else {
                fixed += b.str();
            }
            pos = (size_t)(b.position() + b.length());
        }
        fixed.append(line, pos, std::string::npos);
        out << fixed << "\n";
    }
    return out.str();
}

Node load_yaml_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw ParseError("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return parse_yaml(normalize_sonic_syntax(ss.str()), path);
}

}  // namespace sfh
