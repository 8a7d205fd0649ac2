// sfh_checkpoint.cpp -- restart files (see sfh_checkpoint.hpp).
#include "sfh_checkpoint.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>

namespace sfh {

namespace {

// ---- writer

void put_number(std::ostream& o, double v) {
    char buf[32];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    o << buf;
}

void put_field(std::ostream& o, const char* name, const char* type, int comps, int first, size_t nodes,
               const std::vector<double>& q, bool last) {
    o << "    \"" << name << "\": {\n      \"descriptor\": {\"type\": \"" << type << "\", \"default\": ";
    if (comps == 1) o << "0";
    else o << "[0, 0, 0]";
    o << ", \"output\": false, \"restart\": true},\n      \"size\": " << nodes << ",\n      \"values\": [";
    for (size_t n = 0; n < nodes; ++n)
        for (int c = 0; c < comps; ++c) {
            if (n || c) o << (c ? ", " : ",\n        ");
            else o << "\n        ";
            put_number(o, q[n * 5 + first + c]);
        }
    o << "\n      ]\n    }" << (last ? "\n" : ",\n");
}

// ---- a small JSON reader: objects, arrays, numbers, strings, literals.
// Arrays of numbers are kept as a vector of doubles (a field holds millions).

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    double num = 0.0;
    std::string str;
    std::vector<double> numbers;                 // Array of numbers only
    std::vector<std::unique_ptr<Value>> items;   // Array with other members
    std::map<std::string, std::unique_ptr<Value>> members;
    const Value* get(const std::string& k) const {
        auto it = members.find(k);
        return it == members.end() ? nullptr : it->second.get();
    }
};

class Reader {
  public:
    Reader(const std::string& text, const std::string& path) : s_(text), path_(path) {}

    std::unique_ptr<Value> document() {
        auto v = value();
        skip();
        if (p_ != s_.size()) fail("trailing characters");
        return v;
    }

  private:
    const std::string& s_;
    const std::string& path_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        size_t line = 1;
        for (size_t i = 0; i < p_ && i < s_.size(); ++i) line += s_[i] == '\n';
        throw std::runtime_error(path_ + ":" + std::to_string(line) + ": " + what);
    }
    void skip() {
        while (p_ < s_.size() && std::isspace((unsigned char)s_[p_])) ++p_;
    }
    bool eat(char c) {
        skip();
        if (p_ < s_.size() && s_[p_] == c) {
            ++p_;
            return true;
        }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) fail(std::string("expected '") + c + "'");
    }
    std::string string_token() {
        expect('"');
        std::string out;
        while (p_ < s_.size() && s_[p_] != '"') {
            if (s_[p_] == '\\') {
                if (++p_ >= s_.size()) break;
                const char e = s_[p_];
                out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
            } else {
                out += s_[p_];
            }
            ++p_;
        }
        if (p_ >= s_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
    double number_token() {
        skip();
        const char* b = s_.c_str() + p_;
        char* e = nullptr;
        const double v = std::strtod(b, &e);
        if (e == b) fail("expected a number");
        p_ += size_t(e - b);
        return v;
    }
    std::unique_ptr<Value> value() {
        skip();
        if (p_ >= s_.size()) fail("unexpected end of file");
        auto v = std::make_unique<Value>();
        const char c = s_[p_];
        if (c == '{') {
            ++p_;
            v->kind = Value::Object;
            if (eat('}')) return v;
            do {
                skip();
                const std::string k = string_token();
                expect(':');
                if (v->members.count(k)) fail("duplicate key " + k);
                v->members[k] = value();
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            ++p_;
            v->kind = Value::Array;
            if (eat(']')) return v;
            skip();
            const bool numeric = p_ < s_.size() && (s_[p_] == '-' || s_[p_] == '+' || s_[p_] == '.' ||
                                                    std::isdigit((unsigned char)s_[p_]));
            do {
                if (numeric) v->numbers.push_back(number_token());
                else v->items.push_back(value());
            } while (eat(','));
            expect(']');
        } else if (c == '"') {
            v->kind = Value::String;
            v->str = string_token();
        } else if (s_.compare(p_, 4, "true") == 0 || s_.compare(p_, 5, "false") == 0) {
            v->kind = Value::Bool;
            v->num = s_[p_] == 't';
            p_ += s_[p_] == 't' ? 4 : 5;
        } else if (s_.compare(p_, 4, "null") == 0) {
            p_ += 4;
        } else {
            v->kind = Value::Number;
            v->num = number_token();
        }
        return v;
    }
};

double number_at(const Value& doc, const char* key, const std::string& path) {
    const Value* v = doc.get(key);
    if (!v || v->kind != Value::Number) throw std::runtime_error(path + ": missing number \"" + key + "\"");
    return v->num;
}

}  // namespace

bool write_checkpoint(const std::string& path, const Checkpoint& c) {
    const size_t nodes = size_t(c.nodes[0]) * c.nodes[1] * c.nodes[2];
    if (c.q.size() != nodes * 5 || !std::isfinite(c.time)) return false;
    for (double v : c.q)
        if (!std::isfinite(v)) return false;
    std::ofstream o(path);
    if (!o) return false;
    o << "{\n  \"formatVersion\": 1,\n  \"fields\": {\n";
    put_field(o, "rho", "scalar", 1, 0, nodes, c.q, false);
    put_field(o, "rhoU", "vector", 3, 1, nodes, c.q, false);
    put_field(o, "rhoE", "scalar", 1, 4, nodes, c.q, true);
    o << "  },\n  \"nodes\": [" << c.nodes[0] << ", " << c.nodes[1] << ", " << c.nodes[2] << "],\n  \"time\": ";
    put_number(o, c.time);
    o << ",\n  \"steps\": " << c.steps << ",\n  \"nextOutput\": ";
    if (std::isfinite(c.next_output)) put_number(o, c.next_output);
    else o << "null";
    o << ",\n  \"outputs\": " << c.outputs << "\n}\n";
    return bool(o);
}

Checkpoint read_checkpoint(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot read " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    const auto doc = Reader(text, path).document();
    if (doc->kind != Value::Object) throw std::runtime_error(path + ": a checkpoint is a mapping");
    if (number_at(*doc, "formatVersion", path) != 1.0) throw std::runtime_error(path + ": unsupported field version");
    Checkpoint c;
    const Value* n = doc->get("nodes");
    if (!n || n->kind != Value::Array || n->numbers.size() != 3)
        throw std::runtime_error(path + ": \"nodes\" must hold 3 numbers");
    size_t nodes = 1;
    for (int d = 0; d < 3; ++d) {
        const double x = n->numbers[d];
        if (!(x >= 1) || x != std::floor(x) || x > 1e9) throw std::runtime_error(path + ": invalid node count");
        c.nodes[d] = int(x);
        nodes *= size_t(x);
    }
    c.time = number_at(*doc, "time", path);
    const double steps = number_at(*doc, "steps", path);
    if (!(steps >= 0) || steps != std::floor(steps)) throw std::runtime_error(path + ": invalid step count");
    c.steps = int64_t(steps);
    const Value* no = doc->get("nextOutput");
    c.next_output = (no && no->kind == Value::Number) ? no->num : std::numeric_limits<double>::infinity();
    c.outputs = int(number_at(*doc, "outputs", path));
    const Value* fields = doc->get("fields");
    if (!fields || fields->kind != Value::Object) throw std::runtime_error(path + ": missing \"fields\"");
    c.q.assign(nodes * 5, 0.0);
    struct Want {
        const char* name;
        int comps, first;
    };
    for (const Want& w : {Want{"rho", 1, 0}, Want{"rhoU", 3, 1}, Want{"rhoE", 1, 4}}) {
        const Value* fld = fields->get(w.name);
        if (!fld || fld->kind != Value::Object) throw std::runtime_error(path + ": missing/unwritable field " + w.name);
        const Value* size = fld->get("size");
        const Value* values = fld->get("values");
        if (!size || size->kind != Value::Number || size->num != double(nodes) || !values ||
            values->kind != Value::Array || values->numbers.size() != nodes * size_t(w.comps) ||
            !values->items.empty())
            throw std::runtime_error(path + ": incompatible field " + w.name);
        for (size_t i = 0; i < nodes; ++i)
            for (int k = 0; k < w.comps; ++k) {
                const double v = values->numbers[i * w.comps + k];
                if (!std::isfinite(v)) throw std::runtime_error(path + ": invalid array " + w.name);
                c.q[i * 5 + w.first + k] = v;
            }
    }
    if (!std::isfinite(c.time)) throw std::runtime_error(path + ": invalid time");
    return c;
}

}  // namespace sfh
