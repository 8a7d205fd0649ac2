// sfh_case.cpp -- case directory reader (see sfh_case.hpp).
#include "sfh_case.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>

#include "sfh_yaml.hpp"

namespace sfh {
namespace {

bool exists(const std::string& path) { return std::ifstream(path).good(); }

std::string join(const std::string& dir, const std::string& rel) { return dir + "/" + rel; }

// File of a registry entry (`entry: {type: ..., file: ...}`), else `fallback`.
std::string registry_file(const std::string& dir, const std::string& registry, const std::string& entry,
                          const std::string& fallback) {
    const std::string reg = join(dir, registry);
    if (exists(reg)) {
        const Node r = load_yaml_file(reg);
        if (const Node* e = r.get(entry))
            if (const Node* f = e->get("file")) return join(dir, f->str());
    }
    return join(dir, fallback);
}

std::vector<double> numbers(const Node& n, size_t want, const std::string& what) {
    std::vector<double> v;
    if (n.is_scalar()) v.push_back(n.number());
    else if (n.is_seq())
        for (const auto& x : n.items) v.push_back(x.number());
    if (v.size() != want)
        throw ParseError(what + ": expected " + std::to_string(want) + " component(s)");
    return v;
}

InitialValue initial_value(const Node& n, size_t comps, const std::string& var) {
    InitialValue iv;
    if (!n.is_map()) {  // bare value: uniform
        iv.base = numbers(n, comps, var);
        return iv;
    }
    for (const auto& kv : n.fields) {
        if (kv.first == "uniform" || kv.first == "default") {
            iv.base = numbers(kv.second, comps, var + "." + kv.first);
        } else if (kv.second.is_map()) {
            throw Unsupported("internalField " + var + "." + kv.first +
                              ": generated set values (type: ...) are not supported for " + var);
        } else {
            iv.sets.emplace_back(kv.first, numbers(kv.second, comps, var + "." + kv.first));
        }
    }
    if (iv.base.empty()) iv.base.assign(comps, 0.0);
    return iv;
}

std::string lower(std::string s) {
    for (auto& ch : s) ch = char(std::tolower((unsigned char)ch));
    return s;
}

// The convection recipe token of a numerics file, in either form the
// reference reads: `terms: {convection: weno5Rusanov}`, or
// `convection: {default: WENO5, flux: Rusanov, reconstruction: ...}` whose
// scheme and flux-splitter names compose the same token
// (src/app/application/model/parsing/SF_numericsParser.h:11-162).
std::string convection_token(const Node& nu) {
    if (const Node* terms = nu.get("terms")) {
        for (const auto& kv : terms->fields)
            if (kv.first != "convection")
                throw Unsupported("term '" + kv.first + "': the provider implements the convection term only");
        return terms->at("convection").str();
    }
    const Node* cv = nu.get("convection");
    if (!cv) throw Unsupported("numerics select no convection scheme");
    if (const Node* r = cv->get("reconstruction"))
        if (lower(r->str()) != "characteristic" && lower(r->str()) != "char")
            throw Unsupported("reconstruction '" + r->str() + "': the provider reconstructs characteristic variables");
    // a `diffusion:` block is inert while transport is disabled (checked by the caller)
    const std::string scheme = lower(cv->at("default").str());
    const std::string f = cv->get("flux") ? lower(cv->at("flux").str()) : "rusanov";
    std::string flux;
    if (f == "rusanov" || f == "localaxfriedrichs" || f == "llf") flux = "Rusanov";
    else if (f == "roe") flux = "Roe";
    else if (f == "laxfriedrichs" || f == "lf" || f == "lxf" || f == "laxf") flux = "LaxFriedrichs";
    else if (f == "laxwendroff" || f == "lw") flux = "LaxWendroff";
    else if (f == "stegerwarming" || f == "sw" || f == "steger") flux = "Steger";  // TermRecipeId name
    else throw Unsupported("flux splitter '" + cv->at("flux").str() + "'");
    return scheme + flux;
}

bool switched_on(const Node& n, const std::string& key) {
    const Node* v = n.get(key);
    return v && v->is_scalar() && v->boolean();
}

// Terms a numerics file switches on beyond convection.  A `diffusion:
// default:` scheme is live unless `transport: enable: false` turns it off
// (SF_nativeBinding.cpp:454-462); `sources: default:` names the gravity /
// MRF / wall-heat sources (SF_nativeDecode.cpp:1074-1078, parsed by
// parseSourceKinds, SF_modelConfigParser.h:14-33, none/off/false naming
// none).
void numerics_physics(const Node& nu, std::vector<std::string>& out) {
    bool disabled = false;
    if (const Node* tr = nu.get("transport"))
        if (const Node* en = tr->get("enable")) disabled = !en->boolean();
    if (const Node* df = nu.get("diffusion"))
        if (const Node* d = df->get("default"))
            if (!disabled)
                out.push_back("viscous terms (numerics diffusion '" + d->str() +
                              "' without transport.enable: false): the provider implements the Euler equations");
    if (const Node* src = nu.get("sources"))
        if (const Node* d = src->get("default")) {
            const std::string s = lower(d->str());
            if (!s.empty() && s != "none" && s != "off" && s != "false")
                out.push_back("source terms '" + d->str() + "' (numerics sources)");
        }
}

// Switches of the model modules (models/models.yaml entries by type) and of
// the equation system and ILW entries of solvers/solvers.yaml that select
// physics beyond the inviscid single-fluid Euler equations.  Gravity and MRF
// modules act only through numerics sources; geometry entries only through
// an immersed boundary.
void module_physics(const std::string& dir, std::vector<std::string>& out) {
    std::vector<std::pair<std::string, std::string>> modules;  // type, file
    const std::string reg = join(dir, "models/models.yaml");
    if (exists(reg)) {
        const Node r = load_yaml_file(reg);
        for (const auto& kv : r.fields)
            if (kv.second.is_map() && kv.second.get("type") && kv.second.get("file"))
                modules.emplace_back(kv.second.at("type").str(), join(dir, kv.second.at("file").str()));
    } else {
        for (const char* t : {"IBM", "turbulence", "multiPhase", "phaseChange", "thermophysical"})
            modules.emplace_back(t, join(dir, std::string("models/") + t + ".yaml"));
    }
    for (const auto& m : modules) {
        if (!exists(m.second)) continue;
        const Node f = load_yaml_file(m.second);
        const Node* body = f.get(m.first);  // `IBM: {enabled: ...}` or top-level keys
        const Node& b = body && body->is_map() ? *body : f;
        if (m.first == "IBM" && switched_on(b, "enabled")) {
            out.push_back("immersed boundary (" + m.second.substr(dir.size() + 1) + " enabled)");
        } else if (m.first == "turbulence" && switched_on(b, "enabled")) {
            const std::string st = b.get("simulationType") ? lower(b.at("simulationType").str()) : "";
            if (st != "laminar" && st != "dns" && st != "none")
                out.push_back("turbulence model (simulationType '" + b.at("simulationType").str() + "')");
        } else if (m.first == "multiPhase" && switched_on(f, "multiPhases")) {
            out.push_back("multiphase flow (" + m.second.substr(dir.size() + 1) + ")");
        } else if (m.first == "phaseChange" && switched_on(b, "enabled")) {
            out.push_back("phase change (" + m.second.substr(dir.size() + 1) + ")");
        } else if (m.first == "thermophysical") {
            if (const Node* t = f.get("temperature"))
                if (switched_on(*t, "enabled")) out.push_back("temperature equation (thermophysical temperature.enabled)");
        }
    }
    const std::string eq = registry_file(dir, "solvers/solvers.yaml", "equations", "solvers/equations.yaml");
    if (exists(eq)) {
        const Node e = load_yaml_file(eq);
        if (const Node* p = e.get("preset"))
            if (p->str() != "compressible")
                out.push_back("equation preset '" + p->str() + "': the provider implements 'compressible'");
    }
    const std::string ilw = registry_file(dir, "solvers/solvers.yaml", "ILW", "solvers/ILW.yaml");
    if (exists(ilw)) {
        const Node f = load_yaml_file(ilw);
        const Node* body = f.get("ILW");
        if (body && switched_on(*body, "enabled")) out.push_back("inverse Lax-Wendroff boundaries (ILW enabled)");
    }
}

// One patch entry: `zeroGradient`, `{type: fixedValue, value: V}` or the
// compact `{fixedValue: V}` (compactBoundary, SF_case.cpp:22-29).
FieldCondition condition(const Node& n, const std::string& what) {
    FieldCondition fc;
    auto values = [&](const Node& v) {
        std::vector<double> out;
        if (v.is_scalar()) out.push_back(v.number());
        else if (v.is_seq())
            for (const auto& x : v.items) out.push_back(x.number());
        else if (v.kind != Node::Null) throw ParseError(what + ": value must be a number or a list");
        return out;
    };
    if (n.is_scalar()) {
        fc.type = n.str();
    } else if (n.is_map() && n.get("type")) {
        fc.type = n.at("type").str();
        if (const Node* v = n.get("value")) fc.value = values(*v);
    } else if (n.is_map() && n.fields.size() == 1) {
        fc.type = n.fields[0].first;
        fc.value = values(n.fields[0].second);
    } else {
        throw ParseError(what + ": boundary condition must contain exactly one condition type");
    }
    return fc;
}

}  // namespace

CaseSpec load_case(const std::string& dir) {
    CaseSpec c;
    c.dir = dir;
    if (exists(join(dir, "case.yaml"))) {
        const Node cs = load_yaml_file(join(dir, "case.yaml"));
        if (const Node* nm = cs.get("name")) c.name = nm->str();
    }
    // ---- solvers
    const Node rt = load_yaml_file(registry_file(dir, "solvers/solvers.yaml", "runtime", "solvers/runtime.yaml"));
    if (const Node* v = rt.get("startTime")) c.start_time = v->number();
    c.end_time = rt.at("endTime").number();
    if (const Node* v = rt.get("CFL")) c.cfl = v->number();
    if (const Node* v = rt.get("writeControl")) c.write_control = v->str();
    if (const Node* v = rt.get("writeInterval")) c.write_interval = v->number();
    if (const Node* v = rt.get("writeInitial")) c.write_initial = v->boolean();
    if (const Node* v = rt.get("maxDeltaT")) c.max_dt = v->number();
    if (const Node* o = rt.get("output")) {
        if (const Node* v = o->get("jobName")) c.job_name = v->str();
        if (const Node* v = o->get("outputDir")) c.output_dir = v->str();
    }
    if (c.job_name.empty()) c.job_name = c.name.empty() ? "case" : c.name;
    const Node nu = load_yaml_file(registry_file(dir, "solvers/solvers.yaml", "numerics", "solvers/numerics.yaml"));
    c.time_recipe = nu.at("time").at("default").str();
    c.convection = convection_token(nu);
    if (const Node* tr = nu.get("transport"))
        if (const Node* en = tr->get("enable"))
            if (en->boolean()) throw Unsupported("transport enabled: viscous terms are outside the explicit Euler path");
    numerics_physics(nu, c.unsupported_physics);
    const std::string alg = registry_file(dir, "solvers/solvers.yaml", "algorithm", "solvers/algorithm.yaml");
    c.algorithm = exists(alg) ? load_yaml_file(alg).at("type").str() : "densityBase";
    module_physics(dir, c.unsupported_physics);
    // ---- thermodynamics
    const std::string th = registry_file(dir, "models/models.yaml", "thermoDynamics", "models/thermoDynamics.yaml");
    if (exists(th)) {
        const Node t = load_yaml_file(th);
        if (const Node* td = t.get("thermoDynamics"))
            if (const Node* eos = td->get("equationOfState"))
                if (eos->str() != "perfectGas")
                    throw Unsupported("equationOfState '" + eos->str() + "': the provider implements perfectGas");
        if (const Node* pr = t.get("properties"))
            if (const Node* eos = pr->get("equationOfState")) {
                if (const Node* g = eos->get("gamma")) c.gamma = g->number();
                if (const Node* r = eos->get("R")) c.gas_R = r->number();
            }
    }
    // ---- mesh: one block (structuredMesh generation, decodeParameters,
    // src/infrastructure/io/mesh/SF_meshParameters.cpp:9-48)
    const Node gen = load_yaml_file(registry_file(dir, "mesh/mesh.yaml", "generation", "mesh/generation.yaml"));
    MeshGeneration& m = c.mesh;
    m.scale = gen.get("scale") ? gen.at("scale").number() : 1.0;
    if (!(m.scale > 0) || !std::isfinite(m.scale)) throw ParseError("mesh: scale must be finite and > 0");
    if (const Node* ng = gen.get("nGhost")) c.ghost_layers = int(ng->integer());
    m.n_ghost = c.ghost_layers;
    const Node& verts = gen.at("vertices");
    const Node& blocks = gen.at("blocks");
    if (!blocks.is_seq() || blocks.items.size() != 1)
        throw Unsupported("mesh: the provider runs a single structured block");
    for (const auto& v : verts.items) {
        const auto x = numbers(v, 3, "vertex");
        m.vertices.push_back({x[0], x[1], x[2]});
    }
    const Node& blk = blocks.items[0];
    const auto hex = numbers(blk.at("vertices"), 8, "blocks[0].vertices");
    for (int i = 0; i < 8; ++i) {
        m.verts[i] = int(hex[i]);
        if (m.verts[i] < 0 || m.verts[i] >= int(m.vertices.size()) || double(m.verts[i]) != hex[i])
            throw ParseError("mesh: blocks[0].vertices holds an invalid vertex index");
    }
    const auto cells = numbers(blk.at("cells"), 3, "blocks[0].cells");
    for (int d = 0; d < 3; ++d) {
        c.cells[d] = m.cells[d] = int(cells[d]);
        if (m.cells[d] < 1 || double(m.cells[d]) != cells[d]) throw ParseError("mesh: cells must be positive integers");
    }
    if (const Node* gr = blk.get("grading")) {
        const auto g = numbers(*gr, 3, "grading");
        for (int d = 0; d < 3; ++d) {
            m.grading[d] = g[d];
            if (!(g[d] > 0) || !std::isfinite(g[d])) throw ParseError("mesh: grading must be finite and > 0");
        }
    }
    if (const Node* edges = gen.get("edges")) {
        for (const auto& e : edges->items) {
            if (e.at("type").str() != "arc")
                throw Unsupported("mesh: edge type '" + e.at("type").str() + "' (the generator builds arcs)");
            const auto ends = numbers(e.at("vertices"), 2, "edges[].vertices");
            const auto pt = numbers(e.at("point"), 3, "edges[].point");
            ArcEdge a;
            a.v0 = int(ends[0]);
            a.v1 = int(ends[1]);
            for (int d = 0; d < 3; ++d) a.point[d] = pt[d];
            if (a.v0 < 0 || a.v1 < 0 || a.v0 >= int(m.vertices.size()) || a.v1 >= int(m.vertices.size()))
                throw ParseError("mesh: edges[].vertices holds an invalid vertex index");
            m.edges.push_back(a);
        }
    }
    for (int d = 0; d < 3; ++d) {  // the block's bounding box
        c.lo[d] = 1e300;
        c.hi[d] = -1e300;
        for (int i = 0; i < 8; ++i) {
            c.lo[d] = std::min(c.lo[d], m.vertices[m.verts[i]][d] * m.scale);
            c.hi[d] = std::max(c.hi[d], m.vertices[m.verts[i]][d] * m.scale);
        }
    }
    c.curvilinear = !m.uniform_box();
    // ---- fields
    const std::string inf = registry_file(dir, "fields/fields.yaml", "internalField", "fields/internalField.yaml");
    const Node in = load_yaml_file(inf);
    c.rho = initial_value(in.at("rho"), 1, "rho");
    c.U = initial_value(in.at("U"), 3, "U");
    c.p = initial_value(in.at("p"), 1, "p");
    const Node bc = load_yaml_file(registry_file(dir, "fields/fields.yaml", "boundaries", "fields/boundaries.yaml"));
    for (const char* var : {"rho", "U", "p"}) {
        const Node* vb = bc.get(var);
        if (!vb) continue;
        for (const auto& kv : vb->fields) {
            c.patch_bc[kv.first][var] = condition(kv.second, std::string(var) + "." + kv.first);
            c.bc_order[var].push_back(kv.first);
        }
    }
    // field declarations of the registry (its "fields" registry entries,
    // src/infrastructure/io/case/SF_case.cpp:115-150): output switch and name
    const std::string reg = join(dir, "fields/fields.yaml");
    if (exists(reg)) {
        const Node r = load_yaml_file(reg);
        for (const auto& kv : r.fields) {
            const std::string& k = kv.first;
            if (k == "SonicFile" || k == "default" || k == "internalField" || k == "boundaries") continue;
            CaseSpec::DeclaredField f;
            f.name = f.output_name = k;
            if (kv.second.is_map()) {
                if (const Node* o = kv.second.get("output")) f.output = o->boolean();
                if (const Node* on = kv.second.get("outputName")) f.output_name = on->str();
            }
            c.declared_fields.push_back(f);
        }
    }
    return c;
}

namespace {

// Boundary patches of the structured generator per axis (low end, high end)
// and their aliases.
struct AxisPatches {
    const char* lo;
    const char* hi;
    const char* alt_lo;
    const char* alt_hi;
};
const AxisPatches kPatches[3] = {{"Left", "Right", "inlet", "outlet"},
                                 {"sideWalls", "sideWalls", "walls", "walls"},
                                 {"frontBack", "frontBack", "walls", "walls"}};

using PatchConditions = std::map<std::string, FieldCondition>;

const PatchConditions* patch_condition(const CaseSpec& c, const char* name, const char* alt) {
    auto it = c.patch_bc.find(name);
    if (it != c.patch_bc.end()) return &it->second;
    it = c.patch_bc.find(alt);
    return it != c.patch_bc.end() ? &it->second : nullptr;
}

bool has_type(const PatchConditions& pc, const char* token) {
    for (const auto& kv : pc)
        if (lower(kv.second.type) == token) return true;
    return false;
}

// Law of one field from its token (valueBCTypeValue,
// app/application/model/compatibility/private/SF_valueParser.cpp:146-164:
// case-insensitive; noSlip / slip are velocity laws: fixedValue 0 and
// symmetry).
int field_law(const FieldCondition& fc, bool velocity, const std::string& what, double* value) {
    const std::string t = lower(fc.type);
    const size_t want = velocity ? 3 : 1;
    if (velocity && (t == "noslip" || t == "slip")) {
        if (t == "noslip") value[0] = value[1] = value[2] = 0.0;
        return t == "noslip" ? SFG_LAW_FIXED_VALUE : SFG_LAW_SYMMETRY;
    }
    if (t == "zerogradient" || t == "zero_gradient") return SFG_LAW_ZERO_GRADIENT;
    if (t == "symmetry" || t == "symmetryplane") return SFG_LAW_SYMMETRY;
    if (t == "fixedvalue" || t == "fixed_value") {
        if (fc.value.size() != want)
            throw ParseError(what + ": fixedValue needs " + std::to_string(want) + " number(s)");
        for (size_t i = 0; i < want; ++i) value[i] = fc.value[i];
        return SFG_LAW_FIXED_VALUE;
    }
    throw Unsupported(what + ": condition '" + fc.type +
                      "' is not provided on the GPU (fixedValue, zeroGradient, symmetry, slip, noSlip, periodic, "
                      "empty are)");
}

// Boundary kind (and laws) of one axis end.
int end_kind(const PatchConditions& pc, const char* patch, sfg_boundary_law& law) {
    if (has_type(pc, "periodic") || has_type(pc, "cyclic")) {
        for (const auto& kv : pc) {
            const std::string t = lower(kv.second.type);
            if (t != "periodic" && t != "cyclic")
                throw Unsupported(std::string("patch '") + patch + "': periodic must hold for every field");
        }
        return SFG_BC_PERIODIC;
    }
    const FieldCondition* f[3] = {nullptr, nullptr, nullptr};
    const char* names[3] = {"rho", "U", "p"};
    for (int i = 0; i < 3; ++i) {
        auto it = pc.find(names[i]);
        if (it == pc.end())
            throw Unsupported(std::string("patch '") + patch + "': " + names[i] +
                              " has no condition while other fields have one (the provider needs rho, U and p)");
        f[i] = &it->second;
    }
    const std::string where = std::string("patch '") + patch + "' ";
    law = sfg_boundary_law{};
    law.rho = field_law(*f[0], false, where + "rho", &law.rho_value);
    law.velocity = field_law(*f[1], true, where + "U", law.velocity_value);
    law.pressure = field_law(*f[2], false, where + "p", &law.pressure_value);
    if (law.rho == SFG_LAW_ZERO_GRADIENT && law.velocity == SFG_LAW_ZERO_GRADIENT &&
        law.pressure == SFG_LAW_ZERO_GRADIENT)
        return SFG_BC_TRANSMISSIVE;
    return SFG_BC_LAW;
}

}  // namespace

GridSetup build_grid(const CaseSpec& c) {
    if (c.algorithm != "densityBase")
        throw Unsupported("algorithm '" + c.algorithm + "': the provider implements the densityBase explicit path");
    if (!c.unsupported_physics.empty()) {
        std::string why = c.unsupported_physics[0];
        for (size_t i = 1; i < c.unsupported_physics.size(); ++i) why += "; " + c.unsupported_physics[i];
        throw Unsupported(why);
    }
    GridSetup g;
    bool active[3];
    for (int d = 0; d < 3; ++d) {
        const AxisPatches& P = kPatches[d];
        const PatchConditions* lo = patch_condition(c, P.lo, P.alt_lo);
        const PatchConditions* hi = patch_condition(c, P.hi, P.alt_hi);
        const bool empty = (lo && has_type(*lo, "empty")) || (hi && has_type(*hi, "empty"));
        if (empty || (c.cells[d] <= 1 && !lo && !hi)) {
            active[d] = false;
            continue;
        }
        // a patch without a condition keeps its initial ghost state and its
        // boundary node is advanced (SF_applicator.h:162-187): SFG_BC_FROZEN
        active[d] = true;
        g.grid.bc_lo[d] = lo ? end_kind(*lo, P.lo, g.laws[2 * d]) : SFG_BC_FROZEN;
        g.grid.bc_hi[d] = hi ? end_kind(*hi, P.hi, g.laws[2 * d + 1]) : SFG_BC_FROZEN;
        if ((g.grid.bc_lo[d] == SFG_BC_PERIODIC) != (g.grid.bc_hi[d] == SFG_BC_PERIODIC))
            throw Unsupported(std::string("axis ") + "xyz"[d] + ": periodic must hold at both ends");
    }
    if ((active[1] && !active[0]) || (active[2] && !active[1]))
        throw Unsupported("active axes must be x, x-y or x-y-z (the provider does not permute axes)");
    g.grid.dim = int(active[0]) + int(active[1]) + int(active[2]);
    if (g.grid.dim == 0) throw Unsupported("no active axis");
    for (int d = 0; d < 3; ++d) {
        const double len = c.hi[d] - c.lo[d];
        g.origin[d] = c.lo[d];
        if (active[d]) {
            if (c.cells[d] < 2) throw Unsupported(std::string("axis ") + "xyz"[d] + " needs at least 2 cells");
            g.nodes[d] = g.grid.bc_lo[d] == SFG_BC_PERIODIC ? c.cells[d] : c.cells[d] + 1;
            g.grid.h[d] = len / c.cells[d];
        } else {
            g.nodes[d] = 1;
            g.grid.h[d] = len > 0 ? len : 1.0;
            g.grid.bc_lo[d] = g.grid.bc_hi[d] = SFG_BC_TRANSMISSIVE;
        }
        g.grid.n[d] = g.nodes[d];
        if (!(g.grid.h[d] > 0)) throw Unsupported("degenerate block extent");
        if (c.curvilinear && g.grid.bc_lo[d] == SFG_BC_PERIODIC)
            throw Unsupported("periodic ends on a graded or curved block (the reference has no periodic boundary)");
    }
    // initial state: base values, then the named sets in file order
    const int nx = g.nodes[0], ny = g.nodes[1], nz = g.nodes[2];
    const int split = nx / 2;  // leftHalf: i < nx / 2
    auto value_at = [&](const InitialValue& iv, int i, size_t comp) {
        double v = iv.base[comp];
        for (const auto& s : iv.sets) {
            bool in;
            if (s.first == "leftHalf") in = i < split;
            else if (s.first == "rightHalf") in = i >= split;
            else if (s.first == "all") in = true;
            else throw Unsupported("internalField set '" + s.first + "' is not a generated structured set");
            if (in) v = s.second[comp];
        }
        return v;
    };
    g.q.resize(size_t(nx) * ny * nz * 5);
    const double gm1 = c.gamma - 1.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double rho = value_at(c.rho, i, 0), p = value_at(c.p, i, 0);
                const double u[3] = {value_at(c.U, i, 0), value_at(c.U, i, 1), value_at(c.U, i, 2)};
                if (!(rho > 0) || !(p > 0)) throw Unsupported("initial state has rho <= 0 or p <= 0");
                double* q = &g.q[((size_t(k) * ny + j) * nx + i) * 5];
                q[0] = rho;
                q[1] = rho * u[0];
                q[2] = rho * u[1];
                q[3] = rho * u[2];
                q[4] = p / gm1 + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            }
    return g;
}

}  // namespace sfh
