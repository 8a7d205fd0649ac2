// sfh_catalog.hpp -- the provider catalogs that bind this library into a
// sonicSolver-style compiled plan.
//
// Two registries, with the ids and resolution rules of the reference:
//   * TermCatalog: spatial term providers.  The GPU registers
//     "convection.conservativeFlux" (the id of the reference's CPU provider,
//     src/solver/system/SF_termProviderCatalog.cpp:168-176), matching a `div`
//     term of a ConservativeResidual equation whose selected convection
//     recipe this library implements.  Resolution: exactly one match is
//     Resolved, none is Unsupported, several are Invalid (ambiguous)
//     (SF_termProviderCatalog.cpp:81-143).
//   * ProviderCatalog: runtime providers by capability.  The GPU registers
//     "flow.conservative" with ConservativeExplicit; an operation resolves
//     when the selected provider exists and has every capability the
//     operation requires (src/solver/system/SF_providerCatalog.cpp:29-47).
#pragma once

#include <functional>
#include <string>
#include <vector>

namespace sfh {

enum class BindingStatus { Resolved, Unsupported, Invalid };
const char* to_string(BindingStatus s);

// The facts of a compiled equation term a spatial provider matches on.
struct TermMatch {
    std::string equation;         // equation id, e.g. "Momentum"
    std::string equation_method;  // "ConservativeResidual"
    std::string operator_name;    // "div"
    std::string output;           // "rho", "rhoU", "rhoE"
    int recipe = -1;              // SFG_RECIPE_* from numerics terms.convection; -1: none / not provided here
    std::string recipe_token;     // the case.yaml token as written
};

struct TermProvider {
    std::string id;
    std::function<bool(const TermMatch&)> match;
    std::string owner;
};

struct ResolvedTerm {
    std::string id;
    BindingStatus status = BindingStatus::Unsupported;
    std::string reason;
    std::string owner;
    int recipe = -1;
};

class TermCatalog {
public:
    // Throws std::invalid_argument on an empty id, no matcher or a duplicate id.
    void add(TermProvider p);
    // `selected` (may be empty) restricts the candidates to one provider id.
    ResolvedTerm resolve(const TermMatch& m, const std::string& selected = "") const;
    static TermCatalog gpu();

private:
    std::vector<TermProvider> providers_;
};

enum class Capability { ConservativeExplicit, TemporalSynchronization };

struct RuntimeProvider {
    std::string id;
    std::vector<Capability> capabilities;
};

struct Operation {
    std::string op;
    std::vector<Capability> requirements;
};

struct ResolvedOperation {
    std::string op, provider;
    BindingStatus status = BindingStatus::Unsupported;
    std::string reason;
};

class ProviderCatalog {
public:
    void add(RuntimeProvider p);
    ResolvedOperation resolve(const Operation& op, const std::string& selected) const;
    static ProviderCatalog gpu();

private:
    std::vector<RuntimeProvider> providers_;
};

}  // namespace sfh
