// sfh_catalog.cpp -- provider catalogs (see sfh_catalog.hpp).
#include "sfh_catalog.hpp"

#include <algorithm>
#include <stdexcept>

#include "../../include/sonicsolver_b200.h"

namespace sfh {

const char* to_string(BindingStatus s) {
    switch (s) {
    case BindingStatus::Resolved: return "Resolved";
    case BindingStatus::Unsupported: return "Unsupported";
    case BindingStatus::Invalid: return "Invalid";
    }
    return "?";
}

void TermCatalog::add(TermProvider p) {
    if (p.id.empty() || !p.match) throw std::invalid_argument("term provider needs an id and a matcher");
    for (const auto& q : providers_)
        if (q.id == p.id) throw std::invalid_argument("duplicate term provider: " + p.id);
    providers_.push_back(std::move(p));
}

ResolvedTerm TermCatalog::resolve(const TermMatch& m, const std::string& selected) const {
    std::vector<const TermProvider*> hits;
    for (const auto& p : providers_)
        if ((selected.empty() || p.id == selected) && p.match(m)) hits.push_back(&p);
    std::sort(hits.begin(), hits.end(), [](const TermProvider* a, const TermProvider* b) { return a->id < b->id; });
    ResolvedTerm r;
    r.recipe = m.recipe;
    const std::string what = "equation '" + m.equation + "' term '" + m.operator_name + "'" +
                             (m.recipe_token.empty() ? "" : " with recipe '" + m.recipe_token + "'");
    if (hits.size() == 1) {
        r.id = hits[0]->id;
        r.owner = hits[0]->owner;
        r.status = BindingStatus::Resolved;
    } else if (hits.empty()) {
        r.reason = "no term provider for " + what + (selected.empty() ? "" : " (binding '" + selected + "')");
    } else {
        r.status = BindingStatus::Invalid;
        r.reason = "ambiguous term providers for " + what + ": ";
        for (size_t i = 0; i < hits.size(); ++i) r.reason += (i ? ", " : "") + hits[i]->id;
    }
    return r;
}

TermCatalog TermCatalog::gpu() {
    TermCatalog c;
    c.add({"convection.conservativeFlux",
           [](const TermMatch& m) {
               return m.operator_name == "div" && m.equation_method == "ConservativeResidual" && m.recipe >= 0 &&
                      sfg_recipe_name(m.recipe) != nullptr;
           },
           "sonicsolver_b200"});
    return c;
}

void ProviderCatalog::add(RuntimeProvider p) {
    if (p.id.empty()) throw std::invalid_argument("runtime provider needs an id");
    for (const auto& q : providers_)
        if (q.id == p.id) throw std::invalid_argument("duplicate runtime provider: " + p.id);
    providers_.push_back(std::move(p));
}

ResolvedOperation ProviderCatalog::resolve(const Operation& op, const std::string& selected) const {
    ResolvedOperation r;
    r.op = op.op;
    const auto it = std::find_if(providers_.begin(), providers_.end(),
                                 [&](const RuntimeProvider& p) { return p.id == selected; });
    const auto has_all = [&](const RuntimeProvider& p) {
        return !op.requirements.empty() &&
               std::all_of(op.requirements.begin(), op.requirements.end(), [&](Capability need) {
                   return std::find(p.capabilities.begin(), p.capabilities.end(), need) != p.capabilities.end();
               });
    };
    if (selected.empty()) r.reason = "no runtime provider selected for '" + op.op + "'";
    else if (it == providers_.end()) r.reason = "runtime provider '" + selected + "' is not registered";
    else if (!has_all(*it)) r.reason = "runtime provider '" + selected + "' lacks a capability of '" + op.op + "'";
    else {
        r.provider = it->id;
        r.status = BindingStatus::Resolved;
    }
    return r;
}

ProviderCatalog ProviderCatalog::gpu() {
    ProviderCatalog c;
    c.add({"flow.conservative", {Capability::ConservativeExplicit}});
    return c;
}

}  // namespace sfh
