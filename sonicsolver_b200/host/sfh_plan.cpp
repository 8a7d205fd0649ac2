// sfh_plan.cpp -- plan construction, binding table and executor.
#include "sfh_plan.hpp"

#include <sstream>
#include <stdexcept>

namespace sfh {

void OperationTable::bind(const std::string& op, const std::string& provider, OpFn fn) {
    if (!fn) throw std::invalid_argument("empty operation for '" + op + "'");
    const auto key = std::make_pair(op, provider);
    if (table_.count(key)) throw std::invalid_argument("'" + op + "' is already bound to '" + provider + "'");
    table_.emplace(key, std::move(fn));
}

const OpFn* OperationTable::find(const std::string& op, const std::string& provider) const {
    const auto it = table_.find(std::make_pair(op, provider));
    return it == table_.end() ? nullptr : &it->second;
}

namespace {
void collect_unbound(const OperationTable& t, const PlanNode& n, std::vector<std::string>& out) {
    if (n.kind == PlanKind::Op && !t.find(n.op, n.provider)) out.push_back(n.op + " @ " + n.provider);
    for (const auto& c : n.children) collect_unbound(t, c, out);
}

PlanNode op(const std::string& name, const char* id, const std::string& provider) {
    PlanNode n;
    n.kind = PlanKind::Op;
    n.name = name;
    n.op = id;
    n.provider = provider;
    return n;
}

void describe_into(const PlanNode& n, int depth, std::ostringstream& os) {
    os << std::string(2 * depth, ' ');
    switch (n.kind) {
    case PlanKind::Sequence: os << "sequence " << n.name; break;
    case PlanKind::TimeLoop: os << "time-loop " << n.name; break;
    case PlanKind::StageLoop: os << "stage-loop " << n.name << " x" << n.count; break;
    case PlanKind::Op: os << n.name << " [" << n.op << " @ " << n.provider << "]"; break;
    }
    os << "\n";
    for (const auto& c : n.children) describe_into(c, depth + 1, os);
}
}  // namespace

void OperationTable::validate(const PlanNode& plan) const {
    std::vector<std::string> missing;
    collect_unbound(*this, plan, missing);
    if (missing.empty()) return;
    std::string msg = "unbound plan operations:";
    for (const auto& m : missing) msg += " " + m;
    throw std::runtime_error(msg);
}

PlanNode conservative_explicit_plan(const std::string& provider, int stages) {
    if (stages < 1) throw std::invalid_argument("an explicit method needs at least one stage");
    PlanNode stage_loop;
    stage_loop.kind = PlanKind::StageLoop;
    stage_loop.name = "Explicit.stages";
    stage_loop.count = stages;
    stage_loop.children.push_back(op("Explicit.stage", opid::ExplicitStageExecute, provider));
    // the explicit fragment of every step (SF_builtinProviders.cpp:63-81):
    // prepare, dt, begin, stages; then the commits
    PlanNode step;
    step.kind = PlanKind::TimeLoop;
    step.name = "Explicit.step";
    step.children.push_back(op("Explicit.prepare", opid::FlowStepPrepare, provider));
    step.children.push_back(op("Explicit.dt", opid::FlowDtCompute, provider));
    step.children.push_back(op("Explicit.begin", opid::FlowStepBegin, provider));
    step.children.push_back(std::move(stage_loop));
    step.children.push_back(op("Explicit.commit", opid::FlowStepCommit, provider));
    step.children.push_back(op("Explicit.time.commit", opid::TimeCommit, provider));
    PlanNode root;
    root.kind = PlanKind::Sequence;
    root.name = "ConservativeResidual";
    root.children.push_back(std::move(step));
    return root;
}

std::string describe(const PlanNode& plan) {
    std::ostringstream os;
    describe_into(plan, 0, os);
    return os.str();
}

int PlanExecutor::run(const PlanNode& plan, StepContext& ctx) const {
    ops_.validate(plan);
    return exec(plan, ctx);
}

int PlanExecutor::exec(const PlanNode& n, StepContext& ctx) const {
    switch (n.kind) {
    case PlanKind::Op: return (*ops_.find(n.op, n.provider))(ctx);
    case PlanKind::Sequence:
        for (const auto& c : n.children)
            if (int rc = exec(c, ctx)) return rc;
        return 0;
    case PlanKind::StageLoop:
        for (ctx.stage = 0; ctx.stage < n.count; ++ctx.stage)
            for (const auto& c : n.children)
                if (int rc = exec(c, ctx)) return rc;
        ctx.stage = 0;
        return 0;
    case PlanKind::TimeLoop:
        while (!ctx.stop) {
            for (const auto& c : n.children) {
                if (int rc = exec(c, ctx)) return rc;
                if (ctx.stop) break;  // the dt operation ends the loop at t_end
            }
        }
        return 0;
    }
    return 0;
}

}  // namespace sfh
