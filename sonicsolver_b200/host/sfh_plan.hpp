// sfh_plan.hpp -- the compiled step plan of the conservative explicit method
// and its executor.
//
// The operation ids are the reference's strings
// (src/core/system/SF_operationIds.h), and the plan has the shape the
// reference's ConservativeResidual method lowers to
// (src/solver/system/SF_builtinProviders.cpp:162-235): a preparation, then a
// time loop of dt, step begin, a stage loop of explicit stages, state commit
// and clock commit.  Operations are bound once, by (op id, provider), to
// closures; the executor refuses a plan with an unbound operation before it
// runs anything (PlanExecutor::validateBindings in the reference).
#pragma once

#include <functional>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace sfh {

namespace opid {
constexpr const char* FlowStepPrepare = "flow.step.prepare";
constexpr const char* FlowDtCompute = "flow.dt.compute";
constexpr const char* FlowStepBegin = "flow.step.begin";
constexpr const char* ExplicitStageExecute = "explicit.stage.execute";
constexpr const char* FlowStepCommit = "flow.step.commit";
constexpr const char* TimeCommit = "time.commit";
}  // namespace opid

enum class PlanKind { Sequence, TimeLoop, StageLoop, Op };

struct PlanNode {
    PlanKind kind = PlanKind::Sequence;
    std::string name;
    std::string op;        // PlanKind::Op
    std::string provider;  // PlanKind::Op
    int count = 0;         // PlanKind::StageLoop: number of stages
    std::vector<PlanNode> children;
};

// State the bound operations share while a plan runs.
struct StepContext {
    double t = 0.0;      // physical time at step start
    double dt = 0.0;     // step size of the current step
    int stage = 0;       // current explicit stage
    long long steps = 0;
    bool stop = false;   // set by an operation to end the time loop
    void* user = nullptr;
};

// An operation returns 0 on success, else a status code (the plan stops).
using OpFn = std::function<int(StepContext&)>;

class OperationTable {
public:
    // One binding per (op, provider); a second bind of the same pair throws.
    void bind(const std::string& op, const std::string& provider, OpFn fn);
    const OpFn* find(const std::string& op, const std::string& provider) const;
    // Throws std::runtime_error naming every Op node without a binding.
    void validate(const PlanNode& plan) const;

private:
    std::map<std::pair<std::string, std::string>, OpFn> table_;
};

// The conservative explicit plan for `stages` explicit stages, every
// operation owned by `provider`.
PlanNode conservative_explicit_plan(const std::string& provider, int stages);

// Indented text form of a plan.
std::string describe(const PlanNode& plan);

class PlanExecutor {
public:
    explicit PlanExecutor(const OperationTable& ops) : ops_(ops) {}
    // Validates, then runs; returns the first non-zero operation status.
    int run(const PlanNode& plan, StepContext& ctx) const;

private:
    int exec(const PlanNode& n, StepContext& ctx) const;
    const OperationTable& ops_;
};

}  // namespace sfh
