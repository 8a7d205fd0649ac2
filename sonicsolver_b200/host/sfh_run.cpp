// sfh_run.cpp -- `sfg_run`: runs a sonicSolver case directory on the GPU
// provider, through the same selection steps the reference's compiled plan
// takes:
//   1. read the case (sfh_case), build the grid and the initial state;
//   2. resolve the convection term in the TermCatalog and the plan's
//      operations in the ProviderCatalog (exactly one provider each);
//   3. build the conservative explicit plan, bind every operation id to a
//      C-ABI call of this library, validate the bindings;
//   4. run it, writing .vts output at the case's write times.
//
//   sfg_run --batch CASE_DIR... [--precision fp64|fp32flux] [--graph-steps K]
//           [--variant 1|2] [--dump-dir DIR] [--no-write] [--describe]
//   sfg_run CASE_DIR [--mode graph|plan] [--precision fp64|fp32flux]
//                    [--graph-steps K] [--dump FILE] [--dump-points FILE]
//                    [--dump-metrics FILE] [--checkpoint PREFIX] [--restart FILE]
//                    [--no-write] [--describe]
//
// --mode plan executes the plan operation by operation (one C-ABI call per
// operation, host synchronous).  --mode graph (default) lowers the time loop
// between two output times to one sfg_advance call: the device-resident
// clock runs the same dt, stage and commit sequence inside CUDA graphs.
// --describe stops after step 3 and touches no GPU.  A graded or curved
// block gets the generator's node coordinates and the reference Field's
// metrics (sfh_mesh.hpp); --dump-points writes the node coordinates (x, y, z
// per node, x fastest) and --dump-metrics the metrics handed to the provider
// (10 per point of the Field layout: the recipe's ghost layers on every
// axis), both as raw float64, also under --describe.
// --checkpoint PREFIX writes a restart file PREFIX_NNNN.json at every output
// time (NNNN: the output's number, as in the .vts names) and at the end of
// the run (sfh_checkpoint.hpp); --restart FILE starts from such a file: its
// state, time, step count and output clock replace the case's initial state
// and start time, and the run continues with the bits of the run that wrote
// it (sfg_restore).
// --batch runs several case directories together on the batched provider
// (sfg_batch_*): every case keeps its own recipe, gamma, CFL, maxDeltaT,
// boundary laws and output clipping, cases of one time recipe share a
// batch, and each ends at its own endTime with the steps and bits of its
// single-case graph run.  It writes each case's final state
// (<job>_final.vts in its output directory; with --dump-dir, <case name>.bin
// there) and prints one JSON line per case.  A case the batched kernels do
// not run (3-D, curvilinear, a start time, a flux other than Rusanov / Roe)
// is reported as unsupported and the others run.
// Exit codes: 0 done, 1 error, 2 usage, 3 case not supported by the provider.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "../../include/sonicsolver_b200.h"
#include "sfh_case.hpp"
#include "sfh_checkpoint.hpp"
#include "sfh_catalog.hpp"
#include "sfh_plan.hpp"
#include "sfh_vts.hpp"
#include "sfh_yaml.hpp"

namespace {

using namespace sfh;

struct Options {
    std::string dir, mode = "graph", dump, dump_points, dump_metrics, checkpoint, restart, dump_dir;
    std::vector<std::string> batch_dirs;
    bool batch = false;
    int variant = 0;
    int precision = SFG_PREC_FP64;
    int graph_steps = 32;
    bool write = true, describe_only = false;
};

int usage() {
    std::fprintf(stderr,
                 "usage: sfg_run CASE_DIR [--mode graph|plan] [--precision fp64|fp32flux] [--graph-steps K]\n"
                 "               [--dump FILE] [--dump-points FILE] [--dump-metrics FILE] [--checkpoint PREFIX]\n"
                 "               [--restart FILE] [--no-write] [--describe]\n"
                 "       sfg_run --batch CASE_DIR... [--precision fp64|fp32flux] [--graph-steps K] [--variant 1|2]\n"
                 "               [--dump-dir DIR] [--no-write] [--describe]\n");
    return 2;
}

int time_id(const std::string& token, int& stages) {
    if (token == "forwardEuler") return stages = 1, SFG_TIME_FORWARD_EULER;
    if (token == "SSPRK3") return stages = 3, SFG_TIME_SSPRK3;
    if (token == "classicalRK4") return stages = 4, SFG_TIME_CLASSICAL_RK4;
    throw Unsupported("time recipe '" + token + "': the provider implements forwardEuler, SSPRK3, classicalRK4");
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

// Everything the bound operations share.
struct Run {
    const CaseSpec* c = nullptr;
    const GridSetup* g = nullptr;
    sfg_solver s = nullptr;
    bool write = true;
    double next_out = 0.0;
    int outputs = 0;
    std::string out_dir;
    std::vector<double> host;
    VtsLayout vts;               // the .vts output layout of the case
    std::string checkpoint;      // restart-file prefix (empty: none)
    const Checkpoint* restart = nullptr;  // the restart file this run starts from
};

// Ghost layers of the provider's Field layout for a recipe (WENO3: 2,
// WENO5 / TENO5: 3, WENO7: 4; sfg_ghost_layers).
int recipe_ghosts(const std::string& convection) {
    if (convection.rfind("weno3", 0) == 0) return 2;
    if (convection.rfind("weno7", 0) == 0) return 4;
    return 3;
}

// The geometry of a graded or curved block for the provider: node
// coordinates (x, y, z per node) and the metrics in the provider's Field
// layout (ng_s ghosts on every axis, 10 per point), taken from the
// reference Field (the case's nGhost layers) at the same node offsets.  On
// an inactive axis the provider's one node plane is the block's first.
void block_geometry(const CaseSpec& c, const GridSetup& g, int ng_s, std::vector<double>& points,
                    std::vector<double>& all_points, std::vector<double>& metrics, double* residual,
                    double* tolerance) {
    bool active[3];
    for (int d = 0; d < 3; ++d) active[d] = d < g.grid.dim;
    const int ng_c = c.ghost_layers;
    if (ng_s > ng_c)
        throw Unsupported("mesh: the case's nGhost " + std::to_string(ng_c) + " is below the recipe's " +
                          std::to_string(ng_s) + " ghost layers");
    const FieldGeometry F = field_geometry(c.mesh, ng_c, active);
    *residual = F.identity_residual;
    *tolerance = F.identity_tolerance;
    if (!std::isfinite(F.identity_tolerance) || !(F.identity_tolerance > 0) ||
        F.identity_residual > F.identity_tolerance)
        throw Unsupported("mesh: the discrete metric identity is violated (max residual " +
                          std::to_string(F.identity_residual) + ", tolerance " +
                          std::to_string(F.identity_tolerance) + "), as the reference's audit reports");
    const int* n = g.nodes;
    points.resize(size_t(n[0]) * n[1] * n[2] * 3);
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const long long t = F.at(i + ng_c, j + ng_c, k + ng_c);
                double* p = &points[(((size_t)k * n[1] + j) * n[0] + i) * 3];
                p[0] = F.x[t];
                p[1] = F.y[t];
                p[2] = F.z[t];
            }
    // every node of the block (the written output covers unsolved axes too)
    const int nb[3] = {c.mesh.cells[0] + 1, c.mesh.cells[1] + 1, c.mesh.cells[2] + 1};
    all_points.resize(size_t(nb[0]) * nb[1] * nb[2] * 3);
    for (int k = 0; k < nb[2]; ++k)
        for (int j = 0; j < nb[1]; ++j)
            for (int i = 0; i < nb[0]; ++i) {
                const long long t = F.at(i + ng_c, j + ng_c, k + ng_c);
                double* p = &all_points[(((size_t)k * nb[1] + j) * nb[0] + i) * 3];
                p[0] = F.x[t];
                p[1] = F.y[t];
                p[2] = F.z[t];
            }
    const int e[3] = {n[0] + 2 * ng_s, n[1] + 2 * ng_s, n[2] + 2 * ng_s};
    metrics.resize(size_t(e[0]) * e[1] * e[2] * 10);
    for (int k = 0; k < e[2]; ++k)
        for (int j = 0; j < e[1]; ++j)
            for (int i = 0; i < e[0]; ++i) {
                const long long t = F.at(i - ng_s + ng_c, j - ng_s + ng_c, k - ng_s + ng_c);
                std::memcpy(&metrics[(((size_t)k * e[1] + j) * e[0] + i) * 10], &F.metrics[t * 10],
                            10 * sizeof(double));
            }
}

void write_doubles(const std::string& path, const std::vector<double>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
    if (!f) throw std::runtime_error("cannot write " + path);
}

bool at_or_past(double t, double mark) {
    const double sc = std::fabs(t) < 1.0 ? 1.0 : std::fabs(t);
    return t >= mark - 1e-11 * sc;
}

// A restart file of the current state (the host copy is current).
int write_restart(Run& r, const std::string& path) {
    Checkpoint c;
    for (int d = 0; d < 3; ++d) c.nodes[d] = r.g->nodes[d];
    if (int rc = sfg_time(r.s, &c.time, &c.steps)) return rc;
    c.next_output = r.c->write_interval > 0.0 ? r.next_out : std::numeric_limits<double>::infinity();
    c.outputs = r.outputs;
    c.q = r.host;
    if (!write_checkpoint(path, c)) {
        std::fprintf(stderr, "sfg_run: cannot write the restart file %s\n", path.c_str());
        return SFG_ERR_ARG;
    }
    std::printf("checkpoint t=%.17g %s\n", c.time, path.c_str());
    return 0;
}

std::string restart_name(const Run& r, int number) {
    char name[32];
    std::snprintf(name, sizeof name, "_%04d.json", number);
    return r.checkpoint + name;
}

int write_output(Run& r, double t) {
    if (!r.write && r.checkpoint.empty()) return 0;
    if (int rc = sfg_download(r.s, r.host.data(), SFG_LAYOUT_NODES)) return rc;
    if (!r.write) {
        ++r.outputs;
        return write_restart(r, restart_name(r, r.outputs - 1));
    }
    char name[64];
    std::snprintf(name, sizeof name, "_%04d.vts", r.outputs);
    const std::string path = r.out_dir + "/" + r.c->job_name + name;
    if (!write_vts(path, r.vts, r.host, r.c->gamma)) {
        std::fprintf(stderr, "sfg_run: cannot write %s\n", path.c_str());
        return SFG_ERR_ARG;
    }
    std::printf("write t=%.17g %s\n", t, path.c_str());
    ++r.outputs;
    return r.checkpoint.empty() ? 0 : write_restart(r, restart_name(r, r.outputs - 1));
}

// Clock end / output clipping of Time::Driver (the rule the device clock
// applies too): stop when the remaining time is round-off, else limit dt to
// the end and to the next output time.
bool remaining_limit(const Run& r, double t, double& limit) {
    const double eps = 2.220446049250313e-16;
    const double end = r.c->end_time;
    double sc = std::fmax(std::fabs(t), std::fabs(end));
    sc = sc < 1.0 ? 1.0 : sc;
    const double remaining = end - t;
    if (!(remaining > 64.0 * eps * sc)) return false;
    limit = remaining;
    if (r.c->write_interval > 0.0 && r.next_out - t < limit) limit = r.next_out - t;
    return true;
}

// Output schedule and the initial write, before the time loop.
int start_output(Run& r, double t) {
    if (r.restart) {  // the output clock of the run that wrote the restart file
        r.next_out = r.c->write_interval > 0.0 ? r.restart->next_output : 0.0;
        r.outputs = r.restart->outputs;
        return 0;
    }
    r.next_out = r.c->write_interval > 0.0 ? t + r.c->write_interval : 0.0;
    return r.c->write_initial ? write_output(r, t) : 0;
}

void bind_ops(OperationTable& ops, const std::string& provider, Run& r) {
    ops.bind(opid::FlowStepPrepare, provider, [&r](StepContext& ctx) {
        // the time loop ends before a step's fragment once t_end is reached
        double limit = 0.0;
        if (!remaining_limit(r, ctx.t, limit)) {
            ctx.stop = true;
            return 0;
        }
        // the physical boundary laws of law ends; ghosts of the other ends
        // are index maps inside the kernels
        return sfg_apply_boundary(r.s);
    });
    ops.bind(opid::FlowDtCompute, provider, [&r](StepContext& ctx) {
        double limit = 0.0;
        if (!remaining_limit(r, ctx.t, limit)) {
            ctx.stop = true;
            return 0;
        }
        return sfg_compute_dt(r.s, limit, &ctx.dt);
    });
    ops.bind(opid::FlowStepBegin, provider, [](StepContext&) { return 0; });  // stage 0 snapshots q0
    ops.bind(opid::ExplicitStageExecute, provider,
             [&r](StepContext& ctx) { return sfg_stage(r.s, ctx.stage, ctx.dt); });
    ops.bind(opid::FlowStepCommit, provider, [&r](StepContext&) {
        uint32_t bits = 0;
        if (int rc = sfg_status_word(r.s, &bits, 0)) return rc;
        return bits ? int(SFG_ERR_STATE) : 0;
    });
    ops.bind(opid::TimeCommit, provider, [&r](StepContext& ctx) {
        int64_t steps = 0;
        if (int rc = sfg_time(r.s, &ctx.t, &steps)) return rc;
        ctx.steps = steps;
        if (r.c->write_interval > 0.0 && at_or_past(ctx.t, r.next_out)) {
            r.next_out += r.c->write_interval;
            return write_output(r, ctx.t);
        }
        return 0;
    });
}

// The time loop between output times as one sfg_advance (device clock, CUDA
// graphs of `graph_steps` steps).
int run_graph(Run& r, int graph_steps, StepContext& ctx) {
    if (int rc = start_output(r, ctx.t)) return rc;
    for (;;) {
        double limit = 0.0;
        if (!remaining_limit(r, ctx.t, limit)) return 0;
        const double target =
            r.c->write_interval > 0.0 && r.next_out < r.c->end_time ? r.next_out : r.c->end_time;
        sfg_stats st{};
        if (int rc = sfg_advance(r.s, target, 0, 0.0, graph_steps, nullptr, 0, &st)) return rc;
        if (st.status_bits) return SFG_ERR_STATE;
        int64_t steps = 0;
        if (int rc = sfg_time(r.s, &ctx.t, &steps)) return rc;
        ctx.steps = steps;
        if (r.c->write_interval > 0.0 && at_or_past(ctx.t, r.next_out)) {
            r.next_out += r.c->write_interval;
            if (int rc = write_output(r, ctx.t)) return rc;
        }
    }
}

// Checks of the catalog and plan rules that need no case and no GPU.
int selftest() {
    int failed = 0;
    auto check = [&](bool ok, const char* what) {
        std::printf("%s %s\n", ok ? "ok" : "FAILED", what);
        failed += !ok;
    };
    int weno5 = -1;
    sfg_recipe_from_name("weno5Rusanov", &weno5);
    TermMatch m{"Momentum", "ConservativeResidual", "div", "rhoU", weno5, "weno5Rusanov"};
    TermCatalog gpu = TermCatalog::gpu();
    check(gpu.resolve(m).status == BindingStatus::Resolved, "supported recipe resolves to one provider");
    TermMatch sw = m;
    sw.recipe = -1;
    sw.recipe_token = "weno5StegerWarming";
    const ResolvedTerm r_sw = gpu.resolve(sw);
    check(r_sw.status == BindingStatus::Unsupported && r_sw.reason.find("no term provider") != std::string::npos,
          "recipe without a GPU kernel is Unsupported");
    TermMatch grad = m;
    grad.operator_name = "grad";
    check(gpu.resolve(grad).status == BindingStatus::Unsupported, "other operators are not matched");
    check(gpu.resolve(m, "convection.other").status == BindingStatus::Unsupported, "binding to another id");
    TermCatalog two = TermCatalog::gpu();
    two.add({"convection.second", [](const TermMatch& t) { return t.operator_name == "div"; }, "test"});
    const ResolvedTerm amb = two.resolve(m);
    check(amb.status == BindingStatus::Invalid &&
              amb.reason.find("convection.conservativeFlux, convection.second") != std::string::npos,
          "two matching providers are Invalid (ambiguous, listed in id order)");
    check(two.resolve(m, "convection.second").status == BindingStatus::Resolved, "a binding selects one of them");
    bool threw = false;
    try {
        two.add({"convection.second", [](const TermMatch&) { return false; }, "test"});
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    check(threw, "duplicate term provider id is refused");
    const ProviderCatalog pc = ProviderCatalog::gpu();
    const Operation op{opid::ExplicitStageExecute, {Capability::ConservativeExplicit}};
    check(pc.resolve(op, "flow.conservative").status == BindingStatus::Resolved, "runtime provider resolves");
    check(pc.resolve(op, "flow.pressure").reason.find("not registered") != std::string::npos,
          "unknown runtime provider");
    check(pc.resolve({opid::TimeCommit, {Capability::TemporalSynchronization}}, "flow.conservative")
                  .reason.find("lacks a capability") != std::string::npos,
          "missing capability");
    check(pc.resolve(op, "").status == BindingStatus::Unsupported, "no provider selected");
    const PlanNode plan = conservative_explicit_plan("flow.conservative", 3);
    OperationTable ops;
    ops.bind(opid::FlowStepPrepare, "flow.conservative", [](StepContext&) { return 0; });
    bool unbound = false;
    try {
        ops.validate(plan);
    } catch (const std::runtime_error& e) {
        unbound = std::string(e.what()).find("flow.dt.compute @ flow.conservative") != std::string::npos;
    }
    check(unbound, "a plan with unbound operations is refused before it runs");
    // a counting run of the plan: 2 steps of 3 stages
    OperationTable cnt;
    int stages = 0, dts = 0, commits = 0;
    const std::string p = "flow.conservative";
    cnt.bind(opid::FlowStepPrepare, p, [](StepContext&) { return 0; });
    cnt.bind(opid::FlowDtCompute, p, [&](StepContext& c) {
        c.stop = ++dts > 2;
        return 0;
    });
    cnt.bind(opid::FlowStepBegin, p, [](StepContext&) { return 0; });
    cnt.bind(opid::ExplicitStageExecute, p, [&](StepContext& c) { return c.stage == stages++ % 3 ? 0 : 1; });
    cnt.bind(opid::FlowStepCommit, p, [](StepContext&) { return 0; });
    cnt.bind(opid::TimeCommit, p, [&](StepContext&) { return ++commits, 0; });
    StepContext ctx;
    const int rc = PlanExecutor(cnt).run(plan, ctx);
    check(rc == 0 && stages == 6 && commits == 2 && dts == 3, "plan runs stages 0..2 per step until dt stops it");
    threw = false;
    try {
        cnt.bind(opid::TimeCommit, p, [](StepContext&) { return 0; });
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    check(threw, "an operation is bound once");
    // restart files: a written state reads back to the last bit, with its
    // clock; a damaged one is refused
    {
        Checkpoint ck;
        ck.nodes[0] = 7;
        ck.nodes[1] = 3;
        ck.time = 0.1 + 0.2;
        ck.steps = 42;
        ck.next_output = 1.0 / 3.0;
        ck.outputs = 5;
        for (int i = 0; i < 7 * 3 * 5; ++i) ck.q.push_back(std::ldexp(1.0 + i / 97.0, (i % 9) - 4) * (i % 2 ? -1 : 1));
        char path[] = "/tmp/sfg_selftest_ckXXXXXX";
        const int fd = mkstemp(path);
        bool ok = fd >= 0 && write_checkpoint(path, ck);
        if (fd >= 0) close(fd);
        if (ok) {
            const Checkpoint back = read_checkpoint(path);
            ok = back.q == ck.q && back.time == ck.time && back.steps == 42 && back.next_output == ck.next_output &&
                 back.outputs == 5 && back.nodes[0] == 7 && back.nodes[1] == 3 && back.nodes[2] == 1;
        }
        check(ok, "a restart file reads back bit for bit with its clock");
        bool refused = false;
        if (FILE* f = std::fopen(path, "w")) {
            std::fputs("{\"formatVersion\": 1, \"fields\": {}, \"nodes\": [1, 1, 1], \"time\": 0, \"steps\": 0, "
                       "\"outputs\": 0}", f);
            std::fclose(f);
            try {
                read_checkpoint(path);
            } catch (const std::runtime_error&) {
                refused = true;
            }
        }
        std::remove(path);
        check(refused, "a restart file without its fields is refused");
    }
    std::printf("%s\n", failed ? "selftest FAILED" : "selftest passed");
    return failed ? 1 : 0;
}

}  // namespace

// ---- several case directories on the batched provider

struct BatchCase {
    std::string dir;
    CaseSpec c;
    GridSetup g;
    int recipe = -1, tid = -1, slot = -1;
};

// Why a case cannot run batched (empty: it can).
std::string batch_obstacle(const BatchCase& b) {
    if (b.g.grid.dim > 2) return "3-D grids run on single-grid solvers only";
    if (b.c.curvilinear) return "graded or curved blocks run on single-grid solvers only";
    if (b.c.start_time != 0.0) return "a start time other than 0 (restart cases run on single-grid solvers)";
    const std::string& r = b.c.convection;
    const bool flux_ok = r.size() > 5 && (r.compare(r.size() - 7, 7, "Rusanov") == 0 || r.compare(r.size() - 3, 3, "Roe") == 0);
    if (!flux_ok) return "convection '" + r + "': the batched kernels provide Rusanov and Roe faces";
    return {};
}

int run_batch(const Options& o) {
    std::vector<BatchCase> cases;
    int unsupported = 0;
    for (const auto& dir : o.batch_dirs) {
        BatchCase b;
        b.dir = dir;
        try {
            b.c = load_case(dir);
            b.g = build_grid(b.c);
            int stages = 0;
            b.tid = time_id(b.c.time_recipe, stages);
            if (sfg_recipe_from_name(b.c.convection.c_str(), &b.recipe) != SFG_OK)
                throw Unsupported("convection '" + b.c.convection + "' has no term provider");
            const std::string why = batch_obstacle(b);
            if (!why.empty()) throw Unsupported(why);
        } catch (const Unsupported& e) {
            std::fprintf(stderr, "sfg_run: unsupported: %s: %s\n", dir.c_str(), e.what());
            ++unsupported;
            continue;
        } catch (const std::exception& e) {
            std::fprintf(stderr, "sfg_run: error: %s: %s\n", dir.c_str(), e.what());
            return 1;
        }
        cases.push_back(std::move(b));
    }
    // one batch per time recipe (a batch runs one time recipe and precision)
    std::map<int, std::vector<size_t>> groups;
    for (size_t k = 0; k < cases.size(); ++k) groups[cases[k].tid].push_back(k);
    for (const auto& kv : groups) {
        std::printf("batch time=%s cases=%zu:", cases[kv.second[0]].c.time_recipe.c_str(), kv.second.size());
        for (size_t k : kv.second) std::printf(" %s(%s)", cases[k].c.name.c_str(), cases[k].c.convection.c_str());
        std::printf("\n");
    }
    if (o.describe_only) return unsupported ? 3 : 0;
    int rc_all = 0;
    std::vector<std::string> results(cases.size());  // JSON lines, printed in the order given
    for (const auto& kv : groups) {
        const BatchCase& first = cases[kv.second[0]];
        sfg_numerics_desc nd{first.recipe, kv.first, o.precision, first.c.gamma, first.c.cfl, first.c.max_dt};
        // the slab: every grid's bytes (asked of a probe batch), plus room
        size_t need = 0;
        {
            sfg_batch probe = nullptr;
            if (sfg_batch_create(&nd, 1u << 20, 1, nullptr, &probe) != SFG_OK) {
                std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
                return 1;
            }
            for (size_t k : kv.second) {
                size_t bytes = 0;
                if (sfg_batch_instance_bytes(probe, &cases[k].g.grid, &bytes) != SFG_OK) {
                    std::fprintf(stderr, "sfg_run: %s: %s\n", cases[k].dir.c_str(), sfg_last_error());
                    sfg_batch_destroy(probe);
                    return 1;
                }
                need += bytes + 4096;
            }
            sfg_batch_destroy(probe);
        }
        sfg_batch b = nullptr;
        if (sfg_batch_create(&nd, need + (64u << 20), int(kv.second.size()), nullptr, &b) != SFG_OK) {
            std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
            return 1;
        }
        if (o.variant && sfg_batch_set_variant(b, o.variant) != SFG_OK) {
            std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
            sfg_batch_destroy(b);
            return 1;
        }
        const auto w0 = std::chrono::steady_clock::now();
        for (size_t k : kv.second) {
            BatchCase& bc = cases[k];
            sfg_numerics_desc own{bc.recipe, bc.tid, o.precision, bc.c.gamma, bc.c.cfl, bc.c.max_dt};
            if (sfg_batch_add_laws(b, &bc.g.grid, &own, bc.g.laws, bc.g.q.data(), bc.c.end_time, 0, &bc.slot) != SFG_OK ||
                sfg_batch_set_write_interval(b, bc.slot, bc.c.write_interval) != SFG_OK) {
                std::fprintf(stderr, "sfg_run: %s: %s\n", bc.dir.c_str(), sfg_last_error());
                sfg_batch_destroy(b);
                return 1;
            }
        }
        int active = 0;
        if (sfg_batch_step(b, std::numeric_limits<int>::max(), o.graph_steps, &active) != SFG_OK) {
            std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
            sfg_batch_destroy(b);
            return 1;
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
        for (size_t k : kv.second) {
            BatchCase& bc = cases[k];
            double t = 0;
            int64_t steps = 0;
            int running = 0;
            uint32_t bits = 0;
            int rc = sfg_batch_status(b, bc.slot, &t, &steps, &running, &bits);
            std::vector<double> q(bc.g.q.size());
            if (!rc) rc = sfg_batch_download(b, bc.slot, q.data());
            if (!rc && bits) rc = SFG_ERR_STATE;
            if (!rc && o.write) {
                const std::string out_dir = bc.c.dir + "/" + bc.c.output_dir;
                mkdir(out_dir.c_str(), 0755);
                const std::string path = out_dir + "/" + bc.c.job_name + "_final.vts";
                if (!write_vts(path, vts_layout(bc.c, bc.g, {}), q, bc.c.gamma)) rc = SFG_ERR_ARG;
                else std::printf("write t=%.17g %s\n", t, path.c_str());
            }
            if (!rc && !o.dump_dir.empty()) {
                std::ofstream f(o.dump_dir + "/" + bc.c.name + ".bin", std::ios::binary);
                f.write(reinterpret_cast<const char*>(q.data()), std::streamsize(q.size() * sizeof(double)));
                if (!f) rc = SFG_ERR_ARG;
            }
            if (rc) rc_all = 1;
            char line[1024];
            std::snprintf(line, sizeof line,
                          "{\"case\": \"%s\", \"mode\": \"batch\", \"recipe\": \"%s\", \"time_recipe\": \"%s\", "
                          "\"dim\": %d, \"nodes\": [%d, %d, %d], \"steps\": %lld, \"time\": %.17g, \"status\": %d, "
                          "\"status_bits\": %u, \"batch_wall_s\": %.6f}",
                          json_escape(bc.c.name).c_str(), bc.c.convection.c_str(), bc.c.time_recipe.c_str(),
                          bc.g.grid.dim, bc.g.nodes[0], bc.g.nodes[1], bc.g.nodes[2], (long long)steps, t, rc, bits,
                          wall);
            results[k] = line;
        }
        sfg_batch_destroy(b);
    }
    for (const auto& line : results) std::printf("%s\n", line.c_str());
    if (rc_all) return 1;
    return unsupported ? 3 : 0;
}

int main(int argc, char** argv) {
    if (argc == 2 && std::strcmp(argv[1], "--selftest") == 0) return selftest();
    Options o;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](void) -> std::string { return i + 1 < argc ? argv[++i] : std::string(); };
        if (a == "--mode") o.mode = next();
        else if (a == "--precision") {
            const std::string p = next();
            if (p == "fp64") o.precision = SFG_PREC_FP64;
            else if (p == "fp32flux") o.precision = SFG_PREC_FP32_FLUX;
            else return usage();
        } else if (a == "--graph-steps") o.graph_steps = std::atoi(next().c_str());
        else if (a == "--dump") o.dump = next();
        else if (a == "--dump-points") o.dump_points = next();
        else if (a == "--dump-metrics") o.dump_metrics = next();
        else if (a == "--checkpoint") o.checkpoint = next();
        else if (a == "--restart") o.restart = next();
        else if (a == "--no-write") o.write = false;
        else if (a == "--describe") o.describe_only = true;
        else if (a == "--batch") o.batch = true;
        else if (a == "--dump-dir") o.dump_dir = next();
        else if (a == "--variant") o.variant = std::atoi(next().c_str());
        else if (!a.empty() && a[0] == '-') return usage();
        else if (o.batch) o.batch_dirs.push_back(a);
        else o.dir = a;
    }
    if (o.batch) return o.batch_dirs.empty() ? usage() : run_batch(o);
    if (o.dir.empty() || (o.mode != "graph" && o.mode != "plan")) return usage();
    try {
        const CaseSpec c = load_case(o.dir);
        const GridSetup g = build_grid(c);
        int stages = 0;
        const int tid = time_id(c.time_recipe, stages);
        // ---- provider selection
        TermMatch term{"Momentum", "ConservativeResidual", "div", "rhoU", -1, c.convection};
        int recipe = -1;
        if (sfg_recipe_from_name(c.convection.c_str(), &recipe) == SFG_OK) term.recipe = recipe;
        const ResolvedTerm rt = TermCatalog::gpu().resolve(term);
        if (rt.status != BindingStatus::Resolved)
            throw Unsupported(std::string(to_string(rt.status)) + ": " + rt.reason);
        const std::string provider = "flow.conservative";
        const ProviderCatalog pc = ProviderCatalog::gpu();
        for (const char* op : {opid::FlowStepPrepare, opid::FlowDtCompute, opid::FlowStepBegin,
                               opid::ExplicitStageExecute, opid::FlowStepCommit, opid::TimeCommit}) {
            const ResolvedOperation ro = pc.resolve({op, {Capability::ConservativeExplicit}}, provider);
            if (ro.status != BindingStatus::Resolved)
                throw Unsupported(std::string(to_string(ro.status)) + ": " + ro.reason);
        }
        const PlanNode plan = conservative_explicit_plan(provider, stages);
        std::printf("term %s -> %s (owner %s, recipe %s)\nplan:\n%s", "div", rt.id.c_str(), rt.owner.c_str(),
                    c.convection.c_str(), describe(plan).c_str());
        std::printf("grid dim=%d nodes=%d,%d,%d h=%.17g,%.17g,%.17g bc=%d%d/%d%d/%d%d\n", g.grid.dim, g.nodes[0],
                    g.nodes[1], g.nodes[2], g.grid.h[0], g.grid.h[1], g.grid.h[2], g.grid.bc_lo[0], g.grid.bc_hi[0],
                    g.grid.bc_lo[1], g.grid.bc_hi[1], g.grid.bc_lo[2], g.grid.bc_hi[2]);
        for (int a = 0; a < 3; ++a)
            for (int e = 0; e < 2; ++e) {
                if ((e ? g.grid.bc_hi[a] : g.grid.bc_lo[a]) != SFG_BC_LAW) continue;
                const sfg_boundary_law& L = g.laws[2 * a + e];
                auto law_name = [](int k) {
                    return k == SFG_LAW_FIXED_VALUE ? "fixedValue" : k == SFG_LAW_SYMMETRY ? "symmetry" : "zeroGradient";
                };
                std::printf("law %c%s rho=%s(%.17g) U=%s(%.17g,%.17g,%.17g) p=%s(%.17g)\n", "xyz"[a], e ? "hi" : "lo",
                            law_name(L.rho), L.rho_value, law_name(L.velocity), L.velocity_value[0],
                            L.velocity_value[1], L.velocity_value[2], law_name(L.pressure), L.pressure_value);
            }
        // a graded or curved block: the generator's node coordinates and metrics
        std::vector<double> points, all_points, metrics;
        if (c.curvilinear) {
            double res = 0, tol = 0;
            block_geometry(c, g, recipe_ghosts(c.convection), points, all_points, metrics, &res, &tol);
            std::printf("mesh curvilinear (%s): metric identity residual %.3g, tolerance %.3g\n",
                        c.mesh.edges.empty() ? "trilinear, graded" : "transfinite, arc edges", res, tol);
            if (!o.dump_points.empty()) write_doubles(o.dump_points, points);
            if (!o.dump_metrics.empty()) write_doubles(o.dump_metrics, metrics);
        }
        if (o.describe_only) {
            OperationTable ops;
            Run dummy;
            bind_ops(ops, provider, dummy);
            ops.validate(plan);
            std::printf("bindings valid\n");
            return 0;
        }
        // ---- provider instance and bindings
        sfg_numerics_desc nd{recipe, tid, o.precision, c.gamma, c.cfl, c.max_dt};
        Run r;
        r.c = &c;
        r.g = &g;
        r.write = o.write;
        r.host.resize(g.q.size());
        r.vts = vts_layout(c, g, all_points);
        r.out_dir = c.dir + "/" + c.output_dir;
        if (o.write) mkdir(r.out_dir.c_str(), 0755);
        if (sfg_create(&g.grid, &nd, nullptr, &r.s) != SFG_OK) {
            std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
            return 1;
        }
        for (int a = 0; a < g.grid.dim; ++a)
            for (int e = 0; e < 2; ++e)
                if ((e ? g.grid.bc_hi[a] : g.grid.bc_lo[a]) == SFG_BC_LAW &&
                    sfg_set_boundary_law(r.s, a, e, &g.laws[2 * a + e]) != SFG_OK) {
                    std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
                    sfg_destroy(r.s);
                    return 1;
                }
        if (c.curvilinear && sfg_set_metrics(r.s, metrics.data(), SFG_LAYOUT_FIELD) != SFG_OK) {
            std::fprintf(stderr, "sfg_run: %s\n", sfg_last_error());
            sfg_destroy(r.s);
            return 1;
        }
        r.checkpoint = o.checkpoint;
        Checkpoint restart;
        StepContext ctx;
        ctx.t = c.start_time;
        int rc = 0;
        if (!o.restart.empty()) {
            // a restart file replaces the initial state and the start time
            // (the case's ghost layers of unconditioned ends are re-made from
            // the restart state, as the reference's restart does)
            restart = read_checkpoint(o.restart);
            for (int d = 0; d < 3; ++d)
                if (restart.nodes[d] != g.nodes[d]) {
                    std::fprintf(stderr, "sfg_run: %s holds %d x %d x %d nodes, the case %d x %d x %d\n",
                                 o.restart.c_str(), restart.nodes[0], restart.nodes[1], restart.nodes[2], g.nodes[0],
                                 g.nodes[1], g.nodes[2]);
                    sfg_destroy(r.s);
                    return 1;
                }
            r.restart = &restart;
            rc = sfg_restore(r.s, restart.q.data(), SFG_LAYOUT_NODES, restart.time, restart.steps);
            ctx.t = restart.time;
            ctx.steps = restart.steps;
            std::printf("restart t=%.17g steps=%lld from %s\n", restart.time, (long long)restart.steps,
                        o.restart.c_str());
        } else {
            rc = sfg_upload(r.s, g.q.data(), SFG_LAYOUT_NODES, c.start_time);
        }
        const auto w0 = std::chrono::steady_clock::now();
        if (!rc) {
            if (o.mode == "plan") {
                OperationTable ops;
                bind_ops(ops, provider, r);
                rc = start_output(r, ctx.t);
                if (!rc) rc = PlanExecutor(ops).run(plan, ctx);
            } else {
                rc = run_graph(r, o.graph_steps, ctx);
            }
        }
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
        uint32_t bits = 0;
        double totals[5] = {0, 0, 0, 0, 0};
        if (!rc) rc = sfg_status_word(r.s, &bits, 0);
        if (!rc) rc = sfg_conserved_totals(r.s, totals);
        if (!rc && !o.checkpoint.empty()) {
            rc = sfg_download(r.s, r.host.data(), SFG_LAYOUT_NODES);
            if (!rc) rc = write_restart(r, o.checkpoint + "_end.json");
        }
        if (!rc && !o.dump.empty()) {
            rc = sfg_download(r.s, r.host.data(), SFG_LAYOUT_NODES);
            std::ofstream f(o.dump, std::ios::binary);
            f.write(reinterpret_cast<const char*>(r.host.data()), std::streamsize(r.host.size() * sizeof(double)));
        }
        if (rc) std::fprintf(stderr, "sfg_run: status %d: %s\n", rc, sfg_last_error());
        std::printf("{\"case\": \"%s\", \"mode\": \"%s\", \"term_provider\": \"%s\", \"runtime_provider\": \"%s\", "
                    "\"recipe\": \"%s\", \"time_recipe\": \"%s\", \"dim\": %d, \"nodes\": [%d, %d, %d], "
                    "\"steps\": %lld, \"time\": %.17g, \"status\": %d, \"status_bits\": %u, "
                    "\"totals\": [%.17g, %.17g, %.17g, %.17g, %.17g], \"outputs\": %d, \"wall_s\": %.6f}\n",
                    json_escape(c.name).c_str(), o.mode.c_str(), rt.id.c_str(), provider.c_str(),
                    c.convection.c_str(), c.time_recipe.c_str(), g.grid.dim, g.nodes[0], g.nodes[1], g.nodes[2],
                    (long long)ctx.steps, ctx.t, rc, bits, totals[0], totals[1], totals[2], totals[3], totals[4],
                    r.outputs, wall);
        sfg_destroy(r.s);
        return rc ? 1 : 0;
    } catch (const Unsupported& e) {
        std::fprintf(stderr, "sfg_run: unsupported: %s\n", e.what());
        return 3;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "sfg_run: error: %s\n", e.what());
        return 1;
    }
}
