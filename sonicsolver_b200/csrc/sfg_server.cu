// sfg_server.cu -- continuous-batching request loop over one sfg_batch
// (sfg_server_* in include/sonicsolver_b200.h).
//
// One worker thread owns the batch.  Each turn it
//   1. admits queued requests in FIFO order while a slot is free and the
//      request's state fits the HBM budget (a request larger than the whole
//      budget is rejected at submit);
//   2. runs one CUDA graph of batch steps for everything in flight;
//   3. reads every slot's status in one table read and retires finished
//      requests: result downloaded, slot and slab memory released.
// Requests that arrive while others run are admitted at the next graph
// boundary and step together with them; each request's grid keeps its own CFL
// step, clock and status, so a result does not depend on what it ran with.
#include "../../include/sonicsolver_b200.h"

#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace sfg {
void set_last_error(const char* msg);
int batch_check_numerics(sfg_batch b, const sfg_numerics_desc* n);
const char* law_problem(const sfg_boundary_law& law);
}

namespace {

int sfail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    sfg::set_last_error(buf);
    return code;
}

struct Request {
    int64_t id = 0;
    sfg_grid_desc grid{};
    sfg_numerics_desc num{};  // the request's own numerics (has_num)
    bool has_num = false;
    sfg_boundary_law laws[6] = {};  // [2 axis + end] of its SFG_BC_LAW ends (has_laws)
    bool has_laws = false;
    std::vector<double> input, output;
    double t_end = 0.0;
    int64_t max_steps = 0;
    size_t bytes = 0;
    int state = SFG_REQ_QUEUED;
    int slot = -1;
    bool cancel = false;
    double submit_s = 0.0, admit_s = -1.0, finish_s = -1.0;
    int64_t steps = 0;
    double time = 0.0;
    uint32_t flags = 0;
};

}  // namespace

struct sfg_server_s {
    sfg_batch batch = nullptr;
    int device = 0;
    int graph_steps = 16;
    int max_slots = 0;
    size_t budget = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int64_t> queue;
    std::map<int64_t, Request> reqs;
    std::vector<int64_t> slot_req;
    int64_t next_id = 1;
    int in_system = 0;  // queued + running
    bool stop = false;
    int worker_error = SFG_OK;
    std::string worker_msg;
    std::thread worker;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

void retire(sfg_server_s* s, Request& r, int state) {
    r.state = state;
    r.finish_s = s->now();
    r.input.clear();
    r.input.shrink_to_fit();
    s->in_system -= 1;
}

void worker_loop(sfg_server_s* s) {
    cudaSetDevice(s->device);
    std::vector<int> running;
    std::vector<double> times;
    std::vector<int64_t> steps;
    std::vector<uint32_t> flags;
    for (;;) {
        // 1. admission
        std::vector<Request*> admit;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            if (s->stop) break;
            size_t used = 0, budget = 0;
            int live = 0;
            sfg_batch_info(s->batch, &used, &budget, &live, nullptr);
            size_t free_bytes = budget - used;
            int free_slots = s->max_slots - live;
            while (!s->queue.empty() && free_slots > 0) {
                Request& r = s->reqs[s->queue.front()];
                if (r.cancel) {
                    s->queue.pop_front();
                    retire(s, r, SFG_REQ_CANCELLED);
                    continue;
                }
                if (r.bytes > free_bytes) break;  // FIFO: wait for memory to free up
                s->queue.pop_front();
                admit.push_back(&r);
                free_bytes -= r.bytes;
                free_slots -= 1;
            }
            if (admit.empty() && live == 0) {
                s->cv.wait_for(lock, std::chrono::milliseconds(2));
                continue;
            }
        }
        for (Request* r : admit) {
            int slot = -1;
            int rc = sfg_batch_add_laws(s->batch, &r->grid, r->has_num ? &r->num : nullptr,
                                        r->has_laws ? r->laws : nullptr, r->input.data(), r->t_end, r->max_steps,
                                        &slot);
            std::lock_guard<std::mutex> lock(s->mu);
            if (rc == SFG_ERR_BUDGET) {  // fragmentation: retry at the queue head
                s->queue.push_front(r->id);
                continue;
            }
            if (rc) {
                r->flags = 0xffffffffu;
                retire(s, *r, SFG_REQ_FAILED);
                continue;
            }
            r->slot = slot;
            r->state = SFG_REQ_RUNNING;
            r->admit_s = s->now();
            if ((int)s->slot_req.size() <= slot) s->slot_req.resize(slot + 1, 0);
            s->slot_req[slot] = r->id;
        }
        // 2. one graph of batch steps for everything in flight
        int active = 0;
        int rc = sfg_batch_step(s->batch, s->graph_steps, s->graph_steps, &active);
        if (rc) {
            std::lock_guard<std::mutex> lock(s->mu);
            s->worker_error = rc;
            s->worker_msg = sfg_last_error();
            break;
        }
        // 3. retire finished requests
        const int n = (int)s->slot_req.size();
        running.assign(n, -1);
        times.assign(n, 0.0);
        steps.assign(n, 0);
        flags.assign(n, 0);
        if (n > 0 && sfg_batch_snapshot(s->batch, n, running.data(), times.data(), steps.data(), flags.data())) break;
        for (int slot = 0; slot < n; ++slot) {
            if (running[slot] < 0) continue;
            int64_t id;
            bool cancel;
            {
                std::lock_guard<std::mutex> lock(s->mu);
                id = s->slot_req[slot];
                Request& r = s->reqs[id];
                r.steps = steps[slot];
                r.time = times[slot];
                r.flags = flags[slot];
                cancel = r.cancel;
            }
            if (running[slot] == 1 && !cancel) continue;
            Request* rp;
            {
                std::lock_guard<std::mutex> lock(s->mu);
                rp = &s->reqs[id];
            }
            if (!cancel) {
                rp->output.resize(rp->input.size());
                sfg_batch_download(s->batch, slot, rp->output.data());
            }
            sfg_batch_remove(s->batch, slot);
            std::lock_guard<std::mutex> lock(s->mu);
            s->slot_req[slot] = 0;
            rp->slot = -1;
            retire(s, *rp, cancel ? SFG_REQ_CANCELLED : (flags[slot] ? SFG_REQ_FAILED : SFG_REQ_DONE));
            s->cv.notify_all();
        }
    }
    std::lock_guard<std::mutex> lock(s->mu);
    s->cv.notify_all();
}

}  // namespace

extern "C" {

int sfg_server_create(const sfg_numerics_desc* numerics, size_t hbm_budget_bytes, int max_slots, int graph_steps,
                      sfg_server* out) {
    if (!out) return sfail(SFG_ERR_ARG, "null output handle");
    *out = nullptr;
    if (max_slots < 1) return sfail(SFG_ERR_ARG, "max_slots must be >= 1");
    sfg_batch b = nullptr;
    int rc = sfg_batch_create(numerics, hbm_budget_bytes, max_slots, nullptr, &b);
    if (rc) return rc;
    auto* s = new sfg_server_s;
    s->batch = b;
    s->max_slots = max_slots;
    s->graph_steps = graph_steps > 0 ? graph_steps : 16;
    s->budget = hbm_budget_bytes;
    cudaGetDevice(&s->device);
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return SFG_OK;
}

int sfg_server_destroy(sfg_server s) {
    if (!s) return SFG_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    sfg_batch_destroy(s->batch);
    delete s;
    return SFG_OK;
}

int sfg_server_submit(sfg_server s, const sfg_grid_desc* grid, const double* host_nodes_aos, double t_end,
                      int64_t max_steps, int64_t* request_id) {
    return sfg_server_submit_ex(s, grid, nullptr, host_nodes_aos, t_end, max_steps, request_id);
}

int sfg_server_submit_ex(sfg_server s, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                         const double* host_nodes_aos, double t_end, int64_t max_steps, int64_t* request_id) {
    return sfg_server_submit_laws(s, grid, numerics, nullptr, host_nodes_aos, t_end, max_steps, request_id);
}

int sfg_server_submit_laws(sfg_server s, const sfg_grid_desc* grid, const sfg_numerics_desc* numerics,
                           const sfg_boundary_law* laws, const double* host_nodes_aos, double t_end,
                           int64_t max_steps, int64_t* request_id) {
    if (!s || !grid || !host_nodes_aos || !request_id) return sfail(SFG_ERR_ARG, "null argument");
    if (numerics) {
        int rc = sfg::batch_check_numerics(s->batch, numerics);  // no device work
        if (rc) return rc;
    }
    bool law_ends = false;
    for (int a = 0; a < grid->dim && a < 3; ++a)
        for (int end = 0; end < 2; ++end)
            if ((end ? grid->bc_hi[a] : grid->bc_lo[a]) == SFG_BC_LAW) {
                law_ends = true;
                if (!laws) return sfail(SFG_ERR_ARG, "a grid with SFG_BC_LAW ends needs its laws");
                if (const char* why = sfg::law_problem(laws[2 * a + end]))
                    return sfail(SFG_ERR_ARG, "axis %d end %d: %s", a, end, why);
            }
    size_t bytes = 0;
    int rc = sfg_batch_instance_bytes(s->batch, grid, &bytes);  // validates the grid; no device work
    if (rc) return rc;
    if (bytes > s->budget) return sfail(SFG_ERR_BUDGET, "request needs %zu bytes, budget is %zu", bytes, s->budget);
    const size_t count = 5 * (size_t)grid->n[0] * grid->n[1] * grid->n[2];
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->worker_error) return sfail(s->worker_error, "server stopped: %s", s->worker_msg.c_str());
    Request r;
    r.id = s->next_id++;
    r.grid = *grid;
    if (numerics) {
        r.num = *numerics;
        r.has_num = true;
    }
    if (law_ends) {
        for (int k = 0; k < 2 * grid->dim && k < 6; ++k) r.laws[k] = laws[k];
        r.has_laws = true;
    }
    r.input.assign(host_nodes_aos, host_nodes_aos + count);
    r.t_end = t_end;
    r.max_steps = max_steps;
    r.bytes = bytes;
    r.submit_s = s->now();
    const int64_t id = r.id;
    s->reqs.emplace(id, std::move(r));
    s->queue.push_back(id);
    s->in_system += 1;
    s->cv.notify_all();
    *request_id = id;
    return SFG_OK;
}

int sfg_server_poll(sfg_server s, int64_t request_id, sfg_request_info* info) {
    if (!s || !info) return sfail(SFG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return sfail(SFG_ERR_NOT_FOUND, "unknown request %lld", (long long)request_id);
    const Request& r = it->second;
    info->submit_s = r.submit_s;
    info->admit_s = r.admit_s;
    info->finish_s = r.finish_s;
    info->steps = r.steps;
    info->time = r.time;
    info->flags = r.flags;
    info->state = r.state;
    return SFG_OK;
}

int sfg_server_fetch(sfg_server s, int64_t request_id, double* host_nodes_aos) {
    if (!s || !host_nodes_aos) return sfail(SFG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return sfail(SFG_ERR_NOT_FOUND, "unknown request %lld", (long long)request_id);
    Request& r = it->second;
    if (r.state == SFG_REQ_CANCELLED) return sfail(SFG_ERR_CANCELLED, "request %lld was cancelled", (long long)request_id);
    if (r.state == SFG_REQ_FAILED)
        return sfail(SFG_ERR_STATE, "request %lld failed (flags 0x%x)", (long long)request_id, r.flags);
    if (r.state != SFG_REQ_DONE) return sfail(SFG_ERR_ARG, "request %lld has not finished", (long long)request_id);
    std::copy(r.output.begin(), r.output.end(), host_nodes_aos);
    return SFG_OK;
}

int sfg_server_cancel(sfg_server s, int64_t request_id) {
    if (!s) return sfail(SFG_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return sfail(SFG_ERR_NOT_FOUND, "unknown request %lld", (long long)request_id);
    it->second.cancel = true;
    s->cv.notify_all();
    return SFG_OK;
}

int sfg_server_drain(sfg_server s, double timeout_s) {
    if (!s) return sfail(SFG_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lock(s->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
    while (s->in_system > 0 && !s->worker_error) {
        if (s->cv.wait_until(lock, deadline) == std::cv_status::timeout && s->in_system > 0)
            return sfail(SFG_ERR_TIMEOUT, "%d requests still in the system", s->in_system);
    }
    if (s->worker_error) return sfail(s->worker_error, "server stopped: %s", s->worker_msg.c_str());
    return SFG_OK;
}

double sfg_server_now(sfg_server s) { return s ? s->now() : 0.0; }

}  // extern "C"
