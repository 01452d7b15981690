// wenofv_server.cu -- continuous batching of solve requests on one GPU.
//
// A background engine thread owns one slot Engine whose slot memory is a single arena
// allocated when the server starts (the HBM budget, or what the device has free), so that
// admitting a request calls no cudaMalloc.  Each round it
//   1. admits queued requests in arrival order while a slot is free and the request's device
//      state (three FP64 state buffers and the grid metric) fits in the arena: upload, then
//      one CFL pass per launch group over the new slots only,
//   2. runs a chunk of RK step pairs as one captured graph in which every launch group (one
//      per template key: form, equation, reconstruction, scheme, flux) is its own branch, so
//      groups of different keys run side by side; a persistent launch per RK stage advances
//      every running request of its group, and a request that reaches its end time or step
//      count stops inside the kernel (its work items are skipped) while the others go on.
//      The chunk length follows the measured time per step pair (about CHUNK_TARGET_MS per
//      round), not the shortest remaining request,
//   3. reads the device loop state back, copies finished requests' results to host memory,
//      frees their slots and arena blocks.
// Work lists are rewritten in place in device buffers, so a captured graph stays valid while
// requests come and go; it is re-captured only when a new template key appears or a list
// outgrows its buffer.  Requests arriving while others run join at the next round boundary,
// so their work shares launches with the requests already on the GPU.  submit/poll only touch
// the queue and the result table under a mutex; they never call CUDA.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "wenofv_engine.h"

using namespace wenofv;

namespace {

struct Request {
    int64_t id = 0;
    wenofv_config cfg{};
    wenofv_eq_params eq{};
    std::vector<double> U; // initial state, then the result
    double t_end = 0;
    int64_t max_steps = 0;
    size_t bytes = 0;
    int slot = -1;
    wenofv_request_info info{};
    bool done = false;
};

double now_s(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace

struct wenofv_server {
    Engine eng;
    int device = 0;
    size_t budget = 0, resident = 0;
    int max_slots = 0;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> queue;
    std::map<int64_t, Request *> all;
    std::vector<Request *> active; // by slot
    int64_t next_id = 1, admitted = 0, completed = 0;
    static constexpr double CHUNK_TARGET_MS = 10.0;
    static constexpr int CHUNK_MAX_PAIRS = 32;
    double ms_per_pair = 1.0; // running estimate of one step pair of the current mix
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool stop = false;
    int fatal = 0;
    std::thread th;

    void loop();
    int round();
};

int wenofv_server::round()
{
    // 1. admission (arrival order; a request that does not fit waits, and blocks those behind it)
    std::vector<Request *> admit;
    {
        std::lock_guard<std::mutex> lk(mu);
        int free_slots = 0;
        for (Request *r : active) free_slots += r == nullptr;
        size_t arena_free = eng.arena_free_bytes();
        while (!queue.empty() && free_slots > 0 && resident + queue.front()->bytes <= budget &&
               (queue.front()->bytes + 255) / 256 * 256 <= arena_free) {
            Request *r = queue.front();
            queue.pop_front();
            resident += r->bytes;
            arena_free -= (r->bytes + 255) / 256 * 256;
            admit.push_back(r);
            free_slots--;
        }
    }
    std::vector<int> new_slots;
    std::vector<double> new_tend;
    std::vector<int64_t> new_max;
    std::vector<Request *> started;
    for (Request *r : admit) {
        int slot = -1;
        int rc = eng.add(r->cfg, r->eq, &slot);
        if (!rc) rc = eng.upload(slot, r->U.data(), WENOFV_LAYOUT_SOA);
        std::lock_guard<std::mutex> lk(mu);
        r->info.t_admit = now_s(t0);
        admitted++;
        if (rc) { // e.g. a fragmented arena: the request fails alone, the others go on
            if (slot >= 0) eng.remove(slot);
            resident -= r->bytes;
            r->info.status = rc;
            r->info.t_done = now_s(t0);
            r->done = true;
            completed++;
            cv.notify_all();
            continue;
        }
        r->slot = slot;
        active[slot] = r;
        new_slots.push_back(slot);
        new_tend.push_back(r->t_end);
        new_max.push_back(r->max_steps);
    }
    if (!new_slots.empty()) {
        const int rc = eng.start_many(new_slots, new_tend, new_max);
        if (rc) return rc;
    }
    int running = 0;
    for (Request *r : active) running += r != nullptr;
    if (running == 0) return 0;

    // 2. a chunk of step pairs for every running request, as one captured graph; its length
    //    follows the measured time per pair so that a round takes about CHUNK_TARGET_MS
    int K = 1;
    while (K < CHUNK_MAX_PAIRS && K * ms_per_pair < CHUNK_TARGET_MS / 2) K *= 2;
    cudaEventRecord(ev0, eng.stream);
    int rc = eng.run_graph_pairs(K);
    if (rc) return rc;
    cudaEventRecord(ev1, eng.stream);
    rc = eng.refresh();
    if (rc) return rc;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess && ms > 0) ms_per_pair = 0.5 * ms_per_pair + 0.5 * ms / K;
    (void)cudaGetLastError();

    // 3. collect finished requests
    for (size_t k = 0; k < active.size(); k++) {
        Request *r = active[k];
        if (!r) continue;
        const InstState s = eng.slot_state(r->slot);
        if (!s.done) continue;
        int st = eng.download(r->slot, r->U.data(), WENOFV_LAYOUT_SOA);
        if (!st && (s.flags & (WENOFV_FLAG_NAN_DT | WENOFV_FLAG_BAD_THETA | WENOFV_FLAG_NAN_FLUX | WENOFV_FLAG_NAN_STATE | WENOFV_FLAG_BOUNDS)))
            st = WENOFV_ENUMERIC;
        eng.remove(r->slot);
        std::lock_guard<std::mutex> lk(mu);
        r->info.steps = s.nsteps;
        r->info.flags = s.flags;
        r->info.status = st;
        r->info.t_done = now_s(t0);
        r->done = true;
        resident -= r->bytes;
        active[k] = nullptr;
        completed++;
        cv.notify_all();
    }
    return 0;
}

void wenofv_server::loop()
{
    cudaSetDevice(device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu);
            bool idle = queue.empty();
            for (Request *r : active) idle = idle && r == nullptr;
            if (stop) break;
            if (idle) cv.wait_for(lk, std::chrono::milliseconds(1));
            if (stop) break;
        }
        const int rc = round();
        if (rc) {
            std::lock_guard<std::mutex> lk(mu);
            fatal = rc;
            for (Request *r : active)
                if (r) { r->info.status = rc; r->done = true; }
            for (Request *r : queue) { r->info.status = rc; r->done = true; }
            queue.clear();
            cv.notify_all();
            break;
        }
    }
}

extern "C" {

int wenofv_server_create(int device, size_t hbm_budget_bytes, int max_slots, wenofv_server **out)
{
    if (!out || max_slots < 1 || hbm_budget_bytes == 0) { set_error("bad arguments"); return WENOFV_EINVAL; }
    *out = nullptr;
    wenofv_server *s = new (std::nothrow) wenofv_server;
    if (!s) { set_error("host allocation failed"); return WENOFV_ENOMEM; }
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_slots = max_slots;
    s->t0 = std::chrono::steady_clock::now();
    s->eng.slot_mode = true;
    // the slot arena: the budget, or what the device has free less a margin for the
    // engine's own buffers
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        (void)cudaGetLastError();
        delete s;
        set_error("no CUDA device %d", device);
        return WENOFV_EINVAL;
    }
    const size_t margin = (size_t)1 << 30;
    const size_t arena = std::min(hbm_budget_bytes, free_b > 2 * margin ? free_b - margin : free_b / 2);
    s->budget = arena;
    int rc = s->eng.init_slots(max_slots, device, 2, arena);
    if (!rc && cudaEventCreate(&s->ev0) != cudaSuccess) rc = WENOFV_ECUDA;
    if (!rc && cudaEventCreate(&s->ev1) != cudaSuccess) rc = WENOFV_ECUDA;
    if (rc) { delete s; return rc; }
    s->active.assign(max_slots, nullptr);
    s->th = std::thread([s] { s->loop(); });
    *out = s;
    return WENOFV_OK;
}

void wenofv_server_destroy(wenofv_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    for (auto &kv : s->all) delete kv.second;
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    delete s;
}

int wenofv_server_submit(wenofv_server *s, const wenofv_config *cfg, const wenofv_eq_params *eq, const double *U0,
                         double t_end, int64_t max_steps, int64_t *request_id)
{
    if (!s || !cfg || !eq || !U0 || !request_id) { set_error("null argument"); return WENOFV_EINVAL; }
    int rc = validate(cfg, eq);
    if (rc) return rc;
    if (cfg->rk_method != 2 || cfg->device != s->device) { set_error("the server runs SSP-RK3 on its own device"); return WENOFV_ENOTSUP; }
    if (cfg->bc == WENOFV_BC_NEUMANN2) { set_error("the server takes no NEUMANN2 requests (they need a ghost frame)"); return WENOFV_ENOTSUP; }
    if (!(t_end > 0)) { set_error("t_end must be positive"); return WENOFV_EINVAL; }
    const size_t bytes = Engine::bytes_needed(*cfg, *eq);
    if ((bytes + 255) / 256 * 256 > s->budget) { set_error("request needs %zu bytes, over the HBM budget", bytes); return WENOFV_ENOMEM; }
    Request *r = new (std::nothrow) Request;
    if (!r) { set_error("host allocation failed"); return WENOFV_ENOMEM; }
    const size_t n = (size_t)nvar_of(eq->eq_kind) * cfg->nx * cfg->ny;
    try {
        r->U.assign(U0, U0 + n);
    } catch (...) {
        delete r;
        set_error("host allocation failed");
        return WENOFV_ENOMEM;
    }
    r->cfg = *cfg;
    r->eq = *eq;
    r->t_end = t_end;
    r->max_steps = max_steps > 0 ? max_steps : 0;
    r->bytes = bytes;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->fatal) { delete r; set_error("the server stopped after an error"); return s->fatal; }
    r->id = s->next_id++;
    r->info.t_submit = now_s(s->t0);
    s->queue.push_back(r);
    s->all[r->id] = r;
    *request_id = r->id;
    s->cv.notify_all();
    return WENOFV_OK;
}

int wenofv_server_poll(wenofv_server *s, int64_t id, double *U, wenofv_request_info *info)
{
    if (!s) { set_error("null server"); return WENOFV_EINVAL; }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) { set_error("unknown request %lld", (long long)id); return WENOFV_ENOTFOUND; }
    Request *r = it->second;
    if (!r->done) return WENOFV_EBUSY;
    if (info) *info = r->info;
    if (U && r->info.status == WENOFV_OK) std::memcpy(U, r->U.data(), r->U.size() * sizeof(double));
    const int st = r->info.status;
    if (st) set_error("request %lld failed with status %d", (long long)id, st);
    s->all.erase(it);
    delete r;
    return st;
}

double wenofv_server_clock(wenofv_server *s) { return s ? now_s(s->t0) : 0.0; }

int wenofv_server_stats(wenofv_server *s, int64_t *admitted, int64_t *completed, int64_t *queued, int64_t *active,
                        int64_t *resident_bytes)
{
    if (!s) { set_error("null server"); return WENOFV_EINVAL; }
    std::lock_guard<std::mutex> lk(s->mu);
    int64_t act = 0;
    for (Request *r : s->active) act += r != nullptr;
    if (admitted) *admitted = s->admitted;
    if (completed) *completed = s->completed;
    if (queued) *queued = (int64_t)s->queue.size();
    if (active) *active = act;
    if (resident_bytes) *resident_bytes = (int64_t)s->resident;
    return WENOFV_OK;
}

} // extern "C"
