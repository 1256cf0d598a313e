// serve.cu -- request loop over resident cases (continuous batching).
//
// A server keeps every admitted case's particles and fields resident on the
// device and advances all of them together, one batched graph per gas (the
// batched form, batch.cu), a few steps per scheduling round.  Between rounds
// it admits queued requests in arrival order while the device footprint
// budget and the slot count allow, and retires cases that have run their
// steps, returning their time-averaged densities and potential.  Requests
// that arrive while others are on the device therefore join the running mix
// at the next round; nothing waits for the mix to drain.
//
// The host-side set-up of a request (deck parsing, the BiCGSTAB solves for
// the Laplace bases and the gas temperature, the particle load) is the slow
// part of admission, so worker threads build set-ups ahead, claiming requests
// in submission order, while the device runs the current mix.
//
// A case's steps depend only on its own state (per-case Philox keys and
// step counter, per-case reduction trees), so a result is the same bit for
// bit whatever else shares the device and however its steps are split into
// rounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "capi_internal.hpp"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    std::string deck;
    int64_t nsteps = 0;
    uint64_t seed = 1;
    double t_submit = 0;
    // filled by the worker
    bool built = false;
    hp_status error = HP_OK;
    std::string message;
    hp::Setup setup;
    size_t est_bytes = 0;
};

struct Resident {
    std::unique_ptr<Request> req;
    hp_case *c = nullptr;
    int64_t left = 0;
    double t_admit = 0;
};

struct Done {
    hp_result r{};
    std::vector<double> den, phi;
};

} // namespace

struct hp_server {
    hp_server_opts o{};
    std::mutex mu;
    std::condition_variable cv_work, cv_built;
    std::deque<std::unique_ptr<Request>> queue; // submitted, in order (built or not)
    size_t next_build = 0;                      // queue index the next idle worker claims
    bool stop = false;
    std::vector<std::thread> workers;
    int64_t next_id = 1;
    // owned by the polling thread
    std::vector<Resident> resident;
    std::map<int, hp_batch *> batches; // per gas
    bool dirty = true;
    size_t used_bytes = 0;
    std::deque<Done> done;
};

namespace {

void worker_main(hp_server *s) {
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || s->next_build < s->queue.size(); });
            if (s->stop) return;
            r = s->queue[s->next_build].get(); // claim the oldest request nobody builds yet
            s->next_build++;
        }
        // build outside the lock: the queue only grows at the back, and the
        // poller removes a request only after it is marked built
        hp_case_opts o = s->o.case_opts;
        o.seed = r->seed;
        hp::BuildOpts b;
        b.seed = o.seed;
        b.cap_per_cell = o.cap_per_cell;
        b.gas_temp_mode = o.gas_temp_mode;
        b.defer_load = o.gpu_load != 0;
        hp_status err = HP_OK;
        std::string msg;
        try {
            hp::build_setup(r->deck.data(), r->deck.size(), b, r->setup);

        } catch (const std::exception &e) {
            msg = e.what();
            err = msg.rfind("unsupported", 0) == 0 ? HP_ERR_UNSUPPORTED : HP_ERR_DECK;
        }
        const size_t est = err == HP_OK ? hpi::estimate_device_bytes(r->setup, o) : 0;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            r->error = err;
            r->message = msg;
            r->est_bytes = est;
            r->built = true;
            std::string().swap(r->deck);
        }
        s->cv_built.notify_all();
    }
}

} // namespace

namespace {

hp_status destroy_batches(hp_server *s) {
    for (auto &kv : s->batches) hp_batch_destroy(kv.second);
    s->batches.clear();
    return HP_OK;
}

// one batch per gas over the resident cases
hp_status rebuild_batches(hp_server *s) {
    destroy_batches(s);
    std::map<int, std::vector<hp_case *>> by_gas;
    for (Resident &r : s->resident) by_gas[r.c->s.main_gas].push_back(r.c);
    for (auto &kv : by_gas) {
        hp_batch *b = nullptr;
        hp_status st = hp_batch_create(kv.second.data(), (int)kv.second.size(), &b);
        if (st != HP_OK) return st;
        s->batches[kv.first] = b;
    }
    s->dirty = false;
    return HP_OK;
}

void finish_failed(hp_server *s, std::unique_ptr<Request> &r, hp_status err, const std::string &msg) {
    Done d;
    d.r.request_id = r->id;
    d.r.error = err;
    d.r.t_submit = r->t_submit;
    d.r.t_admit = d.r.t_done = now_s();
    if (!msg.empty()) hpi::set_error(msg);
    s->done.push_back(std::move(d));
}

// Admit queued requests in order while they fit; the head of the queue is
// never overtaken, so a large case cannot be starved by smaller ones.
hp_status admit(hp_server *s, bool wait_for_head) {
    for (;;) {
        std::unique_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->queue.empty()) return HP_OK;
            if (!s->queue.front()->built) {
                if (!wait_for_head) return HP_OK;
                // nothing on the device: wait (bounded) for the worker instead of spinning
                s->cv_built.wait_for(lk, std::chrono::seconds(1), [&] { return s->queue.front()->built; });
                if (!s->queue.front()->built) return HP_OK;
            }
            Request &h = *s->queue.front();
            if (h.error == HP_OK) {
                if (h.est_bytes > s->o.mem_budget_bytes) {
                    h.error = HP_ERR_CAPACITY;
                    h.message = "request needs " + std::to_string(h.est_bytes) + " device bytes, over the budget";
                } else if ((int)s->resident.size() >= s->o.max_slots ||
                           s->used_bytes + h.est_bytes > s->o.mem_budget_bytes) {
                    return HP_OK; // wait for retirements
                }
            }
            r = std::move(s->queue.front());
            s->queue.pop_front();
            s->next_build--;
        }
        if (r->error != HP_OK) {
            finish_failed(s, r, r->error, r->message);
            continue;
        }
        hp_case_opts o = s->o.case_opts;
        o.seed = r->seed;
        hp_case *c = nullptr;
        hp_status st = hpi::case_from_setup_owned(std::move(r->setup), o, &c);
        if (st != HP_OK) {
            finish_failed(s, r, st, "");
            continue;
        }
        Resident res;
        res.c = c;
        res.left = r->nsteps;
        res.t_admit = now_s();
        res.req = std::move(r);
        s->used_bytes += std::max(c->bytes, res.req->est_bytes);
        s->resident.push_back(std::move(res));
        s->dirty = true;
    }
}

hp_status retire(hp_server *s, size_t k) {
    Resident &r = s->resident[k];
    Done d;
    d.r.request_id = r.req->id;
    d.r.error = HP_OK;
    d.r.t_submit = r.req->t_submit;
    d.r.t_admit = r.t_admit;
    d.r.steps = r.req->nsteps;
    d.r.ngx = r.c->s.ngx;
    d.r.ngy = r.c->s.ngy;
    d.r.nsp = r.c->s.nsp;
    hp_status st = hp_case_status(r.c, &d.r.status);
    if (st == HP_OK) st = hp_case_pushes(r.c, &d.r.particle_pushes);
    const size_t G = (size_t)r.c->s.Gsize, nsp = (size_t)r.c->s.nsp;
    d.den.resize(nsp * G);
    d.phi.resize(G);
    int64_t cnt = 0;
    if (st == HP_OK) st = hp_get_average_count(r.c, &cnt);
    if (st == HP_OK) {
        st = hp_get_grid(r.c, HP_GRID_AVE_DEN, d.den.data(), d.den.size() * 8);
        if (st == HP_OK) st = hp_get_grid(r.c, HP_GRID_AVE_PHI, d.phi.data(), d.phi.size() * 8);
    }
    if (st == HP_OK && cnt > 0) { // running sums -> time averages over the case's steps
        for (double &v : d.den) v /= (double)cnt;
        for (double &v : d.phi) v /= (double)cnt;
    }
    if (st != HP_OK) d.r.error = st;
    d.r.t_done = now_s();
    s->used_bytes -= std::min(s->used_bytes, std::max(r.c->bytes, r.req->est_bytes));
    hp_case_destroy(r.c);
    s->done.push_back(std::move(d));
    s->resident.erase(s->resident.begin() + (long)k);
    s->dirty = true;
    return st;
}

} // namespace

extern "C" {

void hp_server_opts_default(hp_server_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->mem_budget_bytes = (size_t)150 << 30;
    o->max_slots = 64;
    o->steps_per_launch = 50;
    hp_case_opts_default(&o->case_opts);
}

hp_status hp_server_create(const hp_server_opts *o, hp_server **out) {
    if (!o || !out) return hpi::set_error("null argument"), HP_ERR_ARG;
    if (o->max_slots < 1 || o->steps_per_launch < 1 || o->mem_budget_bytes == 0)
        return hpi::set_error("server options out of range"), HP_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
        return hpi::set_error("no CUDA device: libhpic has no CPU path"), HP_ERR_NO_CUDA;
    hp_server *s = new hp_server();
    s->o = *o;
    // set-ups of several requests at once (each is partly threaded itself)
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nw = (int)std::min(4u, std::max(1u, hw / 4));
    for (int k = 0; k < nw; k++) s->workers.emplace_back(worker_main, s);
    *out = s;
    return HP_OK;
}

hp_status hp_server_destroy(hp_server *s) {
    if (!s) return HP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &w : s->workers) w.join();
    destroy_batches(s);
    for (Resident &r : s->resident) hp_case_destroy(r.c);
    delete s;
    return HP_OK;
}

hp_status hp_server_submit(hp_server *s, const char *deck, size_t len, int64_t nsteps, uint64_t seed,
                           int64_t *request_id) {
    if (!s || !deck || nsteps < 1) return hpi::set_error("bad request"), HP_ERR_ARG;
    std::unique_ptr<Request> r(new Request());
    r->deck.assign(deck, len);
    r->nsteps = nsteps;
    r->seed = seed;
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        if (request_id) *request_id = r->id;
        s->queue.push_back(std::move(r));
    }
    s->cv_work.notify_one();
    return HP_OK;
}

hp_status hp_server_poll(hp_server *s, void *stream, int *pending) {
    if (!s) return HP_ERR_ARG;
    hp_status st = admit(s, s->resident.empty());
    if (st != HP_OK) return st;
    if (!s->resident.empty()) {
        if (s->dirty) {
            st = rebuild_batches(s);
            if (st != HP_OK) return st;
        }
        int64_t k = s->o.steps_per_launch;
        for (Resident &r : s->resident) k = std::min(k, r.left);
        for (auto &kv : s->batches) {
            st = hp_batch_step(kv.second, (int)k, stream);
            if (st != HP_OK) return st;
        }
        for (Resident &r : s->resident) r.left -= k;
        bool any = false;
        for (Resident &r : s->resident) any |= r.left == 0;
        if (any) {
            // the batches' graphs reference the retiring cases: drop them first
            destroy_batches(s);
            for (size_t q = s->resident.size(); q-- > 0;)
                if (s->resident[q].left == 0) retire(s, q);
            s->dirty = true;
        }
    }
    if (pending) {
        std::lock_guard<std::mutex> lk(s->mu);
        *pending = (int)(s->queue.size() + s->resident.size());
    }
    return HP_OK;
}

hp_status hp_server_take_result(hp_server *s, hp_result *r, double *ave_den, size_t den_cap, double *ave_phi,
                                size_t phi_cap, int *got) {
    if (!s || !r || !got) return HP_ERR_ARG;
    *got = 0;
    if (s->done.empty()) return HP_OK;
    Done &d = s->done.front();
    if (ave_den && den_cap < d.den.size()) return hpi::set_error("ave_den buffer too small"), HP_ERR_ARG;
    if (ave_phi && phi_cap < d.phi.size()) return hpi::set_error("ave_phi buffer too small"), HP_ERR_ARG;
    *r = d.r;
    if (ave_den) std::copy(d.den.begin(), d.den.end(), ave_den);
    if (ave_phi) std::copy(d.phi.begin(), d.phi.end(), ave_phi);
    s->done.pop_front();
    *got = 1;
    return HP_OK;
}

} // extern "C"
