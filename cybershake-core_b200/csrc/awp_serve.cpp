/*
 * awp_serve.cpp -- continuous batching of SGT solves on one GPU.
 *
 * Three host threads share a mutex-protected table of requests:
 *  - the admitter takes queued requests (arrival order, or shortest total
 *    work first) while their footprint fits in the HBM budget, fewer than
 *    max_active solves are resident and the resident solves do not already
 *    fill the GPU, and builds each one (device allocation, media, sources,
 *    points) while the others keep stepping;
 *  - the scheduler keeps one chunk of steps in flight per resident solve,
 *    each on its own CUDA stream, so kernels of different requests overlap;
 *    a chunk is sized to about chunk_cells cell-updates, so small solves are
 *    not stepped in slivers;
 *  - the reaper copies a finished request's SGT file images to the caller's
 *    buffer and releases its device memory (a device-wide synchronisation,
 *    kept off the scheduler's path).
 */
#include <cuda_runtime.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/awp_sgt.h"

extern "C" void awp_set_error_text(const char *msg);

namespace {

struct Req {
    int64_t id;
    awp_request rq;
    awp_request_info info;
    awp_solver *s = nullptr;
    std::atomic<bool> cancel{false};
    bool in_flight = false;
    double cells = 0;      /* cells x components: work of one step */
    double work = 0;       /* cells x components x steps           */
    int sm_share = 0;      /* SMs its grids are sized for (0 = all)  */
};

awp_status fail(awp_status st, const char *msg)
{
    awp_set_error_text(msg);
    return st;
}

}  // namespace

struct awp_server {
    int device;
    int nsm = 148;                   /* SMs of the device                */
    int64_t budget;
    int64_t reserved = 0;
    int max_active;
    int chunk;                       /* fewest steps per chunk         */
    int policy = AWP_SERVE_FIFO;
    double fill_cells = 32.0e6;      /* resident cells x comps that fill the GPU */
    double chunk_cells = 4.0e8;      /* cell-updates per chunk (target) */
    std::mutex mu;
    std::condition_variable cv;      /* scheduler, admitter and reaper wake-up */
    std::condition_variable done_cv; /* a request ended                       */
    std::deque<int64_t> queue;
    std::map<int64_t, Req *> reqs;
    std::vector<Req *> active;       /* resident and stepping            */
    std::deque<Req *> reap;          /* finished stepping, to be released */
    int admitting = 0;
    int64_t next_id = 1;
    bool stop = false;
    bool reap_stop = false;          /* set once nothing can reach the reaper */
    std::thread th_sched, th_admit, th_reap;
    std::chrono::steady_clock::time_point t0;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void sched_loop();
    void admit_loop();
    void reap_loop();
    awp_status share_sms(Req *r, int resident, bool first);
    void end(Req *r, int state, awp_status st);
    awp_status build(Req *r);
    double resident_cells() const
    {
        double c = 0;
        for (const Req *r : active) c += r->cells;
        return c;
    }
    /* memory first (released solves still held by the reaper count), then
     * the number of resident solves and how much of the GPU they fill */
    bool can_admit(const Req *r) const
    {
        if (reserved > 0 && reserved + r->info.footprint > budget) return false;
        const int resident = (int)active.size() + admitting;
        if (resident == 0) return true;
        if (resident >= max_active) return false;
        return resident_cells() + r->cells <= fill_cells;
    }
};

/* called with mu held; the solver is already destroyed */
void awp_server::end(Req *r, int state, awp_status st)
{
    reserved -= r->info.footprint;
    r->info.state = state;
    r->info.status = st;
    r->info.t_done = now();
    done_cv.notify_all();
    cv.notify_all();
}

awp_status awp_server::build(Req *r)
{
    awp_solver *s = nullptr;
    awp_status st = awp_create(&r->rq.params, &s);
    if (st == AWP_OK) st = awp_load_media(s, r->rq.media);
    for (int q = 0; q < r->rq.params.ncomp && st == AWP_OK; q++)
        st = awp_set_source(s, q, r->rq.nsrc[q], r->rq.src_xyz[q], r->rq.stf[q]);
    if (st == AWP_OK) st = awp_set_points(s, r->rq.npts, r->rq.pts);
    if (st != AWP_OK) {
        if (s) awp_destroy(s);
        return st;
    }
    r->s = s;
    return AWP_OK;
}

/* Each resident solve's persistent grids span its share of the SMs (all of
 * them when it is alone), so that solves sharing the GPU run side by side
 * instead of taking turns with grids that each fill the device: equal shares,
 * or under AWP_SERVE_FIFO_SRPT a double share for the solve with the least
 * remaining work (`first`).  The share is set between chunks, when nothing of
 * the solve is in flight; launch shapes do not change results. */
awp_status awp_server::share_sms(Req *r, int resident, bool first)
{
    int want = resident <= 1 ? 0 : (nsm + resident - 1) / resident;
    if (resident > 1 && policy == AWP_SERVE_FIFO_SRPT) want = (nsm * (first ? 2 : 1) + resident) / (resident + 1);
    if (want == r->sm_share) return AWP_OK;
    awp_tuning t;
    awp_status st = awp_get_tuning(r->s, &t);
    if (st != AWP_OK) return st;
    t.sm_limit = want;
    st = awp_set_tuning(r->s, &t);
    if (st == AWP_OK) r->sm_share = want;
    return st;
}

/* steps of the next chunk: about chunk_cells cell-updates, at least `chunk`,
 * a whole number of SGT periods so that the solve keeps replaying graphs */
static int chunk_steps_for(const awp_server *sv, const Req *r)
{
    const double want = sv->chunk_cells / (r->cells > 1 ? r->cells : 1);
    int steps = want > 1e9 ? 1000000000 : (int)want;
    if (steps < sv->chunk) steps = sv->chunk;
    const int gs = r->rq.params.ntiskp_sgt > 0 ? r->rq.params.ntiskp_sgt : 1;
    return ((steps + gs - 1) / gs) * gs;
}

void awp_server::admit_loop()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
        for (auto it = queue.begin(); it != queue.end();) {
            Req *r = reqs[*it];
            if (r->cancel) {
                r->info.footprint = 0;
                end(r, AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
                it = queue.erase(it);
            } else {
                ++it;
            }
        }
        auto pit = queue.begin();
        if (policy == AWP_SERVE_SJF)
            for (auto it = queue.begin(); it != queue.end(); ++it)
                if (reqs[*it]->work < reqs[*pit]->work) pit = it;
        Req *r = pit == queue.end() ? nullptr : reqs[*pit];
        if (!r || !can_admit(r)) {
            cv.wait_for(lk, std::chrono::milliseconds(1));
            continue;
        }
        queue.erase(pit);
        reserved += r->info.footprint;
        r->info.state = AWP_REQ_RUNNING;
        r->info.t_admit = now();
        admitting++;
        lk.unlock();
        const awp_status st = build(r);
        lk.lock();
        admitting--;
        if (st != AWP_OK) end(r, AWP_REQ_FAILED, st);
        else active.push_back(r);
        cv.notify_all();
    }
}

void awp_server::sched_loop()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    std::vector<Req *> snap, done;
    while (!stop) {
        snap = active;
        lk.unlock();
        bool busy = false;
        done.clear();
        for (Req *r : snap) {
            const int q = r->in_flight ? awp_query(r->s) : 1;
            if (q == 0 && !r->cancel) continue;
            awp_status st = AWP_OK;
            int64_t steps = r->info.steps_done;
            if (r->in_flight) {
                st = awp_sync(r->s);
                r->in_flight = false;
                awp_stats stt;
                if (awp_get_stats(r->s, &stt) == AWP_OK) steps = stt.steps_done;
            }
            if (q < 0 && st == AWP_OK) st = AWP_ERR_CUDA;
            if (st == AWP_OK && !r->cancel && steps < r->rq.params.nt) {
                /* least remaining work among the resident solves (ties: lower id) */
                bool first = true;
                const double left = r->cells * (double)(r->rq.params.nt - steps);
                for (Req *o : snap) {
                    if (o == r) continue;
                    const double ol = o->cells * (double)(o->rq.params.nt - o->info.steps_done);
                    if (ol < left || (ol == left && o->id < r->id)) first = false;
                }
                st = share_sms(r, (int)snap.size(), first);
                if (st == AWP_OK) st = awp_run_async(r->s, chunk_steps_for(this, r));
                r->in_flight = st == AWP_OK;
            }
            lk.lock();
            r->info.steps_done = steps;
            if (!r->in_flight) {                 /* finished, failed or cancelled */
                r->info.status = st;
                done.push_back(r);
            }
            lk.unlock();
            busy = true;
        }
        lk.lock();
        for (Req *r : done) {
            for (size_t n = 0; n < active.size(); n++)
                if (active[n] == r) {
                    active.erase(active.begin() + n);
                    break;
                }
            reap.push_back(r);
        }
        if (!done.empty()) cv.notify_all();
        if (!busy) cv.wait_for(lk, std::chrono::microseconds(100));
    }
}

void awp_server::reap_loop()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        if (reap.empty()) {
            if (reap_stop) break;
            cv.wait_for(lk, std::chrono::milliseconds(1));
            continue;
        }
        Req *r = reap.front();
        reap.pop_front();
        const bool complete = r->info.status == AWP_OK && r->info.steps_done >= r->rq.params.nt;
        awp_status st = r->info.status;
        lk.unlock();
        if (complete && r->rq.sgt_out) {
            const int64_t nf = awp_sgt_file_floats(r->s);
            for (int c = 0; c < r->rq.params.ncomp && st == AWP_OK; c++)
                st = awp_get_sgt(r->s, c, r->rq.sgt_out + (size_t)c * (size_t)nf);
        }
        awp_destroy(r->s);
        lk.lock();
        r->s = nullptr;
        if (complete) end(r, st == AWP_OK ? AWP_REQ_DONE : AWP_REQ_FAILED, st);
        else if (r->cancel) end(r, AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
        else end(r, AWP_REQ_FAILED, st == AWP_OK ? AWP_ERR_CUDA : st);
    }
}

extern "C" awp_status awp_server_create(int device, int64_t hbm_budget, int max_active, int chunk_steps,
                                        awp_server **out)
{
    *out = nullptr;
    if (max_active < 1 || chunk_steps < 1) return fail(AWP_ERR_PARAM, "max_active and chunk_steps must be >= 1");
    if (cudaSetDevice(device) != cudaSuccess) return fail(AWP_ERR_CUDA, "cannot select the device");
    size_t fr = 0, tot = 0;
    awp_release_cached_memory();       /* the budget counts idle cached blocks as free */
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaMemGetInfo failed");
    awp_server *sv = new awp_server();
    sv->device = device;
    cudaDeviceGetAttribute(&sv->nsm, cudaDevAttrMultiProcessorCount, device);
    sv->budget = hbm_budget > 0 ? hbm_budget : (int64_t)(0.9 * (double)fr);
    sv->max_active = max_active;
    sv->chunk = chunk_steps;
    sv->t0 = std::chrono::steady_clock::now();
    sv->th_reap = std::thread([sv] { sv->reap_loop(); });
    sv->th_sched = std::thread([sv] { sv->sched_loop(); });
    sv->th_admit = std::thread([sv] { sv->admit_loop(); });
    *out = sv;
    return AWP_OK;
}

extern "C" awp_status awp_server_configure(awp_server *sv, int policy, double fill_cells, double chunk_cells)
{
    if (!sv) return fail(AWP_ERR_PARAM, "null server");
    if (policy != AWP_SERVE_FIFO && policy != AWP_SERVE_SJF && policy != AWP_SERVE_FIFO_SRPT)
        return fail(AWP_ERR_PARAM, "unknown admission policy");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->policy = policy;
    if (fill_cells > 0) sv->fill_cells = fill_cells;
    if (chunk_cells > 0) sv->chunk_cells = chunk_cells;
    sv->cv.notify_all();
    return AWP_OK;
}

extern "C" awp_status awp_submit(awp_server *sv, const awp_request *rq, int64_t *id)
{
    if (!sv || !rq || !id) return fail(AWP_ERR_PARAM, "null argument");
    const int64_t fp = awp_footprint_bytes(&rq->params, rq->npts);
    Req *r = new Req();
    r->rq = *rq;
    memset(&r->info, 0, sizeof r->info);
    r->info.state = AWP_REQ_QUEUED;
    r->info.footprint = fp;
    const awp_params &p = rq->params;
    r->cells = (double)p.nx * p.ny * p.nz * (p.ncomp > 0 ? p.ncomp : 1);
    r->work = r->cells * p.nt;
    std::lock_guard<std::mutex> lk(sv->mu);
    if (fp > sv->budget) {
        delete r;
        return fail(AWP_ERR_BUSY, "request footprint exceeds the server's HBM budget");
    }
    r->id = sv->next_id++;
    r->info.t_submit = sv->now();
    sv->reqs[r->id] = r;
    sv->queue.push_back(r->id);
    *id = r->id;
    sv->cv.notify_all();
    return AWP_OK;
}

extern "C" awp_status awp_poll(awp_server *sv, int64_t id, awp_request_info *info)
{
    if (!sv || !info) return fail(AWP_ERR_PARAM, "null argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return fail(AWP_ERR_PARAM, "unknown request id");
    *info = it->second->info;
    return AWP_OK;
}

extern "C" awp_status awp_cancel(awp_server *sv, int64_t id)
{
    if (!sv) return fail(AWP_ERR_PARAM, "null server");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return fail(AWP_ERR_PARAM, "unknown request id");
    it->second->cancel = true;
    sv->cv.notify_all();
    return AWP_OK;
}

extern "C" awp_status awp_wait(awp_server *sv, int64_t id, double timeout_s, awp_request_info *info)
{
    if (!sv) return fail(AWP_ERR_PARAM, "null server");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return fail(AWP_ERR_PARAM, "unknown request id");
    Req *r = it->second;
    auto ended = [r] { return r->info.state >= AWP_REQ_DONE; };
    if (!sv->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ended)) {
        if (info) *info = r->info;
        return fail(AWP_ERR_TIMEOUT, "request still running");
    }
    if (info) *info = r->info;
    return AWP_OK;
}

extern "C" double awp_server_time(awp_server *sv) { return sv ? sv->now() : 0.0; }

extern "C" awp_status awp_server_destroy(awp_server *sv)
{
    if (!sv) return AWP_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->cv.notify_all();
    }
    sv->th_admit.join();            /* a request being built ends up resident */
    sv->th_sched.join();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        for (Req *r : sv->active) {  /* resident solves: cancelled, released by the reaper */
            r->cancel = true;
            r->info.status = AWP_ERR_CANCELLED;
            sv->reap.push_back(r);
        }
        sv->active.clear();
        for (int64_t id : sv->queue) {
            Req *r = sv->reqs[id];
            r->info.footprint = 0;
            sv->end(r, AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
        }
        sv->queue.clear();
        sv->reap_stop = true;
        sv->cv.notify_all();
    }
    sv->th_reap.join();
    for (auto &kv : sv->reqs) delete kv.second;
    delete sv;
    return AWP_OK;
}
