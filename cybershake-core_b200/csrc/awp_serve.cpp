/*
 * awp_serve.cpp -- continuous batching of SGT solves on one GPU.
 *
 * One scheduler thread owns every resident solver.  It admits queued
 * requests in arrival order while their footprint fits in the HBM budget,
 * keeps one chunk of steps in flight per resident solver (each on its own
 * CUDA stream, so kernels of different requests overlap), finishes requests
 * whose last chunk completed (SGT images copied to the caller's buffer,
 * device memory released) and honours cancellations.  Host threads talk to
 * it through a mutex-protected table of requests.
 */
#include <cuda_runtime.h>
#include <string.h>

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
    bool cancel = false;
    bool in_flight = false;
};

awp_status fail(awp_status st, const char *msg)
{
    awp_set_error_text(msg);
    return st;
}

}  // namespace

struct awp_server {
    int device;
    int64_t budget;
    int64_t reserved = 0;
    int max_active;
    int chunk;
    std::mutex mu;
    std::condition_variable cv;      /* scheduler wake-up   */
    std::condition_variable done_cv; /* request ended       */
    std::deque<int64_t> queue;
    std::map<int64_t, Req *> reqs;
    std::vector<Req *> active;
    int64_t next_id = 1;
    bool stop = false;
    std::thread th;
    std::chrono::steady_clock::time_point t0;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    void loop();
    void finish(Req *r, int state, awp_status st);
    awp_status admit(Req *r);
};

void awp_server::finish(Req *r, int state, awp_status st)
{
    /* called with mu held */
    if (r->s) {
        awp_destroy(r->s);
        r->s = nullptr;
    }
    reserved -= r->info.footprint;
    r->info.state = state;
    r->info.status = st;
    r->info.t_done = now();
    done_cv.notify_all();
}

awp_status awp_server::admit(Req *r)
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

void awp_server::loop()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
        bool busy = false;
        /* admissions, in arrival order */
        while (!queue.empty() && (int)active.size() < max_active) {
            Req *r = reqs[queue.front()];
            if (r->cancel) {
                queue.pop_front();
                r->info.footprint = 0;
                finish(r, AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
                continue;
            }
            if (reserved + r->info.footprint > budget && !active.empty()) break;
            queue.pop_front();
            reserved += r->info.footprint;
            r->info.state = AWP_REQ_RUNNING;
            r->info.t_admit = now();
            lk.unlock();
            awp_status st = admit(r);
            lk.lock();
            if (st != AWP_OK) finish(r, AWP_REQ_FAILED, st);
            else active.push_back(r);
            busy = true;
        }
        /* progress of the resident solves */
        for (size_t n = 0; n < active.size();) {
            Req *r = active[n];
            const int q = r->in_flight ? awp_query(r->s) : 1;
            if (q < 0 || r->cancel) {
                if (r->in_flight) awp_sync(r->s);
                finish(r, r->cancel ? AWP_REQ_CANCELLED : AWP_REQ_FAILED, r->cancel ? AWP_ERR_CANCELLED : AWP_ERR_CUDA);
                active.erase(active.begin() + n);
                busy = true;
                continue;
            }
            if (q == 1) {
                awp_status st = AWP_OK;
                if (r->in_flight) {
                    st = awp_sync(r->s);
                    r->in_flight = false;
                    awp_stats stt;
                    awp_get_stats(r->s, &stt);
                    r->info.steps_done = stt.steps_done;
                }
                if (st == AWP_OK && r->info.steps_done < r->rq.params.nt) {
                    st = awp_run_async(r->s, chunk);
                    r->in_flight = (st == AWP_OK);
                } else if (st == AWP_OK) {
                    const int64_t nf = awp_sgt_file_floats(r->s);
                    for (int c = 0; c < r->rq.params.ncomp && st == AWP_OK; c++)
                        if (r->rq.sgt_out) st = awp_get_sgt(r->s, c, r->rq.sgt_out + (size_t)c * (size_t)nf);
                    finish(r, st == AWP_OK ? AWP_REQ_DONE : AWP_REQ_FAILED, st);
                    active.erase(active.begin() + n);
                    busy = true;
                    continue;
                }
                if (st != AWP_OK) {
                    finish(r, AWP_REQ_FAILED, st);
                    active.erase(active.begin() + n);
                    busy = true;
                    continue;
                }
                busy = true;
            }
            n++;
        }
        if (!busy) cv.wait_for(lk, std::chrono::microseconds(200));
    }
    /* shutdown: cancel what is left */
    for (Req *r : active) {
        if (r->in_flight) awp_sync(r->s);
        finish(r, AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
    }
    active.clear();
    for (int64_t id : queue) {
        reqs[id]->info.footprint = 0;
        finish(reqs[id], AWP_REQ_CANCELLED, AWP_ERR_CANCELLED);
    }
    queue.clear();
}

extern "C" awp_status awp_server_create(int device, int64_t hbm_budget, int max_active, int chunk_steps,
                                        awp_server **out)
{
    *out = nullptr;
    if (max_active < 1 || chunk_steps < 1) return fail(AWP_ERR_PARAM, "max_active and chunk_steps must be >= 1");
    if (cudaSetDevice(device) != cudaSuccess) return fail(AWP_ERR_CUDA, "cannot select the device");
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return fail(AWP_ERR_CUDA, "cudaMemGetInfo failed");
    awp_server *sv = new awp_server();
    sv->device = device;
    sv->budget = hbm_budget > 0 ? hbm_budget : (int64_t)(0.9 * (double)fr);
    sv->max_active = max_active;
    sv->chunk = chunk_steps;
    sv->t0 = std::chrono::steady_clock::now();
    sv->th = std::thread([sv] { sv->loop(); });
    *out = sv;
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
    sv->th.join();
    for (auto &kv : sv->reqs) delete kv.second;
    delete sv;
    return AWP_OK;
}
