// serve.cu -- continuous-batching solve server (include/mrlbm.h, "serving").
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <random>
#include <vector>

#include "../../include/mrlbm.h"
#include "domain.h"

using namespace mrlbm;

namespace {

struct Request {
    mrlbm_request r{};
    int status = MRLBM_EBUSY;
    int steps = 0;
    double residual = 1.0;
    double arrival = 0, admitted = -1, finished = -1;
    int member = -1;
    size_t bytes = 0;
    long long nodes = 0;
    bool cancelled = false;
    std::vector<float> result;
};

}  // namespace

struct mrlbm_server {
    int storage = MRLBM_F16;
    double budget = 0;
    int max_active = 0;
    int steps_per_tick = 100;
    double tol = 1e-6;
    int max_steps = 20000;
    bool keep_results = false;
    mrlbm_batch* batch = nullptr;
    std::deque<int> queue;
    std::map<int, Request> reqs;
    std::vector<int> active;
    double used = 0;
    double capacity = 0;  // lattice nodes the active solves may hold together (0: no limit)
    double active_nodes = 0;
    double lups = 0;
    int next_id = 0;
    std::chrono::steady_clock::time_point t0;
};

static double now_s(const mrlbm_server* s)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

// Run-time description of a request (what a reference case fixes in its
// constants.inc): lid cavity as src/cases/lidDrivenCavity_3D, duct with walls
// on x and y, periodic z, body force and a power-law fluid.
static mrlbm_status request_desc(const mrlbm_server* s, const mrlbm_request& r, mrlbm_desc* d)
{
    if (r.n < 4 || r.n > 1024) return fail(MRLBM_EINVAL, "request edge %d out of range", r.n);
    memset(d, 0, sizeof(*d));
    d->nx = d->ny = d->nz = r.n;
    d->lattice = MRLBM_D3Q19;
    d->storage = s->storage;
    d->rho0 = 1.0;
    if (r.kind == MRLBM_REQ_LID_CAVITY) {
        const double lid = r.lid_u > 0 ? r.lid_u : 0.05;
        if (!(r.re > 0)) return fail(MRLBM_EINVAL, "cavity request needs re > 0");
        d->tau = 0.5 + 3.0 * lid * r.n / r.re;
        d->bc_velocity[1][0] = lid;
    } else if (r.kind == MRLBM_REQ_DUCT) {
        d->periodic[2] = 1;
        d->tau = r.tau > 0.5 ? r.tau : 0.8;
        d->rheology = MRLBM_POWERLAW;
        d->nnf_n = r.nnf_n > 0 ? r.nnf_n : 1.0;
        // Newtonian square duct: u_max = 0.0737 F H^2 / nu, sized for u_max ~ 0.05
        const double nu = (d->tau - 0.5) / 3.0, H = r.n - 1;
        d->force[2] = r.force_z != 0.0 ? r.force_z : 0.05 * nu / (0.0737 * H * H);
    } else {
        return fail(MRLBM_EINVAL, "unknown request kind %d", r.kind);
    }
    return MRLBM_OK;
}

static mrlbm_status request_node_types(const mrlbm_request& r, std::vector<uint32_t>& nt)
{
    const int n = r.n;
    nt.resize((size_t)n * n * n);
    if (r.kind == MRLBM_REQ_LID_CAVITY) return mrlbm_lid_cavity_node_types(n, n, n, 1, nt.data());
    std::vector<uint8_t> solid((size_t)n * n * n, 0);
    std::mt19937_64 rng(r.seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    for (int z = 0; z < n; z++)
        for (int y = 1; y < n - 1; y++)
            for (int x = 1; x < n - 1; x++)
                if (U(rng) < r.solid_fraction) solid[(size_t)x + (size_t)n * (y + (size_t)n * z)] = 1;
    const int periodic[3] = {0, 0, 1};
    return mrlbm_voxel_node_types(n, n, n, solid.data(), periodic, nt.data());
}

extern "C" mrlbm_status mrlbm_request_describe(const mrlbm_request* r, int storage, mrlbm_desc* desc,
                                              uint32_t* node_types)
{
    if (!r || !desc) return fail(MRLBM_EINVAL, "null argument");
    mrlbm_server tmp;
    tmp.storage = storage;
    mrlbm_status st = request_desc(&tmp, *r, desc);
    if (st) return st;
    if (node_types) {
        std::vector<uint32_t> nt;
        if ((st = request_node_types(*r, nt))) return st;
        memcpy(node_types, nt.data(), nt.size() * sizeof(uint32_t));
    }
    return MRLBM_OK;
}

// A standalone domain for a request (same description, node types and
// initial state as the server gives it), e.g. to solve it alone.
extern "C" mrlbm_status mrlbm_request_domain(const mrlbm_request* r, int storage, mrlbm_domain** out)
{
    if (!r || !out) return fail(MRLBM_EINVAL, "null argument");
    mrlbm_server tmp;
    tmp.storage = storage;
    mrlbm_desc d;
    mrlbm_status st = request_desc(&tmp, *r, &d);
    if (st) return st;
    std::vector<uint32_t> nt;
    if ((st = request_node_types(*r, nt))) return st;
    mrlbm_domain* dom = nullptr;
    if ((st = mrlbm_domain_create(&d, &dom))) return st;
    if ((st = mrlbm_set_node_types(dom, nt.data())) || (st = mrlbm_init_uniform(dom, nullptr))) {
        mrlbm_domain_destroy(dom);
        return st;
    }
    *out = dom;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_create(int storage, double budget, int max_active, int steps_per_tick,
                                           double residual_tol, int max_steps, mrlbm_server** out)
{
    if (!out) return fail(MRLBM_EINVAL, "null output handle");
    *out = nullptr;
    if (!(budget > 0) || max_active < 1 || steps_per_tick < 1 || max_steps < 1)
        return fail(MRLBM_EINVAL, "bad server parameters");
    mrlbm_server* s = new mrlbm_server();
    s->storage = storage;
    s->budget = budget;
    s->max_active = max_active;
    s->steps_per_tick = steps_per_tick;
    s->tol = residual_tol;
    s->max_steps = max_steps;
    s->t0 = std::chrono::steady_clock::now();
    mrlbm_status st = mrlbm_batch_create(MRLBM_D3Q19, storage, &s->batch);
    if (st) {
        delete s;
        return st;
    }
    *out = s;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_destroy(mrlbm_server* s)
{
    if (!s) return MRLBM_OK;
    mrlbm_batch_destroy(s->batch);
    delete s;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_set_capacity(mrlbm_server* s, double nodes)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    if (!(nodes >= 0)) return fail(MRLBM_EINVAL, "capacity %g nodes", nodes);
    s->capacity = nodes;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_keep_results(mrlbm_server* s, int on)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    s->keep_results = on != 0;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_submit(mrlbm_server* s, const mrlbm_request* r, int* rid)
{
    if (!s || !r || !rid) return fail(MRLBM_EINVAL, "null argument");
    mrlbm_desc d;
    mrlbm_status st = request_desc(s, *r, &d);
    if (st) return st;
    size_t bytes = 0;
    if ((st = mrlbm_domain_bytes(&d, &bytes))) return st;
    if ((double)bytes > s->budget) return fail(MRLBM_ENOMEM, "request needs %zu bytes, budget %.0f", bytes, s->budget);
    Request q;
    q.r = *r;
    q.bytes = bytes;
    q.nodes = (long long)r->n * r->n * r->n;
    q.arrival = r->arrival >= 0 ? r->arrival : now_s(s);
    const int id = s->next_id++;
    s->reqs.emplace(id, std::move(q));
    // keep the queue in arrival order
    auto pos = std::upper_bound(s->queue.begin(), s->queue.end(), s->reqs[id].arrival,
                                [&](double t, int other) { return t < s->reqs[other].arrival; });
    s->queue.insert(pos, id);
    *rid = id;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_cancel(mrlbm_server* s, int rid)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return fail(MRLBM_ENOTFOUND, "no request %d", rid);
    Request& q = it->second;
    if (q.status != MRLBM_EBUSY) return MRLBM_OK;  // already finished
    q.cancelled = true;
    auto qi = std::find(s->queue.begin(), s->queue.end(), rid);
    if (qi != s->queue.end()) {
        s->queue.erase(qi);
        q.status = MRLBM_ECANCELED;
        q.finished = now_s(s);
    }
    return MRLBM_OK;
}

static mrlbm_status admit(mrlbm_server* s, int rid)
{
    Request& q = s->reqs[rid];
    mrlbm_desc d;
    mrlbm_status st = request_desc(s, q.r, &d);
    if (st) return st;
    std::vector<uint32_t> nt;
    if ((st = request_node_types(q.r, nt))) return st;
    int mid = -1;
    if ((st = mrlbm_batch_add(s->batch, &d, &mid))) return st;
    mrlbm_domain* dom = nullptr;
    if ((st = mrlbm_batch_domain(s->batch, mid, &dom)) || (st = mrlbm_set_node_types(dom, nt.data())) ||
        (st = mrlbm_init_uniform(dom, nullptr))) {
        mrlbm_batch_remove(s->batch, mid);
        return st;
    }
    double r0;
    if ((st = mrlbm_residual(dom, &r0))) {  // first call: snapshot
        mrlbm_batch_remove(s->batch, mid);
        return st;
    }
    q.member = mid;
    q.admitted = now_s(s);
    s->used += (double)q.bytes;
    s->active_nodes += (double)q.nodes;
    s->active.push_back(rid);
    return MRLBM_OK;
}

static mrlbm_status retire(mrlbm_server* s, int rid, int status)
{
    Request& q = s->reqs[rid];
    mrlbm_domain* dom = nullptr;
    mrlbm_status st = mrlbm_batch_domain(s->batch, q.member, &dom);
    if (st) return st;
    if (s->keep_results && status != MRLBM_ECANCELED) {
        int nm = 0;
        mrlbm_num_moments(dom, &nm);
        q.result.resize((size_t)nm * q.nodes);
        if ((st = mrlbm_get_moments(dom, q.result.data()))) return st;
    }
    if ((st = mrlbm_batch_remove(s->batch, q.member))) return st;
    q.member = -1;
    q.status = status;
    q.finished = now_s(s);
    s->used -= (double)q.bytes;
    s->active_nodes -= (double)q.nodes;
    s->active.erase(std::find(s->active.begin(), s->active.end(), rid));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_tick(mrlbm_server* s, int* active_out)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    mrlbm_status st;
    // cancelled running solves leave first
    for (int rid : std::vector<int>(s->active))
        if (s->reqs[rid].cancelled && (st = retire(s, rid, MRLBM_ECANCELED))) return st;
    // admission in arrival order, against the slot limit and the HBM budget
    const double t = now_s(s);
    while (!s->queue.empty() && (int)s->active.size() < s->max_active) {
        const int rid = s->queue.front();
        Request& q = s->reqs[rid];
        if (q.arrival > t) break;
        if (s->used + (double)q.bytes > s->budget) break;
        // the compute limit: a solve joins the running ones only while their
        // nodes together still fit it; with nothing running it always starts
        if (s->capacity > 0 && !s->active.empty() && s->active_nodes + (double)q.nodes > s->capacity) break;
        s->queue.pop_front();
        if ((st = admit(s, rid))) {
            q.status = st;
            q.finished = now_s(s);
            continue;
        }
    }
    if (s->active.size() == 1) {
        // a lone solve runs on the single-domain step kernel: same arithmetic
        // (bit-identical results), no work queue, a grid sized for its grid
        mrlbm_domain* dom = nullptr;
        if ((st = mrlbm_batch_domain(s->batch, s->reqs[s->active[0]].member, &dom))) return st;
        // the single-domain grid's own z chunking (the batch sets its own
        // chunk again before its next step)
        dom->lz = 0;
        if ((st = mrlbm_step(dom, s->steps_per_tick))) return st;
    } else if (!s->active.empty()) {
        if ((st = mrlbm_batch_step(s->batch, s->steps_per_tick))) return st;
    }
    if (!s->active.empty()) {
        for (int rid : s->active) {
            Request& q = s->reqs[rid];
            q.steps += s->steps_per_tick;
            s->lups += (double)q.nodes * s->steps_per_tick;
        }
        // convergence / divergence / step-limit checks
        for (int rid : std::vector<int>(s->active)) {
            Request& q = s->reqs[rid];
            mrlbm_domain* dom = nullptr;
            if ((st = mrlbm_batch_domain(s->batch, q.member, &dom))) return st;
            mrlbm_sums sums;
            if ((st = mrlbm_reduce_fp64(dom, &sums))) return st;
            if (sums.nonfinite > 0 || !(sums.max_speed < 0.3)) {
                if ((st = retire(s, rid, MRLBM_EDIVERGED))) return st;
                continue;
            }
            if ((st = mrlbm_residual(dom, &q.residual))) return st;
            if (q.residual <= s->tol || q.steps >= s->max_steps)
                if ((st = retire(s, rid, MRLBM_OK))) return st;
        }
    }
    if (active_out) *active_out = (int)s->active.size();
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_result(mrlbm_server* s, int rid, mrlbm_request_result* out)
{
    if (!s || !out) return fail(MRLBM_EINVAL, "null argument");
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return fail(MRLBM_ENOTFOUND, "no request %d", rid);
    const Request& q = it->second;
    out->status = q.status;
    out->steps = q.steps;
    out->residual = q.residual;
    out->arrival = q.arrival;
    out->admitted = q.admitted;
    out->finished = q.finished;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_moments(mrlbm_server* s, int rid, float* m, size_t count)
{
    if (!s || !m) return fail(MRLBM_EINVAL, "null argument");
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return fail(MRLBM_ENOTFOUND, "no request %d", rid);
    if (it->second.result.empty()) return fail(MRLBM_ENOTFOUND, "request %d has no kept result", rid);
    if (count != it->second.result.size())
        return fail(MRLBM_EINVAL, "result has %zu values, buffer %zu", it->second.result.size(), count);
    memcpy(m, it->second.result.data(), count * sizeof(float));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_release(mrlbm_server* s, int rid)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return fail(MRLBM_ENOTFOUND, "no request %d", rid);
    if (it->second.status == MRLBM_EBUSY) return fail(MRLBM_EBUSY, "request %d still running", rid);
    s->reqs.erase(it);
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_stats_get(mrlbm_server* s, mrlbm_server_stats* out)
{
    if (!s || !out) return fail(MRLBM_EINVAL, "null argument");
    memset(out, 0, sizeof(*out));
    std::vector<double> lat;
    double first = 1e300, last = 0;
    for (const auto& kv : s->reqs) {
        const Request& q = kv.second;
        if (q.status == MRLBM_OK) {
            out->done++;
            lat.push_back(q.finished - q.arrival);
            first = std::min(first, q.arrival);
            last = std::max(last, q.finished);
        } else if (q.status != MRLBM_EBUSY) {
            out->failed++;
        }
    }
    out->queued = (int)s->queue.size();
    out->active = (int)s->active.size();
    out->hbm_in_use = s->used;
    out->lattice_updates = s->lups;
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double p) {
            const double r = p * (lat.size() - 1);
            const size_t lo = (size_t)std::floor(r), hi = std::min(lat.size() - 1, lo + 1);
            return lat[lo] + (r - lo) * (lat[hi] - lat[lo]);
        };
        out->p50_latency = pct(0.50);
        out->p99_latency = pct(0.99);
        double sum = 0;
        for (double v : lat) sum += v;
        out->mean_latency = sum / lat.size();
        out->solves_per_s = last > first ? out->done / (last - first) : 0.0;
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_now(mrlbm_server* s, double* t)
{
    if (!s || !t) return fail(MRLBM_EINVAL, "null argument");
    *t = now_s(s);
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_server_inject_nan(mrlbm_server* s, int rid)
{
    if (!s) return fail(MRLBM_EINVAL, "null server");
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end() || it->second.member < 0) return fail(MRLBM_ENOTFOUND, "request %d not running", rid);
    mrlbm_domain* dom = nullptr;
    mrlbm_status st = mrlbm_batch_domain(s->batch, it->second.member, &dom);
    if (st) return st;
    int nm = 0;
    mrlbm_num_moments(dom, &nm);
    std::vector<float> m((size_t)nm * it->second.nodes);
    if ((st = mrlbm_get_moments(dom, m.data()))) return st;
    const size_t mid = (size_t)it->second.nodes / 2;
    m[1 * it->second.nodes + mid] = std::nanf("");
    return mrlbm_set_moments(dom, m.data());
}
