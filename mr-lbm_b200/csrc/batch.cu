// batch.cu -- C ABI of domain batches (include/mrlbm.h, "batches").
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/mrlbm.h"
#include "batch_kernel.cuh"
#include "domain.h"

using namespace mrlbm;

#define CK(call)                                                                                               \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess)                                                                                 \
            return fail(MRLBM_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

struct mrlbm_batch {
    int lattice = 19, storage = MRLBM_F32;
    std::vector<mrlbm_domain*> members;  // id -> domain (nullptr: removed)
    std::vector<int> offsets;            // id -> parity offset
    std::vector<BatchDomain> h_doms;
    BatchDomain* d_doms = nullptr;
    int dom_cap = 0;
    BatchItem* d_items = nullptr;
    int item_cap = 0;
    int nitems = 0;
    std::vector<BatchItem> h_items;
    BatchCtl* d_ctl = nullptr;
    long long step = 0;  // host mirror of the device step counter
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int rows = TYI_BULK;   // rows per CTA of the batch kernel (TYI_BULK or TYI_WALL)
    int grid[2] = {148, 148};   // persistent grid per tile kind (tile_kind(rows))
    size_t smem[2] = {0, 0};
    std::map<int, int> lz_by_class;  // autotuned z-chunk per size class
};

namespace {

// the batch kernel's rows per CTA
int batch_rows(const mrlbm_batch* b) { return b->rows; }

// shared memory and persistent grid of the batch kernel of each tile height
template <int Q, typename T, int S, int TYI>
mrlbm_status set_shape(mrlbm_batch* b, int sms)
{
    const int k = tile_kind(TYI);
    b->smem[k] = ZSmem<Q, T, TYI, batch_npm<T, S>(), false, BATCH_STATIC_SMEM, batch_stages(Q)>::bytes;
    cudaError_t e =
        cudaFuncSetAttribute(batch_step<Q, T, S, TYI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem[k]);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "batch attribute: %s", cudaGetErrorString(e));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_step<Q, T, S, TYI>, 32 * (TYI + 2), b->smem[k]);
    b->grid[k] = sms * std::max(per_sm, 1);
    return MRLBM_OK;
}

template <int Q, typename T, int S = 0>
mrlbm_status set_shapes(mrlbm_batch* b, int sms)
{
    mrlbm_status st = set_shape<Q, T, S, TYI_BULK>(b, sms);
    return st ? st : set_shape<Q, T, S, TYI_WALL>(b, sms);
}

template <int Q, typename T, int S = 0>
void launch(mrlbm_batch* b)
{
    const int k = tile_kind(b->rows);
    if (b->rows == TYI_BULK)
        batch_step<Q, T, S, TYI_BULK>
            <<<b->grid[k], 32 * (TYI_BULK + 2), b->smem[k], b->stream>>>(b->d_doms, b->d_items, b->d_ctl);
    else
        batch_step<Q, T, S, TYI_WALL>
            <<<b->grid[k], 32 * (TYI_WALL + 2), b->smem[k], b->stream>>>(b->d_doms, b->d_items, b->d_ctl);
}

void launch_any(mrlbm_batch* b)
{
    if (b->lattice == 19) {
        if (b->storage == MRLBM_F32) launch<19, float>(b);
        else if (b->storage == MRLBM_F16U) launch<19, __half, F_SPLITU>(b);
        else launch<19, __half>(b);
    } else {
        if (b->storage == MRLBM_F32) launch<27, float>(b);
        else if (b->storage == MRLBM_F16U) launch<27, __half, F_SPLITU>(b);
        else launch<27, __half>(b);
    }
}

int size_class(int nx, int ny, int nz)
{
    const int e = std::max(nx, std::max(ny, nz));
    if (e < 32) return 0;
    if (e < 48) return 1;
    if (e < 64) return 2;
    if (e < 96) return 3;
    if (e < 128) return 4;
    if (e < 192) return 5;
    return 6;
}

// switch the batch kernel's tile height (the captured graph holds the old
// launch shape; the next refresh rebuilds the work list for the new height)
void set_rows(mrlbm_batch* b, int rows)
{
    if (rows == b->rows) return;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->rows = rows;
}

int chunk_for(const mrlbm_batch* b, int nx, int ny, int nz)
{
    auto it = b->lz_by_class.find(size_class(nx, ny, nz));
    int lz = it != b->lz_by_class.end() ? it->second : 32;
    return std::max(1, std::min(lz, nz));
}

int batch_flags(const mrlbm_domain* dom)
{
    StepArgs a;
    int flags;
    fill_step_args(dom, a, 0, flags);
    if (flags & (F_FORCE | F_POWERLAW | F_BINGHAM)) flags |= F_BC;
    return flags;
}

bool flags_supported(int f)
{
    f &= ~F_SPLITU;  // every set below also with split-velocity storage
    return f == 0 || f == F_BC || f == (F_BC | F_FORCE) || f == (F_BC | F_FORCE | F_POWERLAW);
}

// Rebuild the per-domain records and the work list from the members; upload
// what changed.  Items are ordered by cost, largest first.
mrlbm_status refresh(mrlbm_batch* b)
{
    const int n = (int)b->members.size();
    if (n > b->dom_cap) {
        const int cap = std::max(2 * n, 64);
        BatchDomain* nd = nullptr;
        CK(cudaMalloc(&nd, cap * sizeof(BatchDomain)));
        cudaFree(b->d_doms);
        b->d_doms = nd;
        b->dom_cap = cap;
        b->h_doms.clear();
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    }
    std::vector<BatchDomain> hd(n);
    std::vector<BatchItem> items;
    for (int id = 0; id < n; id++) {
        memset(&hd[id], 0, sizeof(BatchDomain));
        mrlbm_domain* dom = b->members[id];
        if (!dom) continue;
        dom->lz = chunk_for(b, dom->d.nx, dom->d.ny, dom->d.nz);
        int f;
        for (int p = 0; p < 2; p++) fill_step_args(dom, hd[id].args[p], p, f);
        hd[id].flags = batch_flags(dom);
        if (!flags_supported(hd[id].flags))
            return fail(MRLBM_EINVAL, "batch member %d: physics flag set %d not supported in batches", id, hd[id].flags);
        if (dom->has_outflow)
            return fail(MRLBM_EINVAL, "batch member %d: outflow walls are not supported in batches", id);
        const int ty = batch_rows(b);
        hd[id].map[0] = dom->tmap[0][tile_kind(ty)];
        hd[id].map[1] = dom->tmap[1][tile_kind(ty)];
        hd[id].parity_offset = b->offsets[id];
        const int gx = (dom->d.nx + TILE_X - 1) / TILE_X, gy = (dom->d.ny + ty - 1) / ty;
        for (int z0 = 0; z0 < dom->d.nz; z0 += dom->lz)
            for (int by = 0; by < gy; by++)
                for (int bx = 0; bx < gx; bx++) items.push_back({id, bx * TILE_X, by * ty, z0});
    }
    std::stable_sort(items.begin(), items.end(), [&](const BatchItem& u, const BatchItem& v) {
        const mrlbm_domain* du = b->members[u.dom];
        const mrlbm_domain* dv = b->members[v.dom];
        const int cu = std::min(du->lz, du->d.nz - u.z0), cv = std::min(dv->lz, dv->d.nz - v.z0);
        return cu > cv;
    });
    if (b->h_doms.size() != hd.size() || memcmp(b->h_doms.data(), hd.data(), hd.size() * sizeof(BatchDomain)) != 0) {
        if (!hd.empty())
            CK(cudaMemcpyAsync(b->d_doms, hd.data(), hd.size() * sizeof(BatchDomain), cudaMemcpyHostToDevice, b->stream));
        b->h_doms = hd;
    }
    const int ni = (int)items.size();
    if (ni > b->item_cap) {
        const int cap = std::max(2 * ni, 1024);
        BatchItem* nitm = nullptr;
        CK(cudaMalloc(&nitm, cap * sizeof(BatchItem)));
        cudaFree(b->d_items);
        b->d_items = nitm;
        b->item_cap = cap;
        b->h_items.clear();
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    }
    if (b->h_items.size() != items.size() ||
        memcmp(b->h_items.data(), items.data(), items.size() * sizeof(BatchItem)) != 0) {
        if (ni) CK(cudaMemcpyAsync(b->d_items, items.data(), ni * sizeof(BatchItem), cudaMemcpyHostToDevice, b->stream));
        b->h_items = items;
    }
    if (ni != b->nitems) {
        CK(cudaMemcpyAsync(&b->d_ctl->nitems, &ni, sizeof(int), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));  // ni lives on the host stack
        b->nitems = ni;
    }
    return MRLBM_OK;
}

void advance_members(mrlbm_batch* b, int nsteps)
{
    b->step += nsteps;
    for (size_t id = 0; id < b->members.size(); id++) {
        mrlbm_domain* dom = b->members[id];
        if (!dom) continue;
        dom->cur = (int)((b->step + b->offsets[id]) & 1);
        dom->step += nsteps;
    }
}

mrlbm_status enqueue_steps(mrlbm_batch* b, int nsteps)
{
    if (b->nitems == 0) {
        advance_members(b, 0);
        return MRLBM_OK;
    }
    int left = nsteps;
    if (left >= GRAPH_STEPS) {
        if (!b->graph) {
            cudaGraph_t g;
            CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            for (int s = 0; s < GRAPH_STEPS; s++) launch_any(b);
            CK(cudaStreamEndCapture(b->stream, &g));
            CK(cudaGraphInstantiate(&b->graph, g, 0));
            cudaGraphDestroy(g);
        }
        while (left >= GRAPH_STEPS) {
            CK(cudaGraphLaunch(b->graph, b->stream));
            left -= GRAPH_STEPS;
        }
    }
    for (; left > 0; left--) launch_any(b);
    CK(cudaGetLastError());
    advance_members(b, nsteps);
    return MRLBM_OK;
}

mrlbm_status check_members(mrlbm_batch* b)
{
    for (mrlbm_domain* dom : b->members) {
        if (!dom) continue;
        mrlbm_status st = check_device_error(dom);
        if (st) return st;
    }
    return MRLBM_OK;
}

}  // namespace

extern "C" mrlbm_status mrlbm_batch_create(int lattice, int storage, mrlbm_batch** out)
{
    if (!out) return fail(MRLBM_EINVAL, "null output handle");
    *out = nullptr;
    if (lattice != 19 && lattice != 27) return fail(MRLBM_EINVAL, "lattice must be 19 or 27");
    if (storage != MRLBM_F32 && storage != MRLBM_F16 && storage != MRLBM_F16U)
        return fail(MRLBM_EINVAL, "batches store moments in fp32, fp16 or fp16 with split velocity");
    mrlbm_batch* b = new mrlbm_batch();
    b->lattice = lattice;
    b->storage = storage;
    b->rows = batch_tyi(lattice, storage == MRLBM_F16U ? F_SPLITU : 0);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    mrlbm_status st;
    if (lattice == 19)
        st = storage == MRLBM_F32    ? set_shapes<19, float>(b, sms)
             : storage == MRLBM_F16U ? set_shapes<19, __half, F_SPLITU>(b, sms)
                                     : set_shapes<19, __half>(b, sms);
    else
        st = storage == MRLBM_F32    ? set_shapes<27, float>(b, sms)
             : storage == MRLBM_F16U ? set_shapes<27, __half, F_SPLITU>(b, sms)
                                     : set_shapes<27, __half>(b, sms);
    if (st) { delete b; return st; }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMalloc(&b->d_ctl, sizeof(BatchCtl)) != cudaSuccess ||
        cudaMemset(b->d_ctl, 0, sizeof(BatchCtl)) != cudaSuccess) {
        mrlbm_batch_destroy(b);
        return fail(MRLBM_ECUDA, "batch setup failed");
    }
    *out = b;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_destroy(mrlbm_batch* b)
{
    if (!b) return MRLBM_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (mrlbm_domain* d : b->members)
        if (d) mrlbm_domain_destroy(d);
    cudaFree(b->d_doms);
    cudaFree(b->d_items);
    cudaFree(b->d_ctl);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_add(mrlbm_batch* b, const mrlbm_desc* desc, int* id)
{
    if (!b || !desc || !id) return fail(MRLBM_EINVAL, "null argument");
    if (desc->lattice != b->lattice || desc->storage != b->storage)
        return fail(MRLBM_EINVAL, "member lattice/storage must match the batch");
    mrlbm_domain* dom = nullptr;
    mrlbm_status st = mrlbm_domain_create(desc, &dom);
    if (st) return st;
    if (!flags_supported(batch_flags(dom))) {
        mrlbm_domain_destroy(dom);
        return fail(MRLBM_EINVAL, "physics of this domain are not supported in batches");
    }
    // reuse a free slot
    int slot = -1;
    for (size_t k = 0; k < b->members.size(); k++)
        if (!b->members[k]) { slot = (int)k; break; }
    if (slot < 0) {
        slot = (int)b->members.size();
        b->members.push_back(nullptr);
        b->offsets.push_back(0);
    }
    b->members[slot] = dom;
    b->offsets[slot] = (int)((dom->cur - b->step) & 1);
    *id = slot;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_remove(mrlbm_batch* b, int id)
{
    if (!b || id < 0 || id >= (int)b->members.size() || !b->members[id]) return fail(MRLBM_ENOTFOUND, "no member %d", id);
    CK(cudaStreamSynchronize(b->stream));
    mrlbm_domain_destroy(b->members[id]);
    b->members[id] = nullptr;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_domain(mrlbm_batch* b, int id, mrlbm_domain** dom)
{
    if (!b || !dom || id < 0 || id >= (int)b->members.size() || !b->members[id])
        return fail(MRLBM_ENOTFOUND, "no member %d", id);
    // work queued on the batch stream must finish before single-domain calls
    CK(cudaStreamSynchronize(b->stream));
    *dom = b->members[id];
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_step(mrlbm_batch* b, int nsteps)
{
    if (!b || nsteps < 0) return fail(MRLBM_EINVAL, "bad argument");
    // members may have been re-initialised through their domain handles
    for (size_t id = 0; id < b->members.size(); id++)
        if (b->members[id]) {
            CK(cudaStreamSynchronize(b->members[id]->stream));
            b->offsets[id] = (int)((b->members[id]->cur - b->step) & 1);
        }
    mrlbm_status st = refresh(b);
    if (st) return st;
    return enqueue_steps(b, nsteps);
}

extern "C" mrlbm_status mrlbm_batch_synchronize(mrlbm_batch* b)
{
    if (!b) return fail(MRLBM_EINVAL, "null batch");
    CK(cudaStreamSynchronize(b->stream));
    return check_members(b);
}

extern "C" mrlbm_status mrlbm_batch_time_steps(mrlbm_batch* b, int nsteps, float* ms)
{
    if (!b || !ms) return fail(MRLBM_EINVAL, "null argument");
    for (size_t id = 0; id < b->members.size(); id++)
        if (b->members[id]) {
            CK(cudaStreamSynchronize(b->members[id]->stream));
            b->offsets[id] = (int)((b->members[id]->cur - b->step) & 1);
        }
    mrlbm_status st = refresh(b);
    if (st) return st;
    CK(cudaEventRecord(b->ev0, b->stream));
    st = enqueue_steps(b, nsteps);
    if (st) return st;
    CK(cudaEventRecord(b->ev1, b->stream));
    CK(cudaEventSynchronize(b->ev1));
    CK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
    return check_members(b);
}

extern "C" mrlbm_status mrlbm_batch_info(mrlbm_batch* b, int* members, int* items, long long* nodes)
{
    if (!b) return fail(MRLBM_EINVAL, "null batch");
    int m = 0;
    long long nn = 0;
    for (mrlbm_domain* d : b->members)
        if (d) {
            m++;
            nn += (long long)d->d.nx * d->d.ny * d->d.nz;
        }
    mrlbm_status st = refresh(b);
    if (st) return st;
    if (members) *members = m;
    if (items) *items = b->nitems;
    if (nodes) *nodes = nn;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_chunk_for(mrlbm_batch* b, int nx, int ny, int nz, int* lz)
{
    if (!b || !lz) return fail(MRLBM_EINVAL, "null argument");
    *lz = chunk_for(b, nx, ny, nz);
    return MRLBM_OK;
}

// Coordinate search over the z-chunk length of each size class present, timing
// the whole batch: the chunk trades z-halo work (2 planes per chunk) against
// the number of work items available for load balance.
// Chunk autotuner.  It times candidate chunks on the members themselves, so it
// first copies every member's current moment buffer (ghost shell included)
// aside and afterwards copies it back and restores the step counters: the
// timed steps (an even number, so the buffer parities come back) leave no
// trace in any solve.
extern "C" mrlbm_status mrlbm_batch_set_rows(mrlbm_batch* b, int rows)
{
    if (!b) return fail(MRLBM_EINVAL, "null batch");
    if (rows != TYI_BULK && rows != TYI_WALL)
        return fail(MRLBM_EINVAL, "batch tile height %d: %d or %d rows", rows, TYI_BULK, TYI_WALL);
    CK(cudaStreamSynchronize(b->stream));
    set_rows(b, rows);
    return refresh(b);
}

extern "C" mrlbm_status mrlbm_batch_get_rows(mrlbm_batch* b, int* rows)
{
    if (!b || !rows) return fail(MRLBM_EINVAL, "null argument");
    *rows = b->rows;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_batch_autotune(mrlbm_batch* b)
{
    if (!b) return fail(MRLBM_EINVAL, "null batch");
    std::vector<int> classes;
    for (mrlbm_domain* d : b->members)
        if (d) {
            const int c = size_class(d->d.nx, d->d.ny, d->d.nz);
            if (std::find(classes.begin(), classes.end(), c) == classes.end()) classes.push_back(c);
        }
    // snapshot
    struct Saved {
        mrlbm_domain* dom;
        size_t bytes, off;
        int cur, step;
    };
    std::vector<Saved> saved;
    size_t total = 0;
    for (mrlbm_domain* d : b->members)
        if (d) {
            const size_t bytes = (size_t)d->field * (2 * ((d->nms + 1) / 2)) * d->esize;
            saved.push_back({d, bytes, total, d->cur, d->step});
            total += (bytes + 255) / 256 * 256;
        }
    const long long step0 = b->step;
    char* snap = nullptr;
    if (total) CK(cudaMalloc(&snap, total));
    for (const Saved& s : saved)
        CK(cudaMemcpyAsync(snap + s.off, s.dom->m[s.cur], s.bytes, cudaMemcpyDeviceToDevice, b->stream));

    static const int cand[] = {8, 16, 24, 32, 48, 64, 96};
    auto timed = [&](float* ms) -> mrlbm_status {
        mrlbm_status st = refresh(b);
        if (st) return st;
        st = enqueue_steps(b, 2);
        if (st) return st;
        CK(cudaEventRecord(b->ev0, b->stream));
        st = enqueue_steps(b, 6);
        if (st) return st;
        CK(cudaEventRecord(b->ev1, b->stream));
        CK(cudaEventSynchronize(b->ev1));
        CK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
        return MRLBM_OK;
    };
    // for each tile height: the z chunk per size class by coordinate
    // search, then the whole batch timed with those chunks; the faster
    // height and its chunks are kept
    mrlbm_status st = MRLBM_OK;
    const int rows0 = b->rows;
    int best_rows = rows0;
    float best_total = 1e30f;
    std::map<int, int> best_map = b->lz_by_class;
    for (int rows : {rows0, rows0 == TYI_BULK ? TYI_WALL : TYI_BULK}) {
        set_rows(b, rows);
        for (int c : classes) {
            float best = 1e30f;
            int best_lz = 32;
            for (int lz : cand) {
                b->lz_by_class[c] = lz;
                float ms = 0.f;
                if ((st = timed(&ms))) break;
                if (ms < best * 0.98f) {
                    best = ms;
                    best_lz = lz;
                }
            }
            b->lz_by_class[c] = best_lz;
            if (st) break;
        }
        if (st) break;
        float total = 0.f;
        if ((st = timed(&total))) break;
        // the starting height unless the other is 2 % faster
        if (rows == rows0 || total < best_total * 0.98f) {
            best_total = total;
            best_rows = rows;
            best_map = b->lz_by_class;
        }
    }
    set_rows(b, best_rows);
    b->lz_by_class = best_map;
    // restore the members and the step counters (the device counter too)
    cudaStreamSynchronize(b->stream);
    for (const Saved& s : saved) {
        cudaMemcpyAsync(s.dom->m[s.cur], snap + s.off, s.bytes, cudaMemcpyDeviceToDevice, b->stream);
        s.dom->cur = s.cur;
        s.dom->step = s.step;
    }
    b->step = step0;
    {
        const int dstep = (int)step0;
        cudaMemcpyAsync(&b->d_ctl->step, &dstep, sizeof(int), cudaMemcpyHostToDevice, b->stream);
    }
    cudaError_t e = cudaStreamSynchronize(b->stream);
    cudaFree(snap);
    if (st) return st;
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "autotune restore: %s", cudaGetErrorString(e));
    return refresh(b);
}
