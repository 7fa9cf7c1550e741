// zslab.cu -- caller streams and the z-slab plane exchange (include/mrlbm.h).
//
// A z slab is an ordinary domain, non-periodic in z, whose ghost planes
// z = -1 and z = nz hold its neighbours' boundary planes of the same step.
// In the padded pair layout (domain.h) one z plane of one moment pair is a
// contiguous block of 2 * plane elements, and the blocks of the pairs sit
// 2 * field elements apart, so a plane is npairs contiguous blocks: the
// exchange moves them as they lie (x/y ghost shell included, so the periodic
// x/y copies the step kernel wrote at the boundary planes travel with them and
// the corner ghosts of the receiver are right).
#include <dlfcn.h>
#include <nccl.h>

#include <mutex>

#include "domain.h"

using namespace mrlbm;

#define CK(call)                                                                                            \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            return fail(MRLBM_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

extern "C" mrlbm_status mrlbm_set_stream(mrlbm_domain* dom, void* stream)
{
    if (!dom) return fail(MRLBM_EINVAL, "null domain");
    cudaStream_t ns = stream ? static_cast<cudaStream_t>(stream) : dom->own_stream;
    if (ns == dom->stream) return MRLBM_OK;
    // what is queued on the old stream runs before anything queued on the new one
    CK(cudaEventRecord(dom->xev, dom->stream));
    CK(cudaStreamWaitEvent(ns, dom->xev, 0));
    dom->stream = ns;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_get_stream(mrlbm_domain* dom, void** stream)
{
    if (!dom || !stream) return fail(MRLBM_EINVAL, "null argument");
    *stream = dom->stream;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_zslab_plane(mrlbm_domain* dom, int which, mrlbm_zplane* out)
{
    if (!dom || !out) return fail(MRLBM_EINVAL, "null argument");
    const int nz = dom->d.nz;
    long long zp;  // padded z index (z + 1)
    switch (which) {
    case MRLBM_ZPLANE_FIRST: zp = 1; break;
    case MRLBM_ZPLANE_LAST: zp = nz; break;
    case MRLBM_ZGHOST_BELOW: zp = 0; break;
    case MRLBM_ZGHOST_ABOVE: zp = nz + 1; break;
    default: return fail(MRLBM_EINVAL, "bad plane selector %d", which);
    }
    const long long es = (long long)dom->esize;
    out->base = static_cast<char*>(dom->m[dom->cur]) + zp * dom->plane * 2 * es;
    out->pair_stride = dom->field * 2 * es;
    out->bytes = dom->plane * 2 * es;
    out->npairs = (dom->nms + 1) / 2;
    out->device = dom->device;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_zslab_copy(mrlbm_domain* src, int src_which, mrlbm_domain* dst, int dst_which)
{
    if (!src || !dst) return fail(MRLBM_EINVAL, "null domain");
    if (src_which != MRLBM_ZPLANE_FIRST && src_which != MRLBM_ZPLANE_LAST)
        return fail(MRLBM_EINVAL, "the source plane must be FIRST or LAST (got %d)", src_which);
    if (dst_which != MRLBM_ZGHOST_BELOW && dst_which != MRLBM_ZGHOST_ABOVE)
        return fail(MRLBM_EINVAL, "the destination plane must be a ghost plane (got %d)", dst_which);
    const mrlbm_desc &a = src->d, &b = dst->d;
    if (a.nx != b.nx || a.ny != b.ny || a.lattice != b.lattice || a.storage != b.storage || src->nm != dst->nm)
        return fail(MRLBM_EINVAL, "slabs differ in nx, ny, lattice, storage or moments (%dx%d q%d s%d nm%d vs "
                    "%dx%d q%d s%d nm%d)", a.nx, a.ny, a.lattice, a.storage, src->nm, b.nx, b.ny, b.lattice,
                    b.storage, dst->nm);
    mrlbm_zplane ps, pd;
    mrlbm_status st = mrlbm_zslab_plane(src, src_which, &ps);
    if (st) return st;
    if ((st = mrlbm_zslab_plane(dst, dst_which, &pd))) return st;
    const bool two = src->stream != dst->stream;
    if (two) {
        // the copy overwrites a plane dst's queued work may still read
        CK(cudaEventRecord(dst->xev, dst->stream));
        CK(cudaStreamWaitEvent(src->stream, dst->xev, 0));
    }
    // one strided copy of all pairs, or one copy per pair when the pair
    // stride is beyond the largest pitch a 2-D copy takes
    int maxpitch = 0;
    CK(cudaDeviceGetAttribute(&maxpitch, cudaDevAttrMaxPitch, src->device));
    if (ps.pair_stride <= maxpitch && pd.pair_stride <= maxpitch) {
        CK(cudaMemcpy2DAsync(pd.base, (size_t)pd.pair_stride, ps.base, (size_t)ps.pair_stride, (size_t)ps.bytes,
                             (size_t)ps.npairs, cudaMemcpyDefault, src->stream));
    } else {
        for (int p = 0; p < ps.npairs; p++)
            CK(cudaMemcpyAsync(static_cast<char*>(pd.base) + p * pd.pair_stride,
                               static_cast<const char*>(ps.base) + p * ps.pair_stride, (size_t)ps.bytes,
                               cudaMemcpyDefault, src->stream));
    }
    if (two) {
        CK(cudaEventRecord(src->xev, src->stream));
        CK(cudaStreamWaitEvent(dst->stream, src->xev, 0));
    }
    return MRLBM_OK;
}

// ------------------------------------------------ NCCL exchange (C/C++ callers)
//
// The z-slab exchange across processes without PyTorch: the library opens
// NCCL itself (libnccl.so.2, at the first call; no link-time dependency),
// makes communicators from a unique id the caller distributes, and queues
// each step's plane sends and receives on the domain's stream, in place
// (views of the library's buffers), so nothing waits on the host between
// steps and no kernel reads another GPU's memory.

namespace {

struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
    bool ok = false;
};

NcclApi* nccl_api()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        api.get_unique_id = (decltype(api.get_unique_id))dlsym(h, "ncclGetUniqueId");
        api.comm_init_rank = (decltype(api.comm_init_rank))dlsym(h, "ncclCommInitRank");
        api.comm_destroy = (decltype(api.comm_destroy))dlsym(h, "ncclCommDestroy");
        api.group_start = (decltype(api.group_start))dlsym(h, "ncclGroupStart");
        api.group_end = (decltype(api.group_end))dlsym(h, "ncclGroupEnd");
        api.send = (decltype(api.send))dlsym(h, "ncclSend");
        api.recv = (decltype(api.recv))dlsym(h, "ncclRecv");
        api.error_string = (decltype(api.error_string))dlsym(h, "ncclGetErrorString");
        api.ok = api.get_unique_id && api.comm_init_rank && api.comm_destroy && api.group_start && api.group_end &&
                 api.send && api.recv && api.error_string;
    });
    return api.ok ? &api : nullptr;
}

}  // namespace

#define NK(api, call)                                                                             \
    do {                                                                                          \
        ncclResult_t r_ = (call);                                                                 \
        if (r_ != ncclSuccess) return fail(MRLBM_ECUDA, "%s failed: %s", #call, (api)->error_string(r_)); \
    } while (0)

extern "C" mrlbm_status mrlbm_nccl_unique_id(void* id)
{
    if (!id) return fail(MRLBM_EINVAL, "null argument");
    NcclApi* api = nccl_api();
    if (!api) return fail(MRLBM_ECUDA, "NCCL (libnccl.so.2) could not be loaded");
    ncclUniqueId u;
    NK(api, api->get_unique_id(&u));
    memcpy(id, &u, sizeof(u));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_nccl_comm_init(int nranks, const void* id, int rank, void** comm)
{
    if (!id || !comm || nranks < 1 || rank < 0 || rank >= nranks) return fail(MRLBM_EINVAL, "bad argument");
    NcclApi* api = nccl_api();
    if (!api) return fail(MRLBM_ECUDA, "NCCL (libnccl.so.2) could not be loaded");
    ncclUniqueId u;
    memcpy(&u, id, sizeof(u));
    ncclComm_t c = nullptr;
    NK(api, api->comm_init_rank(&c, nranks, u, rank));
    *comm = c;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_nccl_comm_destroy(void* comm)
{
    if (!comm) return MRLBM_OK;
    NcclApi* api = nccl_api();
    if (!api) return fail(MRLBM_ECUDA, "NCCL (libnccl.so.2) could not be loaded");
    NK(api, api->comm_destroy(static_cast<ncclComm_t>(comm)));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_zslab_exchange_nccl(mrlbm_domain* dom, void* comm, int rank_below, int rank_above)
{
    if (!dom || !comm) return fail(MRLBM_EINVAL, "null argument");
    NcclApi* api = nccl_api();
    if (!api) return fail(MRLBM_ECUDA, "NCCL (libnccl.so.2) could not be loaded");
    mrlbm_zplane first, last, gbelow, gabove;
    mrlbm_status st;
    if ((st = mrlbm_zslab_plane(dom, MRLBM_ZPLANE_FIRST, &first)) || (st = mrlbm_zslab_plane(dom, MRLBM_ZPLANE_LAST, &last)) ||
        (st = mrlbm_zslab_plane(dom, MRLBM_ZGHOST_BELOW, &gbelow)) ||
        (st = mrlbm_zslab_plane(dom, MRLBM_ZGHOST_ABOVE, &gabove)))
        return st;
    ncclComm_t c = static_cast<ncclComm_t>(comm);
    cudaStream_t s = dom->stream;
    auto at = [](const mrlbm_zplane& p, int k) { return static_cast<char*>(p.base) + (size_t)k * p.pair_stride; };
    // the upward stream (last plane to the slab above, received there as its
    // ghost below) before the downward one, pair by pair, on every rank: the
    // k-th send from a to b meets the k-th receive at b from a, also when a
    // and b neighbour each other on both sides or a slab is its own neighbour
    NK(api, api->group_start());
    for (int k = 0; k < first.npairs; k++) {
        if (rank_above >= 0) NK(api, api->send(at(last, k), (size_t)last.bytes, ncclChar, rank_above, c, s));
        if (rank_below >= 0) NK(api, api->recv(at(gbelow, k), (size_t)gbelow.bytes, ncclChar, rank_below, c, s));
        if (rank_below >= 0) NK(api, api->send(at(first, k), (size_t)first.bytes, ncclChar, rank_below, c, s));
        if (rank_above >= 0) NK(api, api->recv(at(gabove, k), (size_t)gabove.bytes, ncclChar, rank_above, c, s));
    }
    NK(api, api->group_end());
    return MRLBM_OK;
}
