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
