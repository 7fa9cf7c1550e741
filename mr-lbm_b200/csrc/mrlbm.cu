// mrlbm.cu -- C ABI (include/mrlbm.h) over the sm_100a MR-LBM kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "aux_kernels.cuh"
#include "domain.h"
#include "kernels.cuh"

using namespace mrlbm;

// ------------------------------------------------------------------ errors

static thread_local std::string g_err;

mrlbm_status mrlbm::fail(mrlbm_status st, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(MRLBM_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                 \
    } while (0)

extern "C" const char* mrlbm_last_error(void) { return g_err.c_str(); }
extern "C" const char* mrlbm_version(void) { return "mrlbm-b200 0.1 (sm_100a)"; }

extern "C" mrlbm_status mrlbm_set_device(int device)
{
    CK(cudaSetDevice(device));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_device_count(int* count)
{
    if (!count) return fail(MRLBM_EINVAL, "null argument");
    CK(cudaGetDeviceCount(count));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_host_alloc(size_t bytes, void** ptr)
{
    if (!ptr) return fail(MRLBM_EINVAL, "null argument");
    *ptr = nullptr;
    cudaError_t e = cudaMallocHost(ptr, bytes);
    if (e != cudaSuccess) return fail(MRLBM_ENOMEM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_host_free(void* ptr)
{
    if (ptr) CK(cudaFreeHost(ptr));
    return MRLBM_OK;
}

// ------------------------------------------------------- BC class building

// h_k(c) = c_a c_b - delta_ab/3 and g_k(c) = coefficient of Pi_k in 4.5 H(c):Pi
static void hg(int i, double* h, double* g)
{
    const double cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
    h[0] = cx * cx - 1.0 / 3.0; h[1] = cx * cy; h[2] = cx * cz;
    h[3] = cy * cy - 1.0 / 3.0; h[4] = cy * cz; h[5] = cz * cz - 1.0 / 3.0;
    g[0] = 4.5 * h[0]; g[1] = 9.0 * h[1]; g[2] = 9.0 * h[2];
    g[3] = 4.5 * h[3]; g[4] = 9.0 * h[4]; g[5] = 4.5 * h[5];
}

uint32_t mrlbm::known_mask(int q, uint32_t octants)
{
    uint32_t known = 0;
    for (int i = 0; i < q; i++) {
        const int d[3] = {-lat_cx(i), -lat_cy(i), -lat_cz(i)};
        bool all = true;
        for (int o = 0; o < 8 && all; o++) {
            const int s[3] = {(o & 1) ? 1 : -1, (o & 2) ? 1 : -1, (o & 4) ? 1 : -1};
            bool consistent = true;
            for (int k = 0; k < 3; k++)
                if (d[k] != 0 && d[k] != s[k]) consistent = false;
            if (consistent && !((octants >> o) & 1u)) all = false;
        }
        if (!all) known |= 1u << i;
    }
    return known;
}

static bool invert7(const double A[7][7], double inv[7][7])
{
    double M[7][14];
    for (int r = 0; r < 7; r++)
        for (int c = 0; c < 14; c++) M[r][c] = c < 7 ? A[r][c] : (c - 7 == r ? 1.0 : 0.0);
    for (int c = 0; c < 7; c++) {
        int best = c;
        for (int r = c + 1; r < 7; r++)
            if (std::fabs(M[r][c]) > std::fabs(M[best][c])) best = r;
        if (std::fabs(M[best][c]) < 1e-12) return false;
        if (best != c)
            for (int k = 0; k < 14; k++) std::swap(M[c][k], M[best][k]);
        const double p = M[c][c];
        for (int k = 0; k < 14; k++) M[c][k] /= p;
        for (int r = 0; r < 7; r++) {
            if (r == c || M[r][c] == 0.0) continue;
            const double f = M[r][c];
            for (int k = 0; k < 14; k++) M[r][k] -= f * M[c][k];
        }
    }
    for (int r = 0; r < 7; r++)
        for (int c = 0; c < 7; c++) inv[r][c] = M[r][c + 7];
    return true;
}

mrlbm_status mrlbm::build_bc_class(int q, int mq, uint32_t word, const double uvel[4][3], double omega0,
                                    BcClass* out)
{
    const uint32_t oct = word & 0xFFu;
    const uint32_t kind = (word >> 8) & 7u;
    const uint32_t vidx = (word >> 11) & 3u;
    if (kind > 2)
        return fail(MRLBM_EINVAL,
                    "node type 0x%x: BC kind %u not supported (no-slip and velocity walls, outflow)", word, kind);
    if (kind == 2) {
        // outflow: the kernel copies the inward neighbour's moments, no system
        memset(out, 0, sizeof(*out));
        out->known = known_mask(q, oct);
        out->valid = 1;
        out->word = word;
        return MRLBM_OK;
    }
    double u[3] = {0, 0, 0};
    if (kind == 1)
        for (int a = 0; a < 3; a++) u[a] = uvel[vidx][a];
    const uint32_t known = known_mask(q, oct);
    const double uu[6] = {u[0] * u[0], u[0] * u[1], u[0] * u[2], u[1] * u[1], u[1] * u[2], u[2] * u[2]};
    double A[7][7] = {};
    double a1 = 0.0, r[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < mq; i++) {
        if (!((known >> i) & 1u)) continue;
        const double w = lat_w(mq, i);
        double h[6], g[6];
        hg(i, h, g);
        const double cu = 3.0 * (lat_cx(i) * u[0] + lat_cy(i) * u[1] + lat_cz(i) * u[2]);
        double guu = 0.0;
        for (int k = 0; k < 6; k++) guu += g[k] * uu[k];
        A[0][0] += w * (1.0 + cu + omega0 * guu);
        a1 += w * guu;
        for (int k = 0; k < 6; k++) {
            A[0][1 + k] += (1.0 - omega0) * w * g[k];
            r[k] += w * g[k];
        }
        for (int rr = 0; rr < 6; rr++) {
            A[1 + rr][0] += w * h[rr] * (1.0 + cu);
            for (int k = 0; k < 6; k++) A[1 + rr][1 + k] += w * h[rr] * g[k];
        }
    }
    double inv[7][7];
    if (!invert7(A, inv))
        return fail(MRLBM_EINVAL, "node type 0x%x: singular moment-BC system at omega=%g", word, omega0);
    const double qv[7] = {a1, -r[0], -r[1], -r[2], -r[3], -r[4], -r[5]};
    double qa[7];
    for (int c = 0; c < 7; c++) {
        qa[c] = 0.0;
        for (int k = 0; k < 7; k++) qa[c] += qv[k] * inv[k][c];
    }
    memset(out, 0, sizeof(*out));
    for (int rr = 0; rr < 7; rr++)
        for (int c = 0; c < 7; c++) out->ainv[rr * 7 + c] = (float)inv[rr][c];
    for (int rr = 0; rr < 7; rr++) {
        out->v[rr] = (float)inv[rr][0];
        out->qa[rr] = (float)qa[rr];
    }
    out->s = (float)qa[0];
    for (int a = 0; a < 3; a++) out->u[a] = (float)u[a];
    out->known = known;
    out->valid = 1;
    out->word = word;
    return MRLBM_OK;
}

// ------------------------------------------------------------ domain setup

// moments a node carries (the reference's NUMBER_MOMENTS for the case) and
// the words it stores: with split-velocity storage three more, the low
// parts of 3u
static int moments_of(const mrlbm_desc& d)
{
    return (d.rheology != MRLBM_NEWTONIAN ? 11 : 10) + (d.thermal ? 4 : 0);
}
static int stored_moments_of(const mrlbm_desc& d)
{
    return moments_of(d) + (d.storage == MRLBM_F16U ? (d.rheology != MRLBM_NEWTONIAN ? 4 : 3) : 0);
}

// G_DIFF_FLUC_COEF from the thermal diffusivity with the reference's fixed
// T_DIFF_REF = 1/6 and G_TAU = 3 T_DIFF_REF + 1/2
// (src/cases/rayleighBenard_Periodic/constants.inc:58-65)
static double thermal_coef(double alpha)
{
    const double diff_ref = 1.0 / 6.0, g_tau = diff_ref * 3.0 + 0.5, g_omega = 1.0 / g_tau;
    const double aaa = 3.0 * (alpha - diff_ref) * g_omega;
    return aaa / (1.0 + aaa);
}

static size_t elem_size(int storage) { return storage == MRLBM_F32 ? 4 : 2; }

void mrlbm::storage_scales(int storage, int nm, float* scale, float* iscale)
{
    for (int k = 0; k < NM_MAX; k++) {
        float s = 1.0f;
        if (is_half_storage(storage)) {
            // powers of two keep values of the shifted moments in the normal
            // range of fp16 (exact, no rounding from the scaling itself);
            // bf16 has fp32's exponent range and needs none
            s = k == 0 ? 256.0f : (k <= 3 ? 8.0f : (k <= 9 ? 64.0f : 1.0f));
            // split storage: the low words of 3u and omega (stored after the
            // nm moments) are what the high word rounds away, at most half
            // an fp16 ulp of the scaled value, so 2^11 times the high word's
            // scale keeps them in fp16's normal range
            if (storage == MRLBM_F16U && k >= nm && k < nm + 3) s = 8.0f * 2048.0f;
            if (storage == MRLBM_F16U && nm == 11 && k == nm + 3) s = 2048.0f;
        }
        scale[k] = s;
        iscale[k] = 1.0f / s;
    }
}

static mrlbm_status validate(const mrlbm_desc* d)
{
    if (!d) return fail(MRLBM_EINVAL, "null descriptor");
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || d->nx > 8192 || d->ny > 8192 || d->nz > 8192)
        return fail(MRLBM_EINVAL, "bad grid %dx%dx%d", d->nx, d->ny, d->nz);
    if (d->lattice != 19 && d->lattice != 27) return fail(MRLBM_EINVAL, "lattice must be 19 or 27");
    if (d->storage < 0 || d->storage > 3) return fail(MRLBM_EINVAL, "bad storage %d", d->storage);
    if (!(d->tau > 0.5)) return fail(MRLBM_EINVAL, "tau must be > 0.5 (got %g)", d->tau);
    if (d->rheology < 0 || d->rheology > 2) return fail(MRLBM_EINVAL, "bad rheology");
    if (d->bc_matrix_q != 0 && d->bc_matrix_q != 19 && d->bc_matrix_q != d->lattice)
        return fail(MRLBM_EINVAL, "bc_matrix_q must be 0, 19 or the lattice size");
    {
        // the step kernel addresses a node within one moment's plane stack
        // with 32-bit offsets
        const long long pitch = (d->nx + XOFF + 1 + 7) / 8 * 8;
        const long long field = pitch * (d->ny + 2) * (long long)(d->nz + 2);
        if (field >= (1LL << 32))
            return fail(MRLBM_EINVAL, "domain %d x %d x %d: %lld padded nodes per moment, the limit is 2^32", d->nx,
                        d->ny, d->nz, field);
    }
    if (d->thermal != 0 && d->thermal != 1) return fail(MRLBM_EINVAL, "thermal must be 0 or 1");
    if (d->thermal) {
        // the second distribution's row exchange and ring fit next to the
        // D3Q19 flow's in shared memory; the reference's thermal cases are
        // D3Q19 Newtonian
        if (d->lattice != 19 || d->storage != MRLBM_F32 || d->rheology != MRLBM_NEWTONIAN)
            return fail(MRLBM_EINVAL, "the thermal scalar needs D3Q19, FP32 storage and a Newtonian fluid");
        if (d->storage == MRLBM_F16U) return fail(MRLBM_EINVAL, "split-velocity storage has no thermal scalar");
        if (!(d->t_diffusivity > 0.0) || !std::isfinite(thermal_coef(d->t_diffusivity)))
            return fail(MRLBM_EINVAL, "bad thermal diffusivity %g", d->t_diffusivity);
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_domain_bytes(const mrlbm_desc* d, size_t* bytes)
{
    mrlbm_status st = validate(d);
    if (st) return st;
    const size_t pitch = (size_t)((d->nx + XOFF + 1 + 7) / 8 * 8);
    const size_t field = pitch * (d->ny + 2) * (d->nz + 2);
    // two buffers of moment pairs (an odd count is padded to the next pair), node classes
    *bytes = 2 * field * (2 * ((stored_moments_of(*d) + 1) / 2)) * elem_size(d->storage) + field;
    return MRLBM_OK;
}

mrlbm_status mrlbm::domain_alloc(mrlbm_domain* dom)
{
    const mrlbm_desc& d = dom->d;
    dom->q = d.lattice;
    dom->nm = moments_of(d);
    dom->nms = stored_moments_of(d);
    dom->esize = elem_size(d.storage);
    dom->pitch = (d.nx + XOFF + 1 + 7) / 8 * 8;
    dom->plane = (long long)dom->pitch * (d.ny + 2);
    dom->field = dom->plane * (d.nz + 2);
    // the step kernel addresses a node within one moment's plane stack with
    // 32-bit offsets
    if (dom->field >= (1LL << 32))
        return fail(MRLBM_EINVAL, "domain %d x %d x %d: %lld padded nodes per moment, the limit is 2^32", d.nx, d.ny,
                    d.nz, dom->field);
    dom->omega0 = 1.0 / d.tau;
    storage_scales(d.storage, dom->nm, dom->scale, dom->iscale);
    // moment pairs: moments 2p and 2p + 1 interleaved per node (an odd count is padded)
    const size_t mbytes = (size_t)dom->field * (2 * ((dom->nms + 1) / 2)) * dom->esize;
    CK(cudaMalloc(&dom->m[0], mbytes));
    CK(cudaMalloc(&dom->m[1], mbytes));
    CK(cudaMemset(dom->m[0], 0, mbytes));
    CK(cudaMemset(dom->m[1], 0, mbytes));
    // exterior state: the reference's initial rest state (stale wall ghosts)
    float ext[NM_MAX];
    {
        const int qs = (d.lattice == 27) ? 19 : 19;
        double pxx = 0, pyy = 0, pzz = 0;
        for (int i = 0; i < qs; i++) {
            const double f = lat_w(d.lattice, i) * d.rho0;
            pxx += f * lat_cx(i) * lat_cx(i);
            pyy += f * lat_cy(i) * lat_cy(i);
            pzz += f * lat_cz(i) * lat_cz(i);
        }
        for (int k = 0; k < NM_MAX; k++) ext[k] = 0.f;
        ext[4] = (float)(4.5 * (pxx / d.rho0 - 1.0 / 3.0));
        ext[7] = (float)(4.5 * (pyy / d.rho0 - 1.0 / 3.0));
        ext[9] = (float)(4.5 * (pzz / d.rho0 - 1.0 / 3.0));
        // thermal: exterior C at the reference temperature, no flux
        if (d.thermal) ext[10] = (float)d.t_reference;
        else ext[10] = (float)dom->omega0;
        // split velocity: the exterior is at rest, its low words are zero
        for (int k = dom->nm; k < dom->nms; k++) ext[k] = 0.f;
    }
    memcpy(dom->ext, ext, sizeof(ext));
    CK(cudaStreamCreateWithFlags(&dom->stream, cudaStreamNonBlocking));
    dom->own_stream = dom->stream;
    CK(cudaGetDevice(&dom->device));
    CK(cudaEventCreate(&dom->ev0));
    CK(cudaEventCreate(&dom->ev1));
    CK(cudaEventCreateWithFlags(&dom->xev, cudaEventDisableTiming));
    CK(cudaMalloc(&dom->cls, (size_t)dom->field));
    CK(cudaMemset(dom->cls, 0, (size_t)dom->field));
    CK(cudaMalloc(&dom->err, sizeof(int)));
    CK(cudaMemset(dom->err, 0, sizeof(int)));
    {
        mrlbm_status st = make_tensor_maps(dom);
        if (st) return st;
    }
    CK(cudaMalloc(&dom->bc, sizeof(BcClass)));
    CK(cudaMemset(dom->bc, 0, sizeof(BcClass)));
    dom->red_blocks = 148 * 4;
    CK(cudaMalloc(&dom->red_scratch, (size_t)(dom->red_blocks * 8 + 8) * sizeof(double)));
    CK(cudaMallocHost(&dom->red_host, 8 * sizeof(double)));
    {
        int dev = 0, nsm = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        dom->nsm = nsm > 0 ? nsm : 148;
    }
    for (int k = 0; k < 2; k++) {
        dom->lz_t[k] = choose_lz(dom, tile_rows_of_kind(k));
        dom->lz_o[k] = choose_lz_overlap(dom, tile_rows_of_kind(k));
    }
    return MRLBM_OK;
}

// z planes per CTA.  A CTA (one per SM at a time) produces lz + 2 planes for
// lz outputs, and the grid runs in ceil(CTAs / SMs) waves, so the step time
// goes as waves * (lz + 2 + start-up): pick the chunk count that minimises it (the last
// wave full, few restarts).
int mrlbm::choose_lz(const mrlbm_domain* dom, int ty)
{
    const mrlbm_desc& d = dom->d;
    const long long cols = (long long)((d.nx + TILE_X - 1) / TILE_X) * ((d.ny + ty - 1) / ty);
    long long best_cost = -1;
    int best = d.nz;
    for (int nzc = 1; nzc <= d.nz; nzc++) {
        const int lz = (d.nz + nzc - 1) / nzc;
        const long long ctas = cols * ((d.nz + lz - 1) / lz);
        const long long slots = (long long)dom->nsm * ctas_per_sm(ty);
        const long long waves = (ctas + slots - 1) / slots;
        const long long cost = waves * (lz + 2 + 3);  // + a CTA start-up of about 3 planes
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = lz;
        }
    }
    return best;
}

// z planes per CTA when steps overlap (tile order): the end of a launch no
// longer idles SMs, so fewer, longer chunks save their start-up cost (two
// extra planes and the ring fill each).  Measured at 256^3 (D3Q19 and D3Q27
// vortex, D3Q19 cavity): 64 planes 2-3 % faster than 32, 86 and 128 slower;
// a grid under about three waves of CTAs loses the overlap (a 128^3 cavity
// ran 37.6 GLUPS at 32 planes, 20.9 at 64).  So: the longest chunk with at
// least 4 chunks a column and 3 waves of CTAs, if longer than the plain choice.
int mrlbm::choose_lz_overlap(const mrlbm_domain* dom, int ty)
{
    const mrlbm_desc& d = dom->d;
    const int plain = choose_lz(dom, ty);
    const long long cols = (long long)((d.nx + TILE_X - 1) / TILE_X) * ((d.ny + ty - 1) / ty);
    const long long slots = (long long)dom->nsm * ctas_per_sm(ty);
    for (int nzc = 4; nzc <= d.nz; nzc++) {
        const int lz = (d.nz + nzc - 1) / nzc;
        if (cols * ((d.nz + lz - 1) / lz) >= 3 * slots) return lz > plain ? lz : plain;
    }
    return plain;
}

bool mrlbm::tile_ordered(const mrlbm_domain* dom, int flags)
{
    return dom->tile_order && !(flags & (F_OUTFLOW | F_THERMAL));
}

extern "C" mrlbm_status mrlbm_domain_create(const mrlbm_desc* desc, mrlbm_domain** out)
{
    if (!out) return fail(MRLBM_EINVAL, "null output handle");
    *out = nullptr;
    mrlbm_status st = validate(desc);
    if (st) return st;
    mrlbm_domain* dom = new mrlbm_domain();
    dom->d = *desc;
    if (dom->d.bc_matrix_q == 0) dom->d.bc_matrix_q = 19;
    if (dom->d.rheology == MRLBM_POWERLAW && dom->d.nnf_k == 0.0)
        dom->d.nnf_k = dom->d.rho0 * (dom->d.tau - 0.5) / 3.0;
    if (dom->d.rheology == MRLBM_BINGHAM && dom->d.nnf_omega_p == 0.0) dom->d.nnf_omega_p = 1.0 / dom->d.tau;
    st = domain_alloc(dom);
    if (st) {
        mrlbm_domain_destroy(dom);
        return st;
    }
    *out = dom;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_domain_destroy(mrlbm_domain* dom)
{
    if (!dom) return MRLBM_OK;
    if (dom->graph_exec) cudaGraphExecDestroy(dom->graph_exec);
    if (dom->stream) cudaStreamSynchronize(dom->stream);
    cudaFree(dom->m[0]);
    cudaFree(dom->m[1]);
    cudaFree(dom->cls);
    cudaFree(dom->err);
    cudaFree(dom->sched);
    cudaFree(dom->bc);
    cudaFree(dom->red_scratch);
    cudaFree(dom->usnap);
    cudaFree(dom->stage);
    if (dom->red_host) cudaFreeHost(dom->red_host);
    if (dom->ev0) cudaEventDestroy(dom->ev0);
    if (dom->ev1) cudaEventDestroy(dom->ev1);
    if (dom->xev) cudaEventDestroy(dom->xev);
    if (dom->own_stream) cudaStreamDestroy(dom->own_stream);
    delete dom;
    return MRLBM_OK;
}

// Wall normal of a face node: the axis whose whole + or - half of the octant
// mask is solid, when exactly one such (axis, side) exists; axis 3 otherwise.
// Stored in the class with its BC kind (outflow and the thermal rules act
// along it).
static mrlbm_status class_normal(uint32_t word, BcClass* c)
{
    const uint32_t oct = word & 0xFFu, kind = (word >> 8) & 7u;
    int axis = 3, side = 0, nfaces = 0;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++) {
            bool all = true;
            for (int o = 0; o < 8; o++)
                if ((((o >> a) & 1) == sd) && !((oct >> o) & 1u)) all = false;
            if (all) { axis = a; side = sd; nfaces++; }
        }
    if (nfaces != 1) axis = 3;
    if (kind == 2 && axis == 3)
        return fail(MRLBM_EINVAL, "node type 0x%x: outflow needs a face node (one solid half)", word);
    c->trule = ((uint32_t)axis << 2) | ((uint32_t)side << 4) | (kind << 8);
    return MRLBM_OK;
}

// Thermal rule of a class (bits 13-16 of its word, include/mrlbm.h
// MRLBM_THERMAL_*): rules 2 and 3 act along the class's wall normal.
static mrlbm_status thermal_rule_of(uint32_t word, const double t_wall[4], BcClass* c)
{
    const uint32_t rule = (word >> 13) & 3u, idx = (word >> 15) & 3u;
    if ((rule == 2 || rule == 3) && ((c->trule >> 2) & 3u) == 3u)
        return fail(MRLBM_EINVAL, "node type 0x%x: thermal rule %u needs a face node (one solid half)", word, rule);
    c->trule |= rule;
    c->twall = (float)t_wall[idx];
    return MRLBM_OK;
}

mrlbm_status mrlbm::classify_nodes(int q, int mq, const uint32_t* nt, long long n, const double uvel[4][3],
                                   double omega0, std::vector<uint8_t>& cls, std::vector<BcClass>& table,
                                   bool& any_bc, bool case_mode, const double* t_wall)
{
    std::map<uint32_t, int> ids;
    table.assign(1, BcClass{});  // class 0: bulk (unused entry)
    cls.resize(n);
    any_bc = false;
    for (long long k = 0; k < n; k++) {
        const uint32_t w = nt[k];
        // run-time classes key on the octant mask, BC kind and velocity index;
        // case mode hands the whole word to the case's own snippet (like the
        // reference: bulk iff the word is BULK, solid iff it is 0xFF)
        const bool bulk = case_mode ? w == 0u : (w & 0xFFu) == 0u;
        const bool solid = case_mode ? w == 0xFFu : (w & 0xFFu) == 0xFFu;
        if (bulk) { cls[k] = CLS_BULK; continue; }
        any_bc = true;
        if (solid) { cls[k] = CLS_SOLID; continue; }
        // (thermal domains also key on the thermal rule and value index)
        const uint32_t key = case_mode ? w : (w & (t_wall ? 0x1FFFFu : 0x1FFFu));
        auto it = ids.find(key);
        if (it == ids.end()) {
            if ((int)table.size() >= 255) return fail(MRLBM_EINVAL, "more than 254 distinct boundary node types");
            BcClass c;
            memset(&c, 0, sizeof(c));
            c.word = key;
            mrlbm_status st = case_mode ? MRLBM_OK : build_bc_class(q, mq, key & 0x1FFFu, uvel, omega0, &c);
            if (st) return st;
            c.word = key;
            if (!case_mode && (st = class_normal(key, &c))) return st;
            if (t_wall && !case_mode && (st = thermal_rule_of(key, t_wall, &c))) return st;
            const int id = (int)table.size();
            table.push_back(c);
            it = ids.emplace(key, id).first;
        }
        cls[k] = (uint8_t)it->second;
    }
    return MRLBM_OK;
}

static mrlbm_status set_node_types_impl(mrlbm_domain* dom, const uint32_t* nt, bool case_mode)
{
    if (!dom || !nt) return fail(MRLBM_EINVAL, "null argument");
    const mrlbm_desc& d = dom->d;
    const long long n = (long long)d.nx * d.ny * d.nz;
    std::vector<uint8_t> cls;
    std::vector<BcClass> table;
    bool any = false;
    mrlbm_status st =
        classify_nodes(dom->q, d.bc_matrix_q, nt, n, d.bc_velocity, dom->omega0, cls, table, any, case_mode,
                       d.thermal ? d.t_wall : nullptr);
    if (st) return st;
    bool outflow = false;
    for (const BcClass& c : table)
        if (!case_mode && ((c.word >> 8) & 7u) == 2u) outflow = true;
    if (outflow && (d.rheology != MRLBM_NEWTONIAN || d.thermal))
        return fail(MRLBM_EINVAL, "outflow walls are supported for Newtonian domains without the thermal scalar");
    // scatter into the padded plane layout
    std::vector<uint8_t> padded((size_t)dom->field, 0);
    for (int z = 0; z < d.nz; z++)
        for (int y = 0; y < d.ny; y++)
            memcpy(&padded[(size_t)pidx(0, y, z, dom->pitch, dom->plane)], &cls[((size_t)z * d.ny + y) * d.nx], d.nx);
    CK(cudaMemcpyAsync(dom->cls, padded.data(), padded.size(), cudaMemcpyHostToDevice, dom->stream));
    cudaFree(dom->bc);
    dom->bc = nullptr;
    CK(cudaMalloc(&dom->bc, table.size() * sizeof(BcClass)));
    CK(cudaMemcpyAsync(dom->bc, table.data(), table.size() * sizeof(BcClass), cudaMemcpyHostToDevice, dom->stream));
    CK(cudaStreamSynchronize(dom->stream));
    dom->has_bc = any;
    dom->has_outflow = outflow;
    dom->nclasses = (int)table.size();
    if (dom->graph_exec) { cudaGraphExecDestroy(dom->graph_exec); dom->graph_exec = nullptr; }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_set_node_types(mrlbm_domain* dom, const uint32_t* nt)
{
    return set_node_types_impl(dom, nt, false);
}

extern "C" mrlbm_status mrlbm_set_node_types_case(mrlbm_domain* dom, const uint32_t* nt)
{
    return set_node_types_impl(dom, nt, true);
}

// ------------------------------------------------------------------- init

template <int Q>
static void launch_init(mrlbm_domain* dom, InitArgs& a)
{
    const int threads = 256;
    const long long n = (long long)dom->d.nx * dom->d.ny * dom->d.nz;
    int blocks = (int)std::min<long long>((n + threads - 1) / threads, 148LL * 32);
    if (dom->d.storage == MRLBM_F32)
        init_kernel<Q, float><<<blocks, threads, 0, dom->stream>>>(a);
    else if (is_half_storage(dom->d.storage))
        init_kernel<Q, __half><<<blocks, threads, 0, dom->stream>>>(a);
    else
        init_kernel<Q, __nv_bfloat16><<<blocks, threads, 0, dom->stream>>>(a);
}

static mrlbm_status run_init(mrlbm_domain* dom, InitArgs& a)
{
    const mrlbm_desc& d = dom->d;
    a.m0 = dom->m[0];
    a.m1 = dom->m[1];
    a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.pitch = dom->pitch;
    a.plane = dom->plane; a.field = dom->field;
    a.nm = dom->nms;
    a.lo0 = dom->nms > dom->nm ? dom->nm : -1;
    a.lom = dom->nms - dom->nm == 4 ? dom->nm + 3 : -1;
    a.qs = 19;  // the reference's D3Q19 second-moment sums (also on D3Q27)
    a.rho0 = (float)d.rho0;
    a.omega0 = (float)dom->omega0;
    a.thermal = d.thermal;
    a.c0 = (float)d.t_reference;
    memcpy(a.scale, dom->scale, sizeof(a.scale));
    if (d.lattice == 19) launch_init<19>(dom, a); else launch_init<27>(dom, a);
    CK(cudaGetLastError());
    {
        mrlbm_status st = fill_ghosts(dom);
        if (st) return st;
    }
    CK(cudaStreamSynchronize(dom->stream));
    dom->cur = 0;
    dom->step = 0;
    dom->have_snap = false;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_init_flow(mrlbm_domain* dom, const float* rho, const float* ux, const float* uy,
                                         const float* uz)
{
    if (!dom || !rho || !ux || !uy || !uz) return fail(MRLBM_EINVAL, "null argument");
    const size_t n = (size_t)dom->d.nx * dom->d.ny * dom->d.nz;
    float* dbuf = nullptr;
    CK(cudaMalloc(&dbuf, 4 * n * sizeof(float)));
    const float* src[4] = {rho, ux, uy, uz};
    for (int k = 0; k < 4; k++) {
        cudaError_t e = cudaMemcpyAsync(dbuf + k * n, src[k], n * sizeof(float), cudaMemcpyHostToDevice, dom->stream);
        if (e != cudaSuccess) { cudaFree(dbuf); return fail(MRLBM_ECUDA, "copy: %s", cudaGetErrorString(e)); }
    }
    InitArgs a{};
    a.kind = 0;
    a.rho = dbuf; a.ux = dbuf + n; a.uy = dbuf + 2 * n; a.uz = dbuf + 3 * n;
    mrlbm_status st = run_init(dom, a);
    cudaFree(dbuf);
    return st;
}

extern "C" mrlbm_status mrlbm_init_uniform(mrlbm_domain* dom, const double u0[3])
{
    if (!dom) return fail(MRLBM_EINVAL, "null domain");
    InitArgs a{};
    a.kind = 1;
    for (int k = 0; k < 3; k++) a.u0[k] = u0 ? (float)u0[k] : 0.f;
    return run_init(dom, a);
}

extern "C" mrlbm_status mrlbm_init_taylor_green(mrlbm_domain* dom, double u0, double L)
{
    if (!dom || !(L > 0)) return fail(MRLBM_EINVAL, "bad argument");
    InitArgs a{};
    a.kind = 2;
    a.tg_u0 = (float)u0;
    a.tg_L = (float)L;
    return run_init(dom, a);
}

// ------------------------------------------------------------------- step

void mrlbm::fill_step_args(const mrlbm_domain* dom, StepArgs& a, int parity, int& flags)
{
    const mrlbm_desc& d = dom->d;
    a.m_out = dom->m[parity ^ 1];
    a.m_in = dom->m[parity];
    a.storage = d.storage;
    for (int p = 0; p < (NM_MAX + 1) / 2; p++)
        a.out_p[p] = 2 * p < dom->nms ? static_cast<char*>(dom->m[parity ^ 1]) + (size_t)p * 2 * dom->field * dom->esize
                                     : nullptr;
    a.err = dom->err;
    a.sched = nullptr;
    a.cls = dom->cls;
    a.bc = dom->bc;
    a.nbc = dom->nclasses;
    a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.pitch = dom->pitch;
    a.plane = dom->plane; a.field = dom->field;
    a.periodic = (d.periodic[0] ? 1 : 0) | (d.periodic[1] ? 2 : 0) | (d.periodic[2] ? 4 : 0);
    a.step = dom->step;
    a.rho0 = (float)d.rho0;
    a.omega0 = (float)dom->omega0;
    a.fx = (float)d.force[0]; a.fy = (float)d.force[1]; a.fz = (float)d.force[2];
    a.nnf_n = (float)d.nnf_n; a.nnf_k = (float)d.nnf_k;
    a.nnf_yield = (float)d.nnf_yield; a.nnf_omega_p = (float)d.nnf_omega_p;
    a.t_coef = d.thermal ? (float)thermal_coef(d.t_diffusivity) : 0.f;
    a.t_ref = (float)d.t_reference;
    for (int k = 0; k < 3; k++) a.t_gb[k] = (float)(d.t_gravity_beta[k] * d.rho0);
    a.t_src = (float)d.t_source;
    memcpy(a.scale, dom->scale, sizeof(a.scale));
    memcpy(a.iscale, dom->iscale, sizeof(a.iscale));
    flags = 0;
    if (dom->has_bc && dom->cls) flags |= F_BC;
    if (d.force[0] != 0.0 || d.force[1] != 0.0 || d.force[2] != 0.0) flags |= F_FORCE;
    if (d.rheology == MRLBM_POWERLAW) flags |= F_POWERLAW;
    if (d.rheology == MRLBM_BINGHAM) flags |= F_BINGHAM;
    if (flags & (F_POWERLAW | F_BINGHAM)) flags |= F_BC;  // nnf variants always read the class map
    if (d.thermal) flags |= F_THERMAL | F_FORCE;           // the Boussinesq force is per node
    if (dom->has_outflow) flags |= F_OUTFLOW;
    if (d.storage == MRLBM_F16U) flags |= F_SPLITU;
    const int kind = tile_kind(tile_rows(flags));
    a.lz = dom->lz > 0 ? dom->lz : tile_ordered(dom, flags) ? dom->lz_o[kind] : dom->lz_t[kind];
}

// Tile-ordered steps (zmarch_step, tile_order_begin): the state is sized and
// zeroed for the step's grid, on stream s, whenever the grid changes.  Flag
// sets whose wall rules read the previous moments through the read-only
// cache (outflow, thermal) keep whole-grid ordering: that cache is only
// coherent across launches that do not overlap.  Returns whether the step
// is tile-ordered and sets the state's grid.
static bool tile_order_state(mrlbm_domain* dom, const StepArgs& a, int flags, cudaStream_t s, bool& reset,
                             mrlbm_status& st)
{
    st = MRLBM_OK;
    reset = false;
    if (!tile_ordered(dom, flags)) return false;
    const dim3 g = zmarch_grid(a.nx, a.ny, a.nz, tile_rows(flags), a.lz);
    const long long key = ((long long)g.z << 42) | ((long long)g.y << 21) | (long long)g.x;
    if (key == dom->sched_key) return true;
    if (dom->graph_exec) {  // its launches carry the old state
        cudaStreamSynchronize(s);
        cudaGraphExecDestroy(dom->graph_exec);
        dom->graph_exec = nullptr;
    }
    const size_t words = 2 + (size_t)g.x * g.y * g.z;
    if (words > dom->sched_words) {
        if (dom->sched) {
            cudaStreamSynchronize(s);
            cudaFree(dom->sched);
            dom->sched = nullptr;
            dom->sched_words = 0;
        }
        cudaError_t e = cudaMalloc(&dom->sched, words * sizeof(unsigned));
        if (e != cudaSuccess) {
            st = fail(MRLBM_ECUDA, "tile-order state: %s", cudaGetErrorString(e));
            return false;
        }
        dom->sched_words = words;
    }
    cudaError_t e = cudaMemsetAsync(dom->sched, 0, words * sizeof(unsigned), s);
    if (e != cudaSuccess) {
        st = fail(MRLBM_ECUDA, "tile-order state: %s", cudaGetErrorString(e));
        return false;
    }
    dom->sched_key = key;
    reset = true;
    return true;
}

mrlbm_status mrlbm::prepare_tile_order(mrlbm_domain* dom, cudaStream_t s)
{
    StepArgs a;
    int flags;
    fill_step_args(dom, a, dom->cur, flags);
    bool reset;
    mrlbm_status st;
    (void)tile_order_state(dom, a, flags, s, reset, st);
    return st;
}

mrlbm_status mrlbm::enqueue_step(mrlbm_domain* dom, int parity, cudaStream_t s, bool chained)
{
    StepArgs a;
    int flags;
    fill_step_args(dom, a, parity, flags);
    bool reset;
    mrlbm_status st;
    if (tile_order_state(dom, a, flags, s, reset, st)) a.sched = dom->sched;
    if (st) return st;
    // a zeroed state follows a memset on the stream: no overlap with it
    const bool pdl = a.sched && chained && !reset;
    const int q = dom->q;
    const int stg = dom->d.storage;
    const CUtensorMap* maps = dom->tmap[parity];
    if (q == 19) {
        if (stg == MRLBM_F32) st = dispatch_step<19, float>(maps, a, flags, s, pdl);
        else if (is_half_storage(stg)) st = dispatch_step<19, __half>(maps, a, flags, s, pdl);
        else st = dispatch_step<19, __nv_bfloat16>(maps, a, flags, s, pdl);
    } else {
        if (stg == MRLBM_F32) st = dispatch_step<27, float>(maps, a, flags, s, pdl);
        else if (is_half_storage(stg)) st = dispatch_step<27, __half>(maps, a, flags, s, pdl);
        else st = dispatch_step<27, __nv_bfloat16>(maps, a, flags, s, pdl);
    }
    return st;
}

extern "C" mrlbm_status mrlbm_step(mrlbm_domain* dom, int nsteps)
{
    if (!dom || nsteps < 0) return fail(MRLBM_EINVAL, "bad argument");
    for (int s = 0; s < nsteps; s++) {
        // launches after the first follow this call's own step on the stream
        mrlbm_status st = enqueue_step(dom, dom->cur, dom->stream, s > 0);
        if (st) return st;
        dom->cur ^= 1;
        dom->step++;
    }
    CK(cudaGetLastError());
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_step_graph(mrlbm_domain* dom, int nsteps)
{
    if (!dom || nsteps < 0) return fail(MRLBM_EINVAL, "bad argument");
    if (nsteps == 0) return MRLBM_OK;
    // One graph of GRAPH_STEPS launches starting from parity 0 (an even count,
    // so replays chain); an odd leading step or a short remainder runs eagerly.
    if (!dom->graph_exec) {
        // the tile-order state is set up outside the capture (a replay must
        // not zero it); the captured launches order whole grids
        mrlbm_status pst = prepare_tile_order(dom, dom->stream);
        if (pst) return pst;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(dom->stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < GRAPH_STEPS; s++) {
            mrlbm_status st = enqueue_step(dom, s & 1, dom->stream, false);
            if (st) {
                cudaStreamEndCapture(dom->stream, &g);
                if (g) cudaGraphDestroy(g);
                return st;
            }
        }
        CK(cudaStreamEndCapture(dom->stream, &g));
        CK(cudaGraphInstantiate(&dom->graph_exec, g, 0));
        cudaGraphDestroy(g);
    }
    int left = nsteps;
    if (dom->cur != 0) {
        mrlbm_status st = mrlbm_step(dom, 1);
        if (st) return st;
        left--;
    }
    while (left >= GRAPH_STEPS) {
        CK(cudaGraphLaunch(dom->graph_exec, dom->stream));
        dom->step += GRAPH_STEPS;
        left -= GRAPH_STEPS;
    }
    if (left > 0) return mrlbm_step(dom, left);
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_time_steps(mrlbm_domain* dom, int nsteps, float* ms)
{
    if (!dom || !ms) return fail(MRLBM_EINVAL, "null argument");
    CK(cudaEventRecord(dom->ev0, dom->stream));
    mrlbm_status st = mrlbm_step(dom, nsteps);
    if (st) return st;
    CK(cudaEventRecord(dom->ev1, dom->stream));
    CK(cudaEventSynchronize(dom->ev1));
    CK(cudaEventElapsedTime(ms, dom->ev0, dom->ev1));
    return check_device_error(dom);
}

mrlbm_status mrlbm::check_device_error(mrlbm_domain* dom)
{
    int h = 0;
    CK(cudaMemcpyAsync(&h, dom->err, sizeof(int), cudaMemcpyDeviceToHost, dom->stream));
    CK(cudaStreamSynchronize(dom->stream));
    if (h) {
        CK(cudaMemsetAsync(dom->err, 0, sizeof(int), dom->stream));
        if (h & 2)
            return fail(MRLBM_EBOUNDS, "a step kernel skipped an out-of-range access (flag 0x%x: kinds 0x%x)", h,
                        (h >> 8) & 0xff);
        return fail(MRLBM_ETIMEDOUT,
                    "a step kernel gave up waiting for its tile loads or for the previous step's tiles (flag 0x%x)",
                    h);
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_synchronize(mrlbm_domain* dom)
{
    if (!dom) return fail(MRLBM_EINVAL, "null domain");
    CK(cudaStreamSynchronize(dom->stream));
    return check_device_error(dom);
}

// Self-test of the bounded waits: one CTA waits on an mbarrier whose single
// expected arrival never comes, gives up after `polls` polls, raises the
// error flag the step kernels raise, and exits; the host reads the flag.
__global__ void bounded_wait_selftest_kernel(int* err, unsigned polls)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const bool ok = mbar_wait(&bar, 0u, polls);
    if (!ok && threadIdx.x == 0) atomicOr(err, 1);
}

extern "C" mrlbm_status mrlbm_selftest_bounded_wait(unsigned polls, double* seconds)
{
    if (polls == 0 || polls > WAIT_LIMIT) return fail(MRLBM_EINVAL, "polls must be in 1..%u", WAIT_LIMIT);
    int* d_err = nullptr;
    CK(cudaMalloc(&d_err, sizeof(int)));
    cudaError_t e = cudaMemset(d_err, 0, sizeof(int));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    int h = 0;
    float ms = 0.f;
    if (e == cudaSuccess) {
        cudaEventRecord(t0);
        bounded_wait_selftest_kernel<<<1, 32>>>(d_err, polls);
        cudaEventRecord(t1);
        e = cudaEventSynchronize(t1);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(d_err);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "bounded-wait self-test: %s", cudaGetErrorString(e));
    if (seconds) *seconds = ms * 1e-3;
    if (h) return fail(MRLBM_ETIMEDOUT, "bounded-wait self-test: the wait gave up after %u polls (%.3f s)", polls,
                       ms * 1e-3);
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_get_step(mrlbm_domain* dom, int* step)
{
    if (!dom || !step) return fail(MRLBM_EINVAL, "null argument");
    *step = dom->step;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_set_z_chunk(mrlbm_domain* dom, int lz)
{
    if (!dom) return fail(MRLBM_EINVAL, "null argument");
    if (lz < 0 || lz > dom->d.nz) return fail(MRLBM_EINVAL, "z chunk %d outside 0..%d", lz, dom->d.nz);
    if (dom->graph_exec) {
        cudaGraphExecDestroy(dom->graph_exec);  // the captured launches carry the old chunk
        dom->graph_exec = nullptr;
    }
    dom->lz = lz;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_set_tile_order(mrlbm_domain* dom, int on)
{
    if (!dom) return fail(MRLBM_EINVAL, "null argument");
    if (on != 0 && on != 1) return fail(MRLBM_EINVAL, "tile order %d is not 0 or 1", on);
    dom->tile_order = on != 0;
    if (dom->graph_exec) {  // the captured launches carry the old setting
        cudaStreamSynchronize(dom->stream);
        cudaGraphExecDestroy(dom->graph_exec);
        dom->graph_exec = nullptr;
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_get_z_chunk(mrlbm_domain* dom, int* lz)
{
    if (!dom || !lz) return fail(MRLBM_EINVAL, "null argument");
    StepArgs a;
    int flags = 0;
    fill_step_args(dom, a, dom->cur, flags);
    *lz = a.lz;
    return MRLBM_OK;
}

// ------------------------------------------------------------ conversions

static mrlbm_status convert(mrlbm_domain* dom, float* hbuf_out, const float* hbuf_in, int mode)
{
    const mrlbm_desc& d = dom->d;
    if ((mode == 2 || mode == 3) && (d.nx % 8 || d.ny % 8 || d.nz % 8))
        return fail(MRLBM_EINVAL, "reference layout needs nx, ny, nz multiples of 8");
    const size_t n = (size_t)d.nx * d.ny * d.nz * dom->nm;
    if (!dom->stage) CK(cudaMalloc(&dom->stage, n * sizeof(float)));
    float* dbuf = dom->stage;
    if (mode == 1 || mode == 3)
        CK(cudaMemcpyAsync(dbuf, hbuf_in, n * sizeof(float), cudaMemcpyHostToDevice, dom->stream));
    ConvArgs a{};
    a.m0 = dom->m[dom->cur];
    a.m1 = dom->m[dom->cur ^ 1];
    a.f = dbuf;
    a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.pitch = dom->pitch;
    a.plane = dom->plane; a.field = dom->field;
    a.nm = dom->nm;
    a.lo0 = dom->nms > dom->nm ? dom->nm : -1;
    a.lom = dom->nms - dom->nm == 4 ? dom->nm + 3 : -1;
    a.mode = mode;
    memcpy(a.scale, dom->scale, sizeof(a.scale));
    memcpy(a.iscale, dom->iscale, sizeof(a.iscale));
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 64);
    if (d.storage == MRLBM_F32) convert_kernel<float><<<blocks, threads, 0, dom->stream>>>(a);
    else if (is_half_storage(d.storage)) convert_kernel<__half><<<blocks, threads, 0, dom->stream>>>(a);
    else convert_kernel<__nv_bfloat16><<<blocks, threads, 0, dom->stream>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && (mode == 0 || mode == 2))
        e = cudaMemcpyAsync(hbuf_out, dbuf, n * sizeof(float), cudaMemcpyDeviceToHost, dom->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(dom->stream);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "convert: %s", cudaGetErrorString(e));
    if (mode == 1 || mode == 3) {
        dom->have_snap = false;
        mrlbm_status st = fill_ghosts(dom);
        if (st) return st;
        CK(cudaStreamSynchronize(dom->stream));
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_num_moments(mrlbm_domain* dom, int* nm)
{
    if (!dom || !nm) return fail(MRLBM_EINVAL, "null argument");
    *nm = dom->nm;
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_get_moments(mrlbm_domain* dom, float* m)
{
    if (!dom || !m) return fail(MRLBM_EINVAL, "null argument");
    return convert(dom, m, nullptr, 0);
}
extern "C" mrlbm_status mrlbm_set_moments(mrlbm_domain* dom, const float* m)
{
    if (!dom || !m) return fail(MRLBM_EINVAL, "null argument");
    return convert(dom, nullptr, m, 1);
}
extern "C" mrlbm_status mrlbm_get_moments_ref_layout(mrlbm_domain* dom, float* m)
{
    if (!dom || !m) return fail(MRLBM_EINVAL, "null argument");
    return convert(dom, m, nullptr, 2);
}
extern "C" mrlbm_status mrlbm_set_moments_ref_layout(mrlbm_domain* dom, const float* m)
{
    if (!dom || !m) return fail(MRLBM_EINVAL, "null argument");
    return convert(dom, nullptr, m, 3);
}

extern "C" mrlbm_status mrlbm_get_macr(mrlbm_domain* dom, float* rho, float* ux, float* uy, float* uz, float* omega)
{
    if (!dom) return fail(MRLBM_EINVAL, "null domain");
    const mrlbm_desc& d = dom->d;
    const size_t n = (size_t)d.nx * d.ny * d.nz;
    std::vector<float> all(n * dom->nm);
    mrlbm_status st = convert(dom, all.data(), nullptr, 0);
    if (st) return st;
    if (rho)
        for (size_t k = 0; k < n; k++) rho[k] = (float)d.rho0 + all[k];
    if (ux) memcpy(ux, &all[n], n * sizeof(float));
    if (uy) memcpy(uy, &all[2 * n], n * sizeof(float));
    if (uz) memcpy(uz, &all[3 * n], n * sizeof(float));
    if (omega) {
        if (d.rheology == MRLBM_NEWTONIAN) return fail(MRLBM_EINVAL, "domain has no omega field");
        memcpy(omega, &all[10 * n], n * sizeof(float));
    }
    return MRLBM_OK;
}

// ------------------------------------------------------- TMA tensor maps

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// 4-D maps over each padded moment buffer with dimension order (x and pair
// element, moment pair, y, z) so that a box of (2 * box width, pairs, rows + 2,
// 1) lands in shared memory as [row][pair][x][2]: one plane of a CTA column
// and its two outer rows per copy; one map per tile height.
mrlbm_status mrlbm::make_tensor_maps(mrlbm_domain* dom)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return fail(MRLBM_ECUDA, "cuTensorMapEncodeTiled unavailable");
    const mrlbm_desc& d = dom->d;
    const CUtensorMapDataType dt = d.storage == MRLBM_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : is_half_storage(d.storage) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                            : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const cuuint64_t es = dom->esize;
    // x runs over the interleaved pair elements (2 per node), the second
    // dimension over moment pairs
    const cuuint32_t npairs = (cuuint32_t)((dom->nms + 1) / 2);
    const cuuint64_t dims[4] = {(cuuint64_t)(2 * dom->pitch), npairs, (cuuint64_t)(d.ny + 2), (cuuint64_t)(d.nz + 2)};
    const cuuint64_t strides[3] = {(cuuint64_t)(2 * dom->field) * es, (cuuint64_t)(2 * dom->pitch) * es,
                                   (cuuint64_t)(2 * dom->plane) * es};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    for (int k = 0; k < 2; k++) {
        const cuuint32_t box[4] = {(cuuint32_t)(2 * box_x_nodes((int)es)), npairs,
                                   (cuuint32_t)(tile_rows_of_kind(k) + 2), 1};
        for (int b = 0; b < 2; b++) {
            CUresult r = enc(&dom->tmap[b][k], dt, 4, dom->m[b], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return fail(MRLBM_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
        }
    }
    return MRLBM_OK;
}

mrlbm_status mrlbm::fill_ghosts(mrlbm_domain* dom)
{
    const mrlbm_desc& d = dom->d;
    GhostArgs g{};
    g.m0 = dom->m[0];
    g.m1 = dom->m[1];
    g.nx = d.nx; g.ny = d.ny; g.nz = d.nz; g.pitch = dom->pitch;
    g.plane = dom->plane; g.field = dom->field;
    g.nm = dom->nms;
    g.periodic = (d.periodic[0] ? 1 : 0) | (d.periodic[1] ? 2 : 0) | (d.periodic[2] ? 4 : 0);
    memcpy(g.ext, dom->ext, sizeof(g.ext));
    memcpy(g.scale, dom->scale, sizeof(g.scale));
    const long long n = (long long)(d.nx + 2) * (d.ny + 2) * (d.nz + 2);
    const int threads = 256;
    const int blocks = (int)std::min<long long>((n + threads - 1) / threads, 148LL * 16);
    // the copy reads buffer 0 and writes both: buffer 0 must be the current state
    if (dom->cur != 0) {
        g.m0 = dom->m[1];
        g.m1 = dom->m[0];
    }
    if (d.storage == MRLBM_F32) ghost_fill_kernel<float><<<blocks, threads, 0, dom->stream>>>(g);
    else if (is_half_storage(d.storage)) ghost_fill_kernel<__half><<<blocks, threads, 0, dom->stream>>>(g);
    else ghost_fill_kernel<__nv_bfloat16><<<blocks, threads, 0, dom->stream>>>(g);
    CK(cudaGetLastError());
    return MRLBM_OK;
}

// ------------------------------------------------------------- reductions

mrlbm_status mrlbm::enqueue_reduce(mrlbm_domain* dom, double* partial, double* out, int residual_mode,
                                   cudaStream_t s)
{
    const mrlbm_desc& d = dom->d;
    RedArgs a{};
    a.m = dom->m[dom->cur];
    a.cls = dom->cls;
    a.has_cls = dom->has_bc && dom->cls;
    a.nx = d.nx; a.ny = d.ny; a.nz = d.nz; a.pitch = dom->pitch;
    a.plane = dom->plane; a.field = dom->field;
    a.nm = dom->nm;
    a.lo0 = dom->nms > dom->nm ? dom->nm : -1;
    a.rho0 = (float)d.rho0;
    memcpy(a.iscale, dom->iscale, sizeof(a.iscale));
    a.partial = partial;
    a.out = out;
    a.nblocks = dom->red_blocks;
    a.usnap = dom->usnap;
    a.residual_mode = residual_mode;
    if (d.storage == MRLBM_F32) reduce_kernel<float><<<a.nblocks, RED_THREADS, 0, s>>>(a);
    else if (is_half_storage(d.storage)) reduce_kernel<__half><<<a.nblocks, RED_THREADS, 0, s>>>(a);
    else reduce_kernel<__nv_bfloat16><<<a.nblocks, RED_THREADS, 0, s>>>(a);
    reduce_finish<<<1, 32, 0, s>>>(partial, a.nblocks, out);
    CK(cudaGetLastError());
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_reduce_fp64(mrlbm_domain* dom, mrlbm_sums* out)
{
    if (!dom || !out) return fail(MRLBM_EINVAL, "null argument");
    double* partial = dom->red_scratch;
    double* res = dom->red_scratch + dom->red_blocks * 8;
    mrlbm_status st = enqueue_reduce(dom, partial, res, 0, dom->stream);
    if (st) return st;
    CK(cudaMemcpyAsync(dom->red_host, res, 8 * sizeof(double), cudaMemcpyDeviceToHost, dom->stream));
    CK(cudaStreamSynchronize(dom->stream));
    const double* h = dom->red_host;
    out->mass = h[0];
    out->momentum[0] = h[1]; out->momentum[1] = h[2]; out->momentum[2] = h[3];
    out->kinetic_energy = h[4];
    out->fluid_nodes = h[5];
    out->max_speed = h[6];
    out->nonfinite = h[7];
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_residual(mrlbm_domain* dom, double* residual)
{
    if (!dom || !residual) return fail(MRLBM_EINVAL, "null argument");
    const size_t n = (size_t)dom->d.nx * dom->d.ny * dom->d.nz;
    if (!dom->usnap) CK(cudaMalloc(&dom->usnap, 3 * n * sizeof(float)));
    double* partial = dom->red_scratch;
    double* res = dom->red_scratch + dom->red_blocks * 8;
    const int mode = dom->have_snap ? 1 : 2;
    mrlbm_status st = enqueue_reduce(dom, partial, res, mode, dom->stream);
    if (st) return st;
    CK(cudaMemcpyAsync(dom->red_host, res, 8 * sizeof(double), cudaMemcpyDeviceToHost, dom->stream));
    CK(cudaStreamSynchronize(dom->stream));
    if (mode == 2) {
        dom->have_snap = true;
        *residual = 1.0;
    } else {
        *residual = std::sqrt(dom->red_host[0]) / (std::sqrt(dom->red_host[1]) + 1e-30);
    }
    return MRLBM_OK;
}
