// kernels.cuh -- device code of the fused MR-LBM collide-stream step.
//
// One step of the moment-representation LBM (the reference's
// gpuMomCollisionStream, src/mlbm.cu:3-714) computes, for every fluid node x,
//   f_i*(x) = f_i^post(x - c_i)   with f^post reconstructed from the stored
//                                 post-collision moments of the source node,
// then the new moments (bulk sums, or the moment-space wall BC), and collides
// them in moment space.  Only the 10 moments (11 with an omega field, 14 with
// the thermal scalar C and its flux) live in HBM.
//
// B200 design (z-marching, ping-pong moments, TMA-fed):
//   * Moments are stored in pairs (moments 2p and 2p + 1 side by side per
//     node, so a node's pair is one 8-byte word in FP32) as padded plane
//     stacks with a one-node ghost shell (x = -1..nx, y = -1..ny,
//     z = -1..nz): half the load and store instructions of one plane stack
//     per moment.  Periodic axes keep
//     the shell equal to the wrapped interior: the kernel writes the extra
//     copies of boundary nodes.  Wall axes keep the shell at the exterior rest
//     state.  So every halo read is an in-bounds tile read with no wrap logic.
//   * A CTA owns a column of 30 x TYI interior nodes in (x, y) and a chunk of
//     LZ planes in z.  Warp w holds row y = Y0 - 1 + w, lane l holds
//     x = X0 - 1 + l: the outer lanes / warps are the one-node halo.
//   * One elected thread streams the planes of the column into a 4-stage
//     shared-memory ring with cp.async.bulk.tensor (TMA) and mbarrier
//     transaction counts; the waits are bounded and a timeout makes every
//     thread leave together with an error flag set.
//   * Each production step reconstructs the post-collision populations of
//     every node of one plane in registers.  Populations that move in x only
//     go through warp shuffles, populations that move in y through a
//     double-buffered shared-memory row exchange packed by (c_x, c_y) into
//     128-bit words (one __syncthreads per plane), populations that move in z
//     stay in registers: a plane's c_z=+1 populations are held until the next
//     plane, its c_z=0 ones until the output of the same plane is formed one
//     step later.  Output plane z is completed when plane z+1 is produced.
//     A pipeline step holds the consumption of plane k-1 and the production
//     of plane k between plain per-plane barriers; they are independent, and
//     their order in the source only steers the compiler's schedule.
//   * The thermal scalar (D3G19) rides the same pipeline with a second row
//     exchange; outflow walls read the inward neighbour from the buffer the
//     step reads (kernel variants launched only for domains that have them).
//   * DRAM traffic is the algorithmic 2*M*s bytes per node; halo re-reads of
//     neighbouring columns hit L2.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <type_traits>

#include "lattice.cuh"

namespace mrlbm {

enum : int {
    F_BC = 1,        // node classes present (walls, solids, velocity BCs)
    F_FORCE = 2,     // non-zero body force
    F_POWERLAW = 4,  // omega field, power-law viscosity
    F_BINGHAM = 8,   // omega field, Bingham viscosity
    F_THERMAL = 16,  // thermal scalar C on D3G19 (4 more stored moments, Boussinesq force)
    F_OUTFLOW = 32,  // some wall class is an outflow (selects the OutflowBC policy at launch)
    F_SPLITU = 64,   // 16-bit storage with each velocity component split in a high and a low word
};

// most stored moments per node: 10 flow moments + omega, or + C and its flux
// (split-velocity fp16 storage of a non-Newtonian flow: 11 moments + 4 low words)
constexpr int NM_MAX = 15;

// CTA geometry: 32 x TYI interior nodes of an (x, y) column (warp w < TYI is
// row y = Y0 + w, lane l is x = X0 + l) plus two helper warps that produce
// what crosses into the column from outside it.
constexpr int TILE_X = 32;   // interior nodes per row (one per lane)
constexpr int XOFF = 4;      // padded column of x = 0 (x = -1 is the ghost column)
// TMA box width in nodes: covers x = X0 - 1 .. X0 + 32 from a 16-byte
// aligned start (X0 - 2 for FP32 pairs, X0 - 4 for 16-bit pairs)
template <typename T>
__host__ __device__ constexpr int box_x()
{
    return sizeof(T) == 4 ? 36 : 40;
}
__host__ __device__ constexpr int box_x_nodes(int esize) { return esize == 4 ? 36 : 40; }
// TMA ring depth: 4 stages where the ring and the row exchange fit in shared
// memory (4 measured 1-3 % faster than 3), else 3 (or 2)
constexpr int NSTAGE_MAX = 4;
// interior rows per CTA: 8 (two CTAs of 10 warps per SM, up to 102 registers
// a thread) for every flow-only set, walls and non-Newtonian viscosity
// included; 14 (one CTA of 16 warps, up to 128 registers) for the thermal
// sets, whose second population pipeline needs them
constexpr int TYI_BULK = 8, TYI_WALL = 14;
__host__ __device__ constexpr int tile_rows(int flags)
{
    return (flags & F_THERMAL) ? TYI_WALL : TYI_BULK;
}
// CTAs resident per SM: two for short columns (their per-plane barriers
// interleave, which measured 2-3 % faster for 8 rows than one CTA of 16), else one
__host__ __device__ constexpr int ctas_per_sm(int tyi) { return tyi <= 8 ? 2 : 1; }
// dynamic shared memory a CTA may take: the opt-in per-block limit for one
// CTA per SM, else an even share of the SM's 228 KB less the 1 KB each
// block reserves
__host__ __device__ constexpr size_t smem_budget(int tyi)
{
    return ctas_per_sm(tyi) == 1 ? 232448 : 233472 / ctas_per_sm(tyi) - 1024;
}
// stored moments and moment pairs of a flag set
__host__ __device__ constexpr int nmoments_of(int flags)
{
    return ((flags & (F_POWERLAW | F_BINGHAM)) ? 11 : 10) + ((flags & F_THERMAL) ? 4 : 0) +
           ((flags & F_SPLITU) ? ((flags & (F_POWERLAW | F_BINGHAM)) ? 4 : 3) : 0);
}
__host__ __device__ constexpr int npairs_of(int flags) { return (nmoments_of(flags) + 1) / 2; }
// index of a tile height among the domain's tensor maps and z chunks
__host__ __device__ constexpr int tile_kind(int tyi) { return tyi == TYI_BULK ? 0 : 1; }
__host__ __device__ constexpr int tile_rows_of_kind(int kind) { return kind == 0 ? TYI_BULK : TYI_WALL; }
constexpr uint8_t CLS_BULK = 0;
constexpr uint8_t CLS_SOLID = 255;
constexpr unsigned WAIT_LIMIT = 1u << 26;  // mbarrier polls before giving up (~seconds)
constexpr unsigned DEP_LIMIT = 1u << 21;   // tile-order polls (an L2 round trip + 64 ns each, ~seconds)

// Bounds-check build (-DMRLBM_BOUNDS_CHECK, libmrlbm_check.so): every
// shared-memory access of the step kernels is checked against the CTA's
// regions (TMA ring, row exchanges, edge buffers), every global store and
// node-class load against the padded field, before it happens; a bad access
// is skipped and sets bit 1 of the device error word (bits 8-15: which kind
// of access).  The exchange and edge buffers are also refilled with NaN after
// every consumption (and at the start of a column), so a slot that a
// consumption reads but the production before it did not write shows up as
// NaN in the moments.  The default build has none of it.
enum : int { BCK_STAGE = 1, BCK_EXCHANGE = 2, BCK_EDGE = 4, BCK_STORE = 8, BCK_CLASS = 16 };
#ifdef MRLBM_BOUNDS_CHECK
struct SmemBounds {
    unsigned stage_lo, stage_hi, ex_lo, ex_hi, edge_lo, edge_hi;
    int* err;
};
__shared__ SmemBounds g_bounds;
__device__ __forceinline__ bool bounds_fail(int kind, int* err)
{
    atomicOr(err, 2 | (kind << 8));
    return false;
}
__device__ __forceinline__ bool smem_ok(const void* p, int bytes, int kind)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    unsigned lo, hi;
    if (kind == BCK_STAGE) { lo = g_bounds.stage_lo; hi = g_bounds.stage_hi; }
    else if (kind == BCK_EXCHANGE) { lo = g_bounds.ex_lo; hi = g_bounds.ex_hi; }
    else { lo = g_bounds.edge_lo; hi = g_bounds.edge_hi; }
    return (a >= lo && a + (unsigned)bytes <= hi) ? true : bounds_fail(kind, g_bounds.err);
}
#define MRLBM_SMEM_OK(p, bytes, kind) smem_ok((p), (bytes), (kind))
#define MRLBM_GLOBAL_OK(cond, kind, err) ((cond) ? true : bounds_fail((kind), (err)))
#else
#define MRLBM_SMEM_OK(p, bytes, kind) true
#define MRLBM_GLOBAL_OK(cond, kind, err) true
#endif

// Moment-space wall BC data of one node class (octant mask + velocity index).
// The BC is the linear system
//   sum_I f_i          = sum_I f^reg_i(rho, u, (1-w) Pi + w u u)
//   sum_I f_i h_k(c_i) = sum_I h_k(c_i) f^reg_i(rho, u, Pi)
// in X = (rho, rho*Pi).  Its matrix is A(w) = A(w0) + (w - w0) e0 q^T, so the
// host stores Ainv = A(w0)^-1, v = Ainv e0, qa = q^T Ainv, s = q^T Ainv e0 and
// the device applies Sherman-Morrison for a per-node omega.
// 72 words, 16-byte aligned, so the kernel can read a class with vector loads.
struct alignas(16) BcClass {
    float ainv[49];
    float v[7];
    float qa[7];
    float s;
    float u[3];        // prescribed wall velocity (unscaled)
    uint32_t known;    // bit i: population i is known (incoming from fluid)
    uint32_t valid;
    uint32_t word;     // the node-type word of the class (nodeTypeMap encoding)
    uint32_t trule;    // thermal rule (bits 0-1), wall normal axis (bits 2-3, 3 = none),
                       // solid side of the normal (bit 4: + side), BC kind (bits 8-10)
    float twall;       // thermal wall value
};
static_assert(sizeof(BcClass) == 288, "BcClass is read as float4 words");

struct StepArgs {
    void* __restrict__ m_out;         // padded planes [nm][nz+2][ny+2][pitch]
    void* out_p[(NM_MAX + 1) / 2];    // plane stack of moment pair p (moments 2p, 2p+1)
    const void* m_in;                 // the buffer being read (outflow and thermal wall rules read it)
    int storage;                      // its element type (mrlbm_storage)
    const uint8_t* __restrict__ cls;  // padded [nz+2][ny+2][pitch]
    const BcClass* __restrict__ bc;
    int* err;                         // bit 0: a bounded wait timed out; bit 2: a tile-order wait did
    unsigned* sched;                  // null, or the tile-order state of the single-domain step (zmarch_step)
    int nx, ny, nz, pitch;
    long long plane, field;  // elements
    int periodic;            // bit a set: axis a periodic
    int lz;                  // planes per CTA / per batch work item
    int step;                // step number (read by case-mode boundary snippets)
    float rho0, omega0;
    float fx, fy, fz;
    float nnf_n, nnf_k, nnf_yield, nnf_omega_p;
    float t_coef;      // thermal: G_DIFF_FLUC_COEF
    float t_ref;       // thermal: T_REFERENCE
    float t_gb[3];     // thermal: t_gravity_beta * rho0
    float t_src;       // thermal: source added to C at bulk nodes
    float scale[NM_MAX];   // storage scale per moment (1 for fp32)
    float iscale[NM_MAX];
    int nbc;           // classes in the table bc
};

__host__ __device__ __forceinline__ long long pidx(int x, int y, int z, int pitch, long long plane)
{
    return (long long)(z + 1) * plane + (long long)(y + 1) * pitch + (x + XOFF);
}

// Element of moment m at padded node offset idx (pidx): moment pairs are
// stacked 2 * field elements apart, the pair's two moments side by side.
__host__ __device__ __forceinline__ long long mphys(int m, long long idx, long long field)
{
    return (long long)(m >> 1) * 2 * field + 2 * idx + (m & 1);
}

// ------------------------------------------------------------------ storage

template <typename T>
struct Stor;
template <>
struct Stor<float> {
    static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ float lds(const float* p) { return *p; }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
template <>
struct Stor<__half> {
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float lds(const __half* p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
};
template <>
struct Stor<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    static __device__ __forceinline__ float lds(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

template <typename T>
constexpr bool is_f32()
{
    return sizeof(T) == 4;
}

// FP16 storage carries power-of-two scales per moment (the shifted moments
// would otherwise fall into its subnormal range); BF16 has FP32's exponent
// range and is stored unscaled, so its loads and stores skip the multiplies.
template <typename T>
constexpr bool scaled_storage()
{
    return std::is_same<T, __half>::value;
}

// a moment pair of one node: 8 bytes (FP32) or 4 bytes (FP16 / BF16)
template <typename T>
struct Stor2;
template <>
struct Stor2<float> {
    static __device__ __forceinline__ float2 lds(const float* p) { return *reinterpret_cast<const float2*>(p); }
    static __device__ __forceinline__ void st(float* p, float a, float b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
};
template <>
struct Stor2<__half> {
    static __device__ __forceinline__ float2 lds(const __half* p)
    {
        return __half22float2(*reinterpret_cast<const __half2*>(p));
    }
    static __device__ __forceinline__ void st(__half* p, float a, float b)
    {
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
    }
};
template <>
struct Stor2<__nv_bfloat16> {
    static __device__ __forceinline__ float2 lds(const __nv_bfloat16* p)
    {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
    }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float a, float b)
    {
        *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(a, b);
    }
};

// ------------------------------------------------------------ per-node math

// Post-collision populations from stored scaled moments (reconstruction of the
// regularized Hermite-2 distribution, src/colrec/MR_LBM/reconstruction.inc:1-35),
// evaluated pairwise: f_i = rw (A_i + B_i), f_ibar = rw (A_i - B_i) with A the
// even (second-moment) part and B = c_i . 3u.
__device__ __forceinline__ void rc_pair(float* f, int i, float rw, float A, float B)
{
    float a = rw * A;
    f[i] = fmaf(rw, B, a);
    f[i + 1] = fmaf(-rw, B, a);
}

template <int Q>
__device__ __forceinline__ void reconstruct(const float* m, float rho0, float* f)
{
    const float rho = rho0 + m[0];
    const float ux = m[1], uy = m[2], uz = m[3];
    const float mxx = m[4], mxy = m[5], mxz = m[6], myy = m[7], myz = m[8], mzz = m[9];
    const float pics2 = 1.0f - (mxx + myy + mzz) * (1.0f / 3.0f);
    constexpr float W0 = (float)lat_w(Q, 0), W1 = (float)lat_w(Q, 1), W2 = (float)lat_w(Q, 7);
    const float rw1 = rho * W1, rw2 = rho * W2;
    f[0] = rho * W0 * pics2;
    const float ax = pics2 + mxx, ay = pics2 + myy, az = pics2 + mzz;
    rc_pair(f, 1, rw1, ax, ux);
    rc_pair(f, 3, rw1, ay, uy);
    rc_pair(f, 5, rw1, az, uz);
    const float pxy = ax + myy, pxz = ax + mzz, pyz = ay + mzz;
    rc_pair(f, 7, rw2, pxy + mxy, ux + uy);
    rc_pair(f, 9, rw2, pxz + mxz, ux + uz);
    rc_pair(f, 11, rw2, pyz + myz, uy + uz);
    rc_pair(f, 13, rw2, pxy - mxy, ux - uy);
    rc_pair(f, 15, rw2, pxz - mxz, ux - uz);
    rc_pair(f, 17, rw2, pyz - myz, uy - uz);
    if constexpr (Q == 27) {
        constexpr float W3 = (float)lat_w(27, 19);
        const float rw3 = rho * W3;
        const float t = pxy + mzz;
        const float s1 = mxy + mxz, s2 = mxy - mxz;
        const float uxy = ux + uy, uxmy = ux - uy;
        rc_pair(f, 19, rw3, t + s1 + myz, uxy + uz);    // ( 1, 1, 1)
        rc_pair(f, 21, rw3, t + s2 - myz, uxy - uz);    // ( 1, 1,-1)
        rc_pair(f, 23, rw3, t - s2 - myz, uxmy + uz);   // ( 1,-1, 1)
        rc_pair(f, 25, rw3, t - s1 + myz, uz - uxmy);   // (-1, 1, 1)
    }
}

// Raw sums over the lattice: rho, j, and sum f c_a c_b (xx, xy, xz, yy, yz,
// zz), as a tensor product.  Reduce along z first (per (c_x, c_y): the
// zeroth, first and second z moments), then along y and x, keeping only the
// per-axis orders that moments up to second order need: 66 additions for
// D3Q27 and 42 for D3Q19, against 111 and 63 summing opposite pairs.
template <int Q>
__host__ __device__ __forceinline__ void lattice_sums(const float* p, float& r, float* j, float* P)
{
    // S*[X + 3Y] with X = c_x + 1, Y = c_y + 1
    float S0[9], S1[9], S2[9];
    static_for<0, 9>([&](auto C) {
        constexpr int X = C % 3, Y = C / 3;
        constexpr int i0 = lat_find(Q, X - 1, Y - 1, 0);
        constexpr int ip = lat_find(Q, X - 1, Y - 1, 1), im = lat_find(Q, X - 1, Y - 1, -1);
        if constexpr (ip < 0) {   // D3Q19 (c_x, c_y) corners carry c_z = 0 only
            S0[C] = p[i0];
            S1[C] = 0.f;
            S2[C] = 0.f;
        } else {
            const float a = p[ip] + p[im];
            S0[C] = a + p[i0];
            S1[C] = p[ip] - p[im];
            S2[C] = a;
        }
    });
    // T<ay><az>[X]: y order ay, z order az, per c_x
    float T00[3], T10[3], T20[3], T01[3], T11[3], T02[3];
    static_for<0, 3>([&](auto XX) {
        constexpr int X = XX;
        const float a0 = S0[X + 6] + S0[X];
        T00[X] = a0 + S0[X + 3];
        T10[X] = S0[X + 6] - S0[X];
        T20[X] = a0;
        if constexpr (Q == 27 || X == 1) {
            const float a1 = S1[X + 6] + S1[X];
            T01[X] = a1 + S1[X + 3];
            T11[X] = S1[X + 6] - S1[X];
            T02[X] = S2[X + 6] + S2[X] + S2[X + 3];
        } else {
            T01[X] = S1[X + 3];
            T11[X] = 0.f;
            T02[X] = S2[X + 3];
        }
    });
    const float b = T00[2] + T00[0];
    r = b + T00[1];
    j[0] = T00[2] - T00[0];
    j[1] = T10[0] + T10[1] + T10[2];
    j[2] = T01[0] + T01[1] + T01[2];
    P[0] = b;
    P[1] = T10[2] - T10[0];
    P[2] = T01[2] - T01[0];
    P[3] = T20[0] + T20[1] + T20[2];
    P[4] = Q == 27 ? T11[0] + T11[1] + T11[2] : T11[1];
    P[5] = T02[0] + T02[1] + T02[2];
}

// Right-hand side of the wall system: sums of the known populations
// (b0 and the traceless second-moment sums).
template <int Q>
__device__ __forceinline__ void bc_known_sums(uint32_t known, const float* p, float* b)
{
    float b0 = 0.f, sxx = 0.f, sxy = 0.f, sxz = 0.f, syy = 0.f, syz = 0.f, szz = 0.f;
    static_for<0, Q>([&](auto I) {
        constexpr int i = I;
        constexpr int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        const float v = ((known >> i) & 1u) ? p[i] : 0.f;
        b0 += v;
        if constexpr (cx != 0) sxx += v;
        if constexpr (cy != 0) syy += v;
        if constexpr (cz != 0) szz += v;
        if constexpr (cx * cy > 0) sxy += v; else if constexpr (cx * cy < 0) sxy -= v;
        if constexpr (cx * cz > 0) sxz += v; else if constexpr (cx * cz < 0) sxz -= v;
        if constexpr (cy * cz > 0) syz += v; else if constexpr (cy * cz < 0) syz -= v;
    });
    const float third = b0 * (1.0f / 3.0f);
    b[0] = b0; b[1] = sxx - third; b[2] = sxy; b[3] = sxz; b[4] = syy - third; b[5] = syz; b[6] = szz - third;
}

// mac = rho, u (unscaled), Pi_hat (unscaled xx,xy,xz,yy,yz,zz) from the
// known-set moment system of class c (the wall-node closed forms of the
// reference's bc_definition.inc, e.g. src/cases/lidDrivenCavity_3D/
// bc_definition.inc:637-663, solved generically).  The class words are read
// one at a time: read as 16-byte vectors they all issue up front and spill at
// the 102 registers a thread of the two-CTA wall kernels may use.
template <bool SH>
__device__ __forceinline__ float class_word(const float* w)
{
    if constexpr (SH) return *w;
    else return __ldg(w);
}
template <bool SH>
__device__ __forceinline__ uint32_t class_word(const uint32_t* w)
{
    if constexpr (SH) return *w;
    else return __ldg(w);
}

// SH: plain loads (c may point at the CTA's shared-memory copy of the class),
// else read-only cache loads from the table in global memory
template <int Q, bool SH = false>
__device__ __forceinline__ void bc_moments(const BcClass* __restrict__ c, const float* p, float omega,
                                           float omega0, float* mac)
{
    float b[7], X[7];
    bc_known_sums<Q>(class_word<SH>(&c->known), p, b);
#pragma unroll
    for (int r = 0; r < 7; r++) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 7; k++) acc = fmaf(class_word<SH>(&c->ainv[r * 7 + k]), b[k], acc);
        X[r] = acc;
    }
    // per-node omega (non-Newtonian): Sherman-Morrison update of A(omega0)^-1;
    // a Newtonian domain (omega == omega0) reads none of its words
    const float dw = omega - omega0;
    if (dw != 0.f) {
        float dot = 0.f;
#pragma unroll
        for (int r = 0; r < 7; r++) dot = fmaf(class_word<SH>(&c->qa[r]), b[r], dot);
        const float corr = dw * dot / (1.0f + dw * class_word<SH>(&c->s));
#pragma unroll
        for (int r = 0; r < 7; r++) X[r] = fmaf(-corr, class_word<SH>(&c->v[r]), X[r]);
    }
    const float rho = X[0], ir = 1.0f / rho;
    mac[0] = rho;
    mac[1] = class_word<SH>(&c->u[0]);
    mac[2] = class_word<SH>(&c->u[1]);
    mac[3] = class_word<SH>(&c->u[2]);
#pragma unroll
    for (int k = 0; k < 6; k++) mac[4 + k] = X[1 + k] * ir;
}

// Stored moment m at padded node offset idx of the buffer the step reads, in
// the stored scaling (FP32, or 16-bit times its storage scale).
template <typename T>
__device__ __forceinline__ float load_stored(const StepArgs& a, int m, long long idx)
{
    const float v = Stor<T>::ld(static_cast<const T*>(a.m_in) + mphys(m, idx, a.field));
    return scaled_storage<T>() ? v * a.iscale[m] : v;
}

// Outflow (nodeTypeMap BC_OUTFLOW, src/cases/mountedCube/bc_definition.inc:18-33,
// 55-67): the node takes the moments its inward neighbour stored in the
// previous step, unscaled, and collides them like any node.  (The reference
// reads its in-place array, whose neighbour entry another thread may or may
// not have rewritten already in the same step.)
template <typename T>
__device__ __forceinline__ void outflow_moments(const StepArgs& a, uint32_t kw, int x, int y, int z, float* mac)
{
    const int axis = (int)((kw >> 2) & 3u);
    const int side = (kw >> 4) & 1u ? 1 : -1;
    int n[3] = {x, y, z};
    n[axis] -= side;
    const long long idx = pidx(n[0], n[1], n[2], a.pitch, a.plane);
    mac[0] = a.rho0 + load_stored<T>(a, 0, idx);
    mac[1] = load_stored<T>(a, 1, idx) / 3.0f;
    mac[2] = load_stored<T>(a, 2, idx) / 3.0f;
    mac[3] = load_stored<T>(a, 3, idx) / 3.0f;
    mac[4] = load_stored<T>(a, 4, idx) / 4.5f;
    mac[5] = load_stored<T>(a, 5, idx) / 9.0f;
    mac[6] = load_stored<T>(a, 6, idx) / 9.0f;
    mac[7] = load_stored<T>(a, 7, idx) / 4.5f;
    mac[8] = load_stored<T>(a, 8, idx) / 9.0f;
    mac[9] = load_stored<T>(a, 9, idx) / 4.5f;
}

constexpr uint32_t BC_KIND_OUTFLOW = 2;  // nodeTypeMap bits 8-10

// Boundary-node policies of the step kernels: the run-time class table solved
// by bc_moments (the default), the same with outflow classes (launched only
// for domains that have them: the extra branch costs the wall kernels 4-6 %),
// or a case's own bc_definition snippet compiled into a policy of the same
// shape (case mode).
__device__ __forceinline__ void thermal_wall(const StepArgs& a, const BcClass* __restrict__ c, const float* pg,
                                             unsigned oidx, float& C, float* q);

// D3Q19 flow-only wall kernels stage the first classes of the table in shared
// memory (ZSmem::CT of them, in the space the ring leaves; the count staged
// is a word of the 128-byte header), so the wall solve's 50-odd class words
// come from shared memory instead of the read-only cache.  Classes past the
// staged count are read from global memory.
constexpr int HDR_STAGED_CLASSES = 40;  // byte offset of the count in the header
constexpr int HDR_TICKET = 48;          // tile-ordered step: the CTA's work index and step index
__device__ __forceinline__ unsigned char* dyn_smem()
{
    extern __shared__ __align__(128) unsigned char dyn_smem_base[];
    return dyn_smem_base;
}
__device__ __forceinline__ int staged_classes()
{
    return *reinterpret_cast<const int*>(dyn_smem() + HDR_STAGED_CLASSES);
}
__device__ __forceinline__ const BcClass* staged_class(int cls)
{
    return reinterpret_cast<const BcClass*>(dyn_smem() + 128) + cls;
}
// The run-time class table, read from global memory (D3Q27, thermal and
// batch kernels: a second inlined copy of the solve, or the shared copy's
// generic loads, measured slower or spilled there).
struct TableBC {
    template <int Q, typename T>
    static __device__ __forceinline__ void apply(const StepArgs& a, uint8_t cls, const float* p, float omega,
                                                 int x, int y, int z, float* mac)
    {
        bc_moments<Q>(a.bc + cls, p, omega, a.omega0, mac);
    }
    // C and 3 sum g c at a thermal boundary node: the class's run-time rule
    template <typename T>
    static __device__ __forceinline__ void thermal(const StepArgs& a, uint8_t cls, const float* pg, unsigned oidx,
                                                   int x, int y, int z, float& C, float* q)
    {
        thermal_wall(a, a.bc + cls, pg, oidx, C, q);
    }
};

struct OutflowBC {
    template <int Q, typename T>
    static __device__ __forceinline__ void apply(const StepArgs& a, uint8_t cls, const float* p, float omega,
                                                 int x, int y, int z, float* mac)
    {
        const BcClass* c = a.bc + cls;
        const uint32_t kw = __ldg(&c->trule);
        if (((kw >> 8) & 7u) == BC_KIND_OUTFLOW) outflow_moments<T>(a, kw, x, y, z, mac);
        else bc_moments<Q>(c, p, omega, a.omega0, mac);
    }
    template <typename T>
    static __device__ __forceinline__ void thermal(const StepArgs& a, uint8_t cls, const float* pg, unsigned oidx,
                                                   int x, int y, int z, float& C, float* q)
    {
        thermal_wall(a, a.bc + cls, pg, oidx, C, q);
    }
};

// The class table staged in shared memory, for the Newtonian D3Q19 wall
// kernels: a staged class is solved with shared-memory loads, any other from
// global memory (two inlined copies of the solve, which fit their registers:
// +11 % on a 128^3 cavity against TableBC).
struct TableBCShared : TableBC {
    template <int Q, typename T>
    static __device__ __forceinline__ void apply(const StepArgs& a, uint8_t cls, const float* p, float omega,
                                                 int x, int y, int z, float* mac)
    {
        if ((int)cls < staged_classes()) bc_moments<Q, true>(staged_class(cls), p, omega, a.omega0, mac);
        else bc_moments<Q>(a.bc + cls, p, omega, a.omega0, mac);
    }
};

// The class table staged in shared memory, for the non-Newtonian D3Q19 wall
// kernels: one solve through a generic pointer to the shared or the global
// copy (two copies spill there; +7 % on a power-law duct against TableBC).
struct TableBCGeneric : TableBC {
    template <int Q, typename T>
    static __device__ __forceinline__ void apply(const StepArgs& a, uint8_t cls, const float* p, float omega,
                                                 int x, int y, int z, float* mac)
    {
        const BcClass* c = (int)cls < staged_classes() ? staged_class(cls) : a.bc + cls;
        bc_moments<Q, true>(c, p, omega, a.omega0, mac);
    }
};

// policies whose kernels stage the class table
template <typename BCP>
struct stages_classes : std::false_type {};
template <>
struct stages_classes<TableBCShared> : std::true_type {};
template <>
struct stages_classes<TableBCGeneric> : std::true_type {};

// the class-table policy of a single-domain wall kernel
template <int Q, int FLAGS>
using table_policy_t =
    std::conditional_t<Q == 19 && (FLAGS & F_THERMAL) == 0,
                       std::conditional_t<(FLAGS & (F_POWERLAW | F_BINGHAM)) != 0, TableBCGeneric, TableBCShared>,
                       TableBC>;

// Power-law omega by Newton iteration (src/nnf.h:61-89 with its compile
// defects fixed) and Bingham (src/nnf.h:92-98).
__device__ __forceinline__ float nnf_powerlaw(float omega_old, float smag, float n, float K, float rho0)
{
    if (smag < 1e-6f) return 0.f;
    float omega = omega_old;
    // powers of positive bases on the special-function unit (__powf:
    // 2^(y log2 x)), with omega^(n-1) as omega^n / omega: one power an
    // iteration instead of two full powf; the two quotients by fast division
    // (2 ulp; omega and the derivative are O(0.1-10) here, +5 % on a
    // power-law duct).  omega = 0 (a node the cut-off
    // stopped in an earlier step) keeps powf's limits: 0^(n-1) is +inf for
    // n < 1, so the step vanishes and omega stays 0, as in the reference.
    const float a = K * __powf(smag / (rho0 * (1.0f / 3.0f)), n);
    const float b = 0.5f * smag, c = -smag;
    for (int it = 0; it < 7; it++) {
        float on, on1;
        if (omega > 0.f) {
            on = __powf(omega, n);
            on1 = __fdividef(on, omega);
        } else {
            on = powf(omega, n);
            on1 = powf(omega, n - 1.0f);
        }
        const float fx = fmaf(a, on, fmaf(b, omega, c));
        const float dfx = fmaf(a * n, on1, b);
        const float dx = __fdividef(fx, dfx);
        if (fabsf(dx) < 1e-6f) break;
        omega = omega - dx;
    }
    return omega;
}

// Scale to the stored form, update omega (non-Newtonian), collide
// (src/colrec/MR_LBM/collision.inc:2-14), write the 10/11 stored moments.
// The collision on the stored (scaled) moments: 3u, 4.5 Pi_ii, 9 Pi_ij
// (src/colrec/MR_LBM/collision.inc:2-14); writes the 10/11 stored moments.
template <int FLAGS>
__device__ __forceinline__ void collide_scaled(const StepArgs& a, float rho, float ux, float uy, float uz, float mxx,
                                               float mxy, float mxz, float myy, float myz, float mzz, float omega,
                                               float* out, float Fx, float Fy, float Fz)
{
    // every multiply-add is written as fmaf: the same bits wherever the
    // collision is inlined, whichever product the compiler would otherwise fuse
    const float t_om = 1.0f - omega, om_d2 = 0.5f * omega;
    if constexpr ((FLAGS & F_FORCE) != 0) {
        const float ir = 1.0f / rho;
        const float tt_om = 1.0f - 0.5f * omega;
        ux = fmaf(3.0f * ir, Fx, ux);
        uy = fmaf(3.0f * ir, Fy, uy);
        uz = fmaf(3.0f * ir, Fz, uz);
        const float c15 = 1.5f * ir * tt_om, c3 = 3.0f * tt_om * ir;
        mxx = fmaf(c15, 2.0f * Fx * ux, fmaf(t_om, mxx, om_d2 * ux * ux));
        myy = fmaf(c15, 2.0f * Fy * uy, fmaf(t_om, myy, om_d2 * uy * uy));
        mzz = fmaf(c15, 2.0f * Fz * uz, fmaf(t_om, mzz, om_d2 * uz * uz));
        mxy = fmaf(c3, fmaf(Fx, uy, Fy * ux), fmaf(t_om, mxy, omega * ux * uy));
        mxz = fmaf(c3, fmaf(Fx, uz, Fz * ux), fmaf(t_om, mxz, omega * ux * uz));
        myz = fmaf(c3, fmaf(Fy, uz, Fz * uy), fmaf(t_om, myz, omega * uy * uz));
    } else {
        mxx = fmaf(t_om, mxx, om_d2 * ux * ux);
        myy = fmaf(t_om, myy, om_d2 * uy * uy);
        mzz = fmaf(t_om, mzz, om_d2 * uz * uz);
        mxy = fmaf(t_om, mxy, omega * ux * uy);
        mxz = fmaf(t_om, mxz, omega * ux * uz);
        myz = fmaf(t_om, myz, omega * uy * uz);
    }
    out[0] = rho - a.rho0;
    out[1] = ux; out[2] = uy; out[3] = uz;
    out[4] = mxx; out[5] = mxy; out[6] = mxz; out[7] = myy; out[8] = myz; out[9] = mzz;
    out[10] = omega;
}

// Scale to the stored form, update omega (non-Newtonian), collide.
template <int FLAGS>
__device__ __forceinline__ void collide(const StepArgs& a, const float* mac, float omega, float* out, float Fx, float Fy,
                                        float Fz)
{
    const float rho = mac[0];
    if constexpr ((FLAGS & (F_POWERLAW | F_BINGHAM)) != 0) {
        // shear magnitude from the non-equilibrium second moments, src/mlbm.cu:526-546
        const float sxx = rho * (mac[4] - mac[1] * mac[1]), syy = rho * (mac[7] - mac[2] * mac[2]);
        const float szz = rho * (mac[9] - mac[3] * mac[3]), sxy = rho * (mac[5] - mac[1] * mac[2]);
        const float sxz = rho * (mac[6] - mac[1] * mac[3]), syz = rho * (mac[8] - mac[2] * mac[3]);
        const float gxx = sxx + mac[1] * Fx, gyy = syy + mac[2] * Fy, gzz = szz + mac[3] * Fz;
        const float gxy = sxy + 0.5f * (mac[1] * Fy + mac[2] * Fx);
        const float gxz = sxz + 0.5f * (mac[1] * Fz + mac[3] * Fx);
        const float gyz = syz + 0.5f * (mac[2] * Fz + mac[3] * Fy);
        const float smag = sqrtf(0.5f * (gxx * gxx + gyy * gyy + gzz * gzz + 2.0f * (gxy * gxy + gxz * gxz + gyz * gyz)));
        if constexpr ((FLAGS & F_POWERLAW) != 0)
            omega = nnf_powerlaw(omega, smag, a.nnf_n, a.nnf_k, a.rho0);
        else
            omega = a.nnf_omega_p * fmaxf(0.f, 1.0f - a.nnf_yield / smag);
    }
    collide_scaled<FLAGS>(a, rho, 3.0f * mac[1], 3.0f * mac[2], 3.0f * mac[3], 4.5f * mac[4], 9.0f * mac[5],
                          9.0f * mac[6], 4.5f * mac[7], 9.0f * mac[8], 4.5f * mac[9], omega, out, Fx, Fy, Fz);
}

// ---------------------------------------------------- TMA / mbarrier helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on the phase with the given parity; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned limit = WAIT_LIMIT)
{
    const uint32_t a = smem_u32(bar);
    for (unsigned it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 4-D tiled TMA load (x, moment, y, z) into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int m, int y, int z,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(m), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------- the step kernel

// Populations with c_y != 0 are exchanged between warp rows through shared
// memory, packed by (c_x, c_y): group g = 3*(c_y > 0) + c_x + 1 holds the
// c_z = -1, 0, +1 members in .x, .y, .z of a float4 (D3Q27: all six groups
// full; D3Q19: only the c_x = 0 groups are full, the four diagonal ones have
// one member and use a scalar slot).
__host__ __device__ constexpr int ex_group(int i) { return 3 * (lat_cy(i) > 0 ? 1 : 0) + lat_cx(i) + 1; }
__host__ __device__ constexpr bool ex_packed(int Q, int i) { return Q == 27 || lat_cx(i) == 0; }
// scalar slot for D3Q19 diagonal groups: (cx,cy) = (-1,-1),(1,-1),(-1,1),(1,1) -> 0..3
__host__ __device__ constexpr int ex_scalar_slot(int i) { return (lat_cy(i) > 0 ? 2 : 0) + (lat_cx(i) > 0 ? 1 : 0); }

template <int Q, int G>
__host__ __device__ constexpr bool ex_group_used()
{
    for (int i = 1; i < Q; i++)
        if (lat_cy(i) != 0 && ex_group(i) == G && ex_packed(Q, i)) return true;
    return false;
}

// float4 slot of group G: D3Q27 packs all six groups, D3Q19 only the two
// c_x = 0 ones (G = 1, 4)
__host__ __device__ constexpr int ex_npack(int Q) { return Q == 27 ? 6 : 2; }
__host__ __device__ constexpr int ex_slot4(int Q, int G) { return Q == 27 ? G : (G == 1 ? 0 : 1); }

// Exchange buffers hold TYI + 2 rows of EX_COLS slots per group: row
// er = y - Y0 + 1 (0: the row below the column, TYI + 1: the row above it),
// column ec = x - X0 + 1 (0 and 33: the nodes left and right of the column).
// An interior node's own slot is (w + 1, lane + 1), and the slot it reads a
// group from (row w + 1 - c_y, column lane + 1 - c_x) is a compile-time offset
// from it, so no index arithmetic runs per access.  The outer rows and
// columns are written by the helper warps.
constexpr int EX_COLS = TILE_X + 2;

template <int Q, int TYI>
struct Exchange {
    static constexpr int NPACK = ex_npack(Q);        // float4 groups
    static constexpr int NSCAL = Q == 19 ? 4 : 0;    // scalar slots
    static constexpr int rows = TYI + 2;
    static constexpr int plane = rows * EX_COLS;     // slots of one group
    static constexpr int buf4 = NPACK * plane;       // float4 per buffer
    static constexpr int buf1 = NSCAL * plane;       // floats per buffer
    static constexpr size_t bytes_per_buffer = (size_t)plane * (NPACK * 16 + NSCAL * 4);
    __host__ __device__ __forceinline__ static constexpr int slot(int er, int ec) { return er * EX_COLS + ec; }
};

// store group G of this lane's populations (its c_z = -1, 0, +1 members);
// e4t is this thread's slot of group 0 in the buffer being written
template <int Q, int G, int TYI>
__device__ __forceinline__ void ex_write(const float* f, float4* e4t)
{
    if constexpr (ex_group_used<Q, G>()) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        static_for<1, Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) != 0 && ex_group(i) == G && ex_packed(Q, i)) {
                if constexpr (lat_cz(i) < 0) v.x = f[i];
                else if constexpr (lat_cz(i) == 0) v.y = f[i];
                else v.z = f[i];
            }
        });
        float4* d = e4t + ex_slot4(Q, G) * Exchange<Q, TYI>::plane;
        if (MRLBM_SMEM_OK(d, 16, BCK_EXCHANGE)) *d = v;
    }
}

// every exchanged population (c_y != 0) of this node: packed groups and, on
// D3Q19, the four scalar slots
template <int Q, int TYI>
__device__ __forceinline__ void ex_write_all(const float* f, float4* e4t, float* e1t)
{
    ex_write<Q, 0, TYI>(f, e4t);
    ex_write<Q, 1, TYI>(f, e4t);
    ex_write<Q, 2, TYI>(f, e4t);
    ex_write<Q, 3, TYI>(f, e4t);
    ex_write<Q, 4, TYI>(f, e4t);
    ex_write<Q, 5, TYI>(f, e4t);
    if constexpr (Q == 19) {
        static_for<1, Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) != 0 && !ex_packed(Q, i)) {
                float* d = e1t + ex_scalar_slot(i) * Exchange<Q, TYI>::plane;
                if (MRLBM_SMEM_OK(d, 4, BCK_EXCHANGE)) *d = f[i];
            }
        });
    }
}

// the exchanged populations of a node outside the column that cross into it:
// CY = +1 / -1 selects the c_y of a row below / above the column (any c_x),
// CX = +1 / -1 the c_x of a node left / right of it (c_y = +-1; its c_y = 0
// members go to the edge buffer, ex_write_edge)
template <int Q, int TYI, int CX, int CY>
__device__ __forceinline__ void ex_write_sel(const float* f, float4* e4t, float* e1t)
{
    static_for<0, 6>([&](auto GG) {
        constexpr int G = GG;
        constexpr int gx = (G % 3) - 1, gy = G >= 3 ? 1 : -1;
        if constexpr ((CX == 0 || gx == CX) && (CY == 0 || gy == CY)) ex_write<Q, G, TYI>(f, e4t);
    });
    if constexpr (Q == 19) {
        static_for<1, Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) != 0 && !ex_packed(Q, i) && (CX == 0 || lat_cx(i) == CX) &&
                          (CY == 0 || lat_cy(i) == CY))
            {
                float* d = e1t + ex_scalar_slot(i) * Exchange<Q, TYI>::plane;
                if (MRLBM_SMEM_OK(d, 4, BCK_EXCHANGE)) *d = f[i];
            }
        });
    }
}

// the c_y = 0 populations with c_x = CX of an edge node (c_z = -1, 0, +1)
template <int Q, int CX>
__device__ __forceinline__ float4 edge_pops(const float* f)
{
    constexpr int im = lat_find(Q, CX, 0, -1), i0 = lat_find(Q, CX, 0, 0), ip = lat_find(Q, CX, 0, 1);
    return make_float4(f[im], f[i0], f[ip], 0.f);
}

// fetch group G arriving from row w - c_y, lane - c_x
template <int Q, int G, int TYI>
__device__ __forceinline__ void ex_read(float* g, const float4* e4t)
{
    if constexpr (ex_group_used<Q, G>()) {
        constexpr int cx = (G % 3) - 1, cy = G >= 3 ? 1 : -1;
        const float4* sp = e4t + ex_slot4(Q, G) * Exchange<Q, TYI>::plane - cy * EX_COLS - cx;
        const float4 v = MRLBM_SMEM_OK(sp, 16, BCK_EXCHANGE) ? *sp : make_float4(0.f, 0.f, 0.f, 0.f);
        static_for<1, Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) != 0 && ex_group(i) == G && ex_packed(Q, i))
                g[i] = lat_cz(i) < 0 ? v.x : (lat_cz(i) == 0 ? v.y : v.z);
        });
    }
}

// every population arriving at an interior node through the exchange
// (c_y != 0) and along x (c_y = 0: the shuffled gsh, or at the column's two
// outer lanes the edge buffer's float4 ee)
template <int Q, int TYI>
__device__ __forceinline__ void gather_pops(float* g, const float4* e4t, const float* e1t, const float (&gsh)[Q],
                                            float4 ee, bool xlo, bool xhi)
{
    ex_read<Q, 0, TYI>(g, e4t);
    ex_read<Q, 1, TYI>(g, e4t);
    ex_read<Q, 2, TYI>(g, e4t);
    ex_read<Q, 3, TYI>(g, e4t);
    ex_read<Q, 4, TYI>(g, e4t);
    ex_read<Q, 5, TYI>(g, e4t);
    if constexpr (Q == 19) {
        static_for<1, Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) != 0 && !ex_packed(Q, i))
            {
                const float* sp = e1t + ex_scalar_slot(i) * Exchange<Q, TYI>::plane - lat_cy(i) * EX_COLS - lat_cx(i);
                g[i] = MRLBM_SMEM_OK(sp, 4, BCK_EXCHANGE) ? *sp : 0.f;
            }
        });
    }
    static_for<0, Q>([&](auto I) {
        constexpr int i = I;
        if constexpr (lat_cy(i) == 0) {
            constexpr int cz = lat_cz(i);
            const float e = cz < 0 ? ee.x : (cz == 0 ? ee.y : ee.z);
            if constexpr (lat_cx(i) > 0) g[i] = xlo ? e : gsh[i];
            else if constexpr (lat_cx(i) < 0) g[i] = xhi ? e : gsh[i];
            else g[i] = gsh[i];
        }
    });
}

// a node's stored moments (unscaled to the FP32 stored form) from its element
// pair of moments 0, 1 in a TMA stage (pair p is 2 box_x<T>() elements further);
// with split storage (NML < NM) the stored words after the NML moments are the
// low parts of 3u (and of omega, moment 10, when NM - NML = 4), added to the
// high parts
template <int NM, typename T, int NML = NM>
__device__ __forceinline__ void stage_moments(const StepArgs& a, const T* sp, float* mc)
{
#pragma unroll
    for (int p = 0; p < (NM + 1) / 2; p++) {
        const T* q = sp + p * 2 * box_x<T>();
        const float2 v = MRLBM_SMEM_OK(q, 2 * (int)sizeof(T), BCK_STAGE) ? Stor2<T>::lds(q) : make_float2(0.f, 0.f);
        mc[2 * p] = scaled_storage<T>() ? v.x * a.iscale[2 * p] : v.x;
        if (2 * p + 1 < NM) mc[2 * p + 1] = scaled_storage<T>() ? v.y * a.iscale[2 * p + 1] : v.y;
    }
    if constexpr (NML < NM) {
        mc[1] += mc[NML];
        mc[2] += mc[NML + 1];
        mc[3] += mc[NML + 2];
        if constexpr (NM - NML == 4) mc[10] += mc[NML + 3];
    }
}

// split storage: the low words (stored words NML.., FP32 before the storage
// scaling) hold what the 16-bit high words of 3u (moments 1-3, stored with
// scale[1..3]) and of omega (moment 10, when NM - NML = 4) round away
template <int NM, int NML>
__device__ __forceinline__ void split_words(const StepArgs& a, float* o)
{
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float hi = __half2float(__float2half_rn(o[1 + c] * a.scale[1 + c])) * a.iscale[1 + c];
        o[NML + c] = o[1 + c] - hi;
    }
    if constexpr (NM - NML == 4) {
        const float hi = __half2float(__float2half_rn(o[10] * a.scale[10])) * a.iscale[10];
        o[NML + 3] = o[10] - hi;
    }
}

// thermal populations on D3G19 (the D3Q19 directions and weights):
// g_i = C w_i (1 + c_i . (u3 + ud3)), ud3 = coef (q3 / C - u3) with the
// node's stored flow velocity u3 = 3u and flux q3 = 3 sum g c
// (src/colrec/G_SCALAR/reconstruction.inc:1-25, src/mlbm.cu:159-169)
__device__ __forceinline__ void thermal_pops(const StepArgs& a, const float* mc, float* g)
{
    const float C = mc[10], iC = 1.0f / C;
    const float vx = fmaf(a.t_coef, fmaf(mc[11], iC, -mc[1]), mc[1]);
    const float vy = fmaf(a.t_coef, fmaf(mc[12], iC, -mc[2]), mc[2]);
    const float vz = fmaf(a.t_coef, fmaf(mc[13], iC, -mc[3]), mc[3]);
    static_for<0, 19>([&](auto I) {
        constexpr int i = I;
        float t = 1.0f;
        if constexpr (lat_cx(i) > 0) t += vx; else if constexpr (lat_cx(i) < 0) t -= vx;
        if constexpr (lat_cy(i) > 0) t += vy; else if constexpr (lat_cy(i) < 0) t -= vy;
        if constexpr (lat_cz(i) > 0) t += vz; else if constexpr (lat_cz(i) < 0) t -= vz;
        g[i] = (C * (float)lat_w(19, i)) * t;
    });
}

// Production of plane k at an interior node (first half of a pipeline
// step): the plane's moments come from TMA stage `stage`, its post-collision
// populations are reconstructed, the c_y != 0 ones are written to exchange
// buffer k&1 and the c_y = 0 ones are exchanged along x with shuffles into gsh
// (kept in registers until the plane is consumed, one step later; lanes 0 and
// 31 take their inward c_x members from the edge buffer then).
// sp: this thread's element pair of moments 0, 1 in the plane's TMA stage;
// e4t / e1t: this thread's exchange slots in the buffer this production writes.
template <int Q, int NM, typename T, int TYI, bool TH = false, int NML = NM>
__device__ __forceinline__ void prod_a(const StepArgs& a, const T* sp, float4* e4t, float* e1t, float (&gsh)[Q],
                                       float& om_node, float4* e4g = nullptr, float* e1g = nullptr,
                                       float* gshg = nullptr)
{
    float mc[NM];
    stage_moments<NM, T, NML>(a, sp, mc);
    float f[Q];
    reconstruct<Q>(mc, a.rho0, f);
    ex_write_all<Q, TYI>(f, e4t, e1t);
    static_for<0, Q>([&](auto I) {
        constexpr int i = I;
        if constexpr (lat_cy(i) == 0) {
            if constexpr (lat_cx(i) > 0) gsh[i] = __shfl_up_sync(0xffffffffu, f[i], 1);
            else if constexpr (lat_cx(i) < 0) gsh[i] = __shfl_down_sync(0xffffffffu, f[i], 1);
            else gsh[i] = f[i];
        }
    });
    om_node = mc[NML - 1];   // omega (moment 10) when the viscosity is per node
    if constexpr (TH) {
        float g[19];
        thermal_pops(a, mc, g);
        ex_write_all<19, TYI>(g, e4g, e1g);
        static_for<0, 19>([&](auto I) {
            constexpr int i = I;
            if constexpr (lat_cy(i) == 0) {
                if constexpr (lat_cx(i) > 0) gshg[i] = __shfl_up_sync(0xffffffffu, g[i], 1);
                else if constexpr (lat_cx(i) < 0) gshg[i] = __shfl_down_sync(0xffffffffu, g[i], 1);
                else gshg[i] = g[i];
            }
        });
    }
}

// Production of plane k by a helper warp: SIDE = -1 (bottom helper) produces
// the c_y = +1 populations of row Y0 - 1 (lane l: x = X0 + l) and the c_x = +1
// populations of the nodes x = X0 - 1 of rows Y0 - 1 .. Y0 + TYI (lane k:
// exchange row k); SIDE = +1 (top helper) the c_y = -1 populations of row
// Y0 + TYI and the c_x = -1 populations of the nodes x = X0 + 32.  Only the
// populations that cross into the column are formed (the others are dead code).
// hp / ep: the halo-row and edge node's element pair of moments 0, 1 in the
// stage; e4h / e1h and e4e / e1e: their exchange slots; edge: the edge buffer
// of this side and parity (one float4 per exchange row).
template <int Q, int NM, typename T, int TYI, int SIDE, bool TH = false, int NML = NM>
__device__ __forceinline__ void prod_helper(const StepArgs& a, int lane, const T* hp, const T* ep, float4* e4h,
                                            float* e1h, float4* e4e, float* e1e, float4* edge, float4* e4hg = nullptr,
                                            float* e1hg = nullptr, float4* e4eg = nullptr, float* e1eg = nullptr,
                                            float4* edgeg = nullptr)
{
    {
        float mc[NM], f[Q];
        stage_moments<NM, T, NML>(a, hp, mc);
        reconstruct<Q>(mc, a.rho0, f);
        ex_write_sel<Q, TYI, 0, -SIDE>(f, e4h, e1h);
        if constexpr (TH) {
            float g[19];
            thermal_pops(a, mc, g);
            ex_write_sel<19, TYI, 0, -SIDE>(g, e4hg, e1hg);
        }
    }
    if (lane < TYI + 2) {
        float mc[NM], f[Q];
        stage_moments<NM, T, NML>(a, ep, mc);
        reconstruct<Q>(mc, a.rho0, f);
        ex_write_sel<Q, TYI, -SIDE, 0>(f, e4e, e1e);
        if (MRLBM_SMEM_OK(edge + lane, 16, BCK_EDGE)) edge[lane] = edge_pops<Q, -SIDE>(f);
        if constexpr (TH) {
            float g[19];
            thermal_pops(a, mc, g);
            ex_write_sel<19, TYI, -SIDE, 0>(g, e4eg, e1eg);
            if (MRLBM_SMEM_OK(edgeg + lane, 16, BCK_EDGE)) edgeg[lane] = edge_pops<19, -SIDE>(g);
        }
    }
}

// D3Q19 direction with component `axis` of direction i negated
__host__ __device__ constexpr int lat_mirror19(int i, int axis)
{
    const int cx = axis == 0 ? -lat_cx(i) : lat_cx(i);
    const int cy = axis == 1 ? -lat_cy(i) : lat_cy(i);
    const int cz = axis == 2 ? -lat_cz(i) : lat_cz(i);
    return lat_find(19, cx, cy, cz);
}

// C and 3 sum g c at a boundary node of a thermal domain, by the class's rule
// (include/mrlbm.h MRLBM_THERMAL_*; the reference's per-case
// g_bc_definition.inc, e.g. src/cases/rayleighBenard_Periodic/g_bc_definition.inc,
// src/cases/rayleighBenard_Closed/g_bc_definition.inc).  pg: the streamed
// populations; values "from the previous step" come from the buffer this step
// reads (the reference reads its in-place buffer, whose neighbour entries may
// or may not have been updated already).
__device__ __forceinline__ void thermal_wall(const StepArgs& a, const BcClass* __restrict__ c, const float* pg,
                                             unsigned oidx, float& C, float* q)
{
    const uint32_t tr = c->trule;
    const int rule = (int)(tr & 3u), axis = (int)((tr >> 2) & 3u);
    const int side = (tr >> 4) & 1u ? 1 : -1;
    if (rule == 0) {
        // the stored values stand (node types without a thermal rule)
        const float* m_in = static_cast<const float*>(a.m_in);   // thermal domains store FP32
        C = m_in[mphys(10, oidx, a.field)];
        for (int k = 0; k < 3; k++) q[k] = m_in[mphys(11 + k, oidx, a.field)];
    } else if (rule == 1 || axis == 3) {
        C = c->twall;
        q[0] = q[1] = q[2] = 0.f;
    } else if (rule == 2) {
        // normal flux of the inward neighbour
        C = c->twall;
        q[0] = q[1] = q[2] = 0.f;
        const long long stride = axis == 0 ? 1LL : (axis == 1 ? (long long)a.pitch : a.plane);
        const long long nb = (long long)oidx - side * stride;
        q[axis] = static_cast<const float*>(a.m_in)[mphys(11 + axis, nb, a.field)];
    } else {
        // adiabatic: what arrives from the solid side is the mirror image of
        // what leaves towards it
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        static_for<0, 19>([&](auto I) {
            constexpr int i = I;
            const int ca = axis == 0 ? lat_cx(i) : (axis == 1 ? lat_cy(i) : lat_cz(i));
            const float mv = axis == 0 ? pg[lat_mirror19(i, 0)] : (axis == 1 ? pg[lat_mirror19(i, 1)] : pg[lat_mirror19(i, 2)]);
            const float v = ca == -side ? mv : pg[i];
            s0 += v;
            if constexpr (lat_cx(i) > 0) s1 += v; else if constexpr (lat_cx(i) < 0) s1 -= v;
            if constexpr (lat_cy(i) > 0) s2 += v; else if constexpr (lat_cy(i) < 0) s2 -= v;
            if constexpr (lat_cz(i) > 0) s3 += v; else if constexpr (lat_cz(i) < 0) s3 -= v;
        });
        C = s0;
        q[0] = 3.0f * s1; q[1] = 3.0f * s2; q[2] = 3.0f * s3;
    }
}

// store of the node at padded offset idx (< 2^32: a domain's moment field is
// limited to that at creation) through the per-pair base pointers: one
// 8-byte (FP32) or 4-byte (16-bit) store per moment pair
template <typename T, int NM>
__device__ __forceinline__ void store_node32(const StepArgs& a, unsigned idx, const float* o)
{
    if (!MRLBM_GLOBAL_OK((long long)idx < a.field, BCK_STORE, a.err)) return;
#pragma unroll
    for (int p = 0; p < NM / 2; p++) Stor2<T>::st(reinterpret_cast<T*>(a.out_p[p]) + 2 * (size_t)idx, o[2 * p], o[2 * p + 1]);
    if constexpr (NM % 2 != 0) Stor<T>::st(reinterpret_cast<T*>(a.out_p[NM / 2]) + 2 * (size_t)idx, o[NM - 1]);
}

template <typename T, int NM>
__device__ __forceinline__ void store_node(const StepArgs& a, long long idx, const float* o)
{
    if (!MRLBM_GLOBAL_OK(idx >= 0 && idx < a.field, BCK_STORE, a.err)) return;
    T* outp = reinterpret_cast<T*>(a.m_out);
#pragma unroll
    for (int m = 0; m < NM; m++) Stor<T>::st(outp + mphys(m, idx, a.field), o[m]);
}

// Consumption of plane k (second half): the c_y != 0 populations arriving from
// the neighbouring rows are read from exchange buffer k&1; with gsh they
// complete the populations that plane k sends.  Those with c_z = -1 complete
// output plane k-1 (= zp - 1), which is formed, collided and stored; the
// c_z = +1 and 0 ones enter the z pipeline.  The arithmetic is branch-free
// over the warp (so it interleaves with the next production); only the BC
// solve and the stores are predicated.
template <int Q, int NM, int NUP, int NMID, typename T, int FLAGS, int TYI, typename BCP, bool LIGHT = false>
__device__ __forceinline__ void prod_b(const StepArgs& a, int k, int zp, const float4* e4t, const float* e1t,
                                       const float4* eet, bool xlo, bool xhi, bool interior, int x, int y,
                                       const float (&gsh)[Q], float (&up_old)[NUP], float (&mid)[NMID], float om_out,
                                       const float4* e4g = nullptr, const float* e1g = nullptr,
                                       const float4* eetg = nullptr, const float* gshg = nullptr,
                                       float* upg_old = nullptr, float* midg = nullptr)
{
    constexpr bool TH = (FLAGS & F_THERMAL) != 0;
    // thermal populations arriving at the node (same three sources as the flow's)
    float gg[19], pg[19];
    if constexpr (TH) {
        float gshg19[19];
        static_for<0, 19>([&](auto I) { gshg19[I] = gshg[I]; });
        const float4 eeg = MRLBM_SMEM_OK(eetg, 16, BCK_EDGE) ? *eetg : make_float4(0.f, 0.f, 0.f, 0.f);
        gather_pops<19, TYI>(gg, e4g, e1g, gshg19, eeg, xlo, xhi);
        static_for<0, 19>([&](auto I) {
            constexpr int i = I;
            constexpr int slot = lat_cz_slot(19, i);
            if constexpr (lat_cz(i) > 0) pg[i] = upg_old[slot];
            else if constexpr (lat_cz(i) == 0) pg[i] = midg[slot];
            else pg[i] = gg[i];
        });
    }
    float g[Q];
    const float4 ee = MRLBM_SMEM_OK(eet, 16, BCK_EDGE) ? *eet : make_float4(0.f, 0.f, 0.f, 0.f);
    gather_pops<Q, TYI>(g, e4t, e1t, gsh, ee, xlo, xhi);

    if constexpr (!LIGHT) {
        // consumptions 0 and 1 complete no plane: the column runs them LIGHT
        // (only the z pipeline below moves)
        const bool live = interior && k >= 2;
        const int zd = zp - 1;
        float p[Q];
        static_for<0, Q>([&](auto I) {
            constexpr int i = I;
            constexpr int slot = lat_cz_slot(Q, i);
            if constexpr (lat_cz(i) > 0) p[i] = up_old[slot];
            else if constexpr (lat_cz(i) == 0) p[i] = mid[slot];
            else p[i] = g[i];
        });
        constexpr bool OMF = (FLAGS & (F_POWERLAW | F_BINGHAM)) != 0;
        const float omega = OMF ? om_out : a.omega0;
        const unsigned oidx = (unsigned)(zd + 1) * (unsigned)a.plane + (unsigned)((y + 1) * a.pitch + x + XOFF);
        uint8_t cls = CLS_BULK;
        if constexpr ((FLAGS & F_BC) != 0)
            cls = (live && MRLBM_GLOBAL_OK((long long)oidx < a.field, BCK_CLASS, a.err)) ? __ldg(a.cls + oidx) : CLS_SOLID;
        float o[NM_MAX];
        float r, j[3], P[6];
        lattice_sums<Q>(p, r, j, P);
        float Fx = 0.f, Fy = 0.f, Fz = 0.f;
        if constexpr ((FLAGS & F_FORCE) != 0) { Fx = a.fx; Fy = a.fy; Fz = a.fz; }
        float tC = 0.f, tq[3] = {0.f, 0.f, 0.f};
        if constexpr (TH) {
            // C = sum g + source, q3 = 3 sum g c at bulk nodes (src/mlbm.cu:180-188) and
            // the Boussinesq force there (src/mlbm.cu:515-522); walls by their rule
            if (cls == CLS_BULK) {
                float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
                static_for<0, 19>([&](auto I) {
                    constexpr int i = I;
                    s0 += pg[i];
                    if constexpr (lat_cx(i) > 0) s1 += pg[i]; else if constexpr (lat_cx(i) < 0) s1 -= pg[i];
                    if constexpr (lat_cy(i) > 0) s2 += pg[i]; else if constexpr (lat_cy(i) < 0) s2 -= pg[i];
                    if constexpr (lat_cz(i) > 0) s3 += pg[i]; else if constexpr (lat_cz(i) < 0) s3 -= pg[i];
                });
                tC = s0 + a.t_src;
                tq[0] = 3.0f * s1; tq[1] = 3.0f * s2; tq[2] = 3.0f * s3;
                const float dC = tC - a.t_ref;
                Fx = fmaf(a.t_gb[0], dC, Fx);
                Fy = fmaf(a.t_gb[1], dC, Fy);
                Fz = fmaf(a.t_gb[2], dC, Fz);
            } else if (cls != CLS_SOLID) {
                BCP::template thermal<T>(a, cls, pg, oidx, x, y, zd, tC, tq);
            }
        }
        if constexpr ((FLAGS & (F_BC | F_POWERLAW | F_BINGHAM)) == 0) {
            // bulk-only domains: the moments straight in the stored scaling
            // (3u = 3 j / rho, 4.5 Pi_ii = 4.5 P_ii / rho - 1.5, 9 Pi_ij)
            const float ir = 1.0f / r;
            const float i3 = 3.0f * ir, i45 = 4.5f * ir, i9 = 9.0f * ir;
            collide_scaled<FLAGS>(a, r, j[0] * i3, j[1] * i3, j[2] * i3, fmaf(P[0], i45, -1.5f), P[1] * i9, P[2] * i9,
                                  fmaf(P[3], i45, -1.5f), P[4] * i9, fmaf(P[5], i45, -1.5f), omega, o, Fx, Fy, Fz);
        } else {
            float mac[10];
            const float ir = 1.0f / r;
            mac[0] = r;
            mac[1] = j[0] * ir; mac[2] = j[1] * ir; mac[3] = j[2] * ir;
            mac[4] = P[0] * ir - (1.0f / 3.0f);
            mac[5] = P[1] * ir;
            mac[6] = P[2] * ir;
            mac[7] = P[3] * ir - (1.0f / 3.0f);
            mac[8] = P[4] * ir;
            mac[9] = P[5] * ir - (1.0f / 3.0f);
            if constexpr ((FLAGS & F_BC) != 0) {
                if (cls != CLS_BULK && cls != CLS_SOLID) BCP::template apply<Q, T>(a, cls, p, omega, x, y, zd, mac);
            }
            collide<FLAGS>(a, mac, omega, o, Fx, Fy, Fz);
        }
        if constexpr (TH) {
            o[10] = tC;
            o[11] = tq[0]; o[12] = tq[1]; o[13] = tq[2];
        }
        if constexpr ((FLAGS & F_SPLITU) != 0) split_words<NM, nmoments_of(FLAGS & ~F_SPLITU)>(a, o);
        if constexpr (scaled_storage<T>()) {
#pragma unroll
            for (int m = 0; m < NM; m++) o[m] = o[m] * a.scale[m];
        }
        if (live && cls != CLS_SOLID) {
            store_node32<T, NM>(a, oidx, o);
            // periodic axes: keep the ghost shell equal to the wrapped interior
            const bool gx = (a.periodic & 1) && (x == 0 || x == a.nx - 1);
            const bool gy = (a.periodic & 2) && (y == 0 || y == a.ny - 1);
            const bool gz = (a.periodic & 4) && (zd == 0 || zd == a.nz - 1);
            if (gx || gy || gz) {
                if ((gx && a.nx == 1) || (gy && a.ny == 1) || (gz && a.nz == 1)) {
                    // degenerate one-node axis: the node has both ghost copies
#pragma unroll 1
                    for (int iz = 0; iz < 3; iz++)
#pragma unroll 1
                        for (int iy = 0; iy < 3; iy++)
#pragma unroll 1
                            for (int ix = 0; ix < 3; ix++) {
                                const bool vz = iz == 0 || (gz && (iz == 1 ? zd == 0 : zd == a.nz - 1));
                                const bool vy = iy == 0 || (gy && (iy == 1 ? y == 0 : y == a.ny - 1));
                                const bool vx = ix == 0 || (gx && (ix == 1 ? x == 0 : x == a.nx - 1));
                                if (!(vx && vy && vz) || (ix == 0 && iy == 0 && iz == 0)) continue;
                                const int cz = iz == 0 ? zd : (iz == 1 ? a.nz : -1);
                                const int cy = iy == 0 ? y : (iy == 1 ? a.ny : -1);
                                const int cxx = ix == 0 ? x : (ix == 1 ? a.nx : -1);
                                store_node<T, NM>(a, pidx(cxx, cy, cz, a.pitch, a.plane), o);
                            }
                } else {
                    const int xa = x == 0 ? a.nx : -1, ya = y == 0 ? a.ny : -1, za = zd == 0 ? a.nz : -1;
                    if (gx) store_node<T, NM>(a, pidx(xa, y, zd, a.pitch, a.plane), o);
                    if (gy) store_node<T, NM>(a, pidx(x, ya, zd, a.pitch, a.plane), o);
                    if (gz) store_node<T, NM>(a, pidx(x, y, za, a.pitch, a.plane), o);
                    if (gx && gy) store_node<T, NM>(a, pidx(xa, ya, zd, a.pitch, a.plane), o);
                    if (gx && gz) store_node<T, NM>(a, pidx(xa, y, za, a.pitch, a.plane), o);
                    if (gy && gz) store_node<T, NM>(a, pidx(x, ya, za, a.pitch, a.plane), o);
                    if (gx && gy && gz) store_node<T, NM>(a, pidx(xa, ya, za, a.pitch, a.plane), o);
                }
            }
        }
    }
    // advance the z pipeline: the consumed U(zp-2) slot now holds U(zp)
    static_for<0, Q>([&](auto I) {
        constexpr int i = I;
        constexpr int slot = lat_cz_slot(Q, i);
        if constexpr (lat_cz(i) > 0) up_old[slot] = g[i];
        else if constexpr (lat_cz(i) == 0) mid[slot] = g[i];
    });
    if constexpr (TH) {
        static_for<0, 19>([&](auto I) {
            constexpr int i = I;
            constexpr int slot = lat_cz_slot(19, i);
            if constexpr (lat_cz(i) > 0) upg_old[slot] = gg[i];
            else if constexpr (lat_cz(i) == 0) midg[slot] = gg[i];
        });
    }
}

// Shared-memory carve-up used by every z-march kernel: barriers, TMA ring,
// double-buffered exchange, edge buffers.  Ring slots hold NPM moment pairs
// (kernels that switch between flag sets at run time size them for the
// largest set), and the ring has NSTAGE_MAX stages when they fit next to the
// exchange buffers, else fewer.
template <int Q, typename T, int TYI, int NPM, bool TH = false, int RESERVE = 0, bool WC = false>
struct ZSmem {
    static constexpr int NR = TYI + 2;  // stage rows = exchange rows
    static constexpr size_t stage_max = ((size_t)NR * NPM * 2 * box_x<T>() * sizeof(T) + 127) / 128 * 128;
    // the thermal populations have a row exchange of their own (D3Q19 layout)
    static constexpr size_t ex_bytes =
        2 * Exchange<Q, TYI>::bytes_per_buffer + (TH ? 2 * Exchange<19, TYI>::bytes_per_buffer : 0);
    // c_y = 0 populations of the edge nodes: [side][parity][row] float4
    // (flow, then thermal)
    static constexpr int edge_n = 2 * 2 * NR;
    static constexpr size_t edge_bytes = (size_t)(TH ? 2 : 1) * edge_n * 16;
    static constexpr size_t fixed = 128 + ex_bytes + edge_bytes;
    // RESERVE: the kernel's static shared memory, which the CTA's share holds too
    static constexpr size_t budget = smem_budget(TYI) - RESERVE;
    static constexpr int NS = fixed + NSTAGE_MAX * stage_max <= budget         ? NSTAGE_MAX
                              : fixed + (NSTAGE_MAX - 1) * stage_max <= budget ? NSTAGE_MAX - 1
                                                                               : NSTAGE_MAX - 2;
    static constexpr size_t ring_bytes = fixed + NS * stage_max;
    // WC: the wall kernel's class table, as many classes as the space the
    // ring leaves holds (at most 255), right after the header
    static constexpr size_t ct_bytes_of(int n) { return ((size_t)n * sizeof(BcClass) + 127) / 128 * 128; }
    static constexpr int ct_fit()
    {
        int n = WC ? (int)((budget - ring_bytes) / sizeof(BcClass)) : 0;
        if (n > 255) n = 255;
        while (n > 0 && ring_bytes + ct_bytes_of(n) > budget) n--;
        return n;
    }
    static constexpr int CT = ct_fit();
    static constexpr size_t ct_bytes = ct_bytes_of(CT);
    static constexpr size_t bytes = ring_bytes + ct_bytes;
    static_assert(bytes <= budget, "shared memory over the sm_100 limit");
    uint64_t* bars;   // the ring's mbarriers, then the CTA's timeout flag (bars + NSTAGE_MAX)
    unsigned char* stages;
    float4* ex4;
    float* ex1;
    float4* exg4;   // thermal exchange (TH only)
    float* exg1;
    float4* edge;   // flow edge buffer
    float4* edgeg;  // thermal edge buffer (TH only)
    __device__ __forceinline__ explicit ZSmem(unsigned char* smem)
    {
        bars = reinterpret_cast<uint64_t*>(smem);
        stages = smem + 128 + ct_bytes;
        ex4 = reinterpret_cast<float4*>(stages + NS * stage_max);
        ex1 = reinterpret_cast<float*>(ex4 + 2 * Exchange<Q, TYI>::buf4);
        exg4 = reinterpret_cast<float4*>(ex1 + 2 * Exchange<Q, TYI>::buf1);
        exg1 = reinterpret_cast<float*>(exg4 + (TH ? 2 * Exchange<19, TYI>::buf4 : 0));
        edge = reinterpret_cast<float4*>(exg1 + (TH ? 2 * Exchange<19, TYI>::buf1 : 0));
        edgeg = edge + edge_n;
    }
};



// Per-CTA pipeline state of the z-march over one column.  The TMA ring is
// indexed by a running production count `g0 + k` so a persistent CTA can
// chain columns without re-initialising its mbarriers.  Warps 0 .. TYI-1 run
// the interior pipeline (interior_loop), warps TYI and TYI+1 the helper one
// (helper_loop); both take the same barriers in the same order.
template <int Q, typename T, int FLAGS, int TYI, typename BCP, int NPM, int RES = 0, bool WC = false>
struct ZMarch {
    static constexpr int NR = TYI + 2;
    static constexpr int BX = box_x<T>();
    static constexpr int NUP = lat_num_cz(Q, 1);
    static constexpr int NMID = lat_num_cz(Q, 0);
    static constexpr bool OMF = (FLAGS & (F_POWERLAW | F_BINGHAM)) != 0;
    static constexpr bool TH = (FLAGS & F_THERMAL) != 0;
    static constexpr int NM = nmoments_of(FLAGS);
    static constexpr int NML = nmoments_of(FLAGS & ~F_SPLITU);  // moments before the split storage's low words
    static constexpr int NP = (NM + 1) / 2;  // moment pairs in a stage row
    static constexpr int ROW = NP * 2 * BX;  // elements of a stage row
    static constexpr size_t stage_bytes = (size_t)NR * ROW * sizeof(T);
    using EX = Exchange<Q, TYI>;
    using EXG = Exchange<19, TYI>;
    using SM = ZSmem<Q, T, TYI, NPM, TH, RES, WC>;
    static constexpr int NS = SM::NS;
    static constexpr int TMA_THREAD = 32 * TYI;  // lane 0 of the bottom helper
    static_assert(NP <= NPM, "ring slots sized for fewer moment pairs");

    const StepArgs& a;
    const CUtensorMap* map;
    const SM& sm;
    unsigned g0;
    int X0, Y0, z0, p0, nprod;
    int cs;           // ring slot of the next production to wait for
    unsigned cph;     // its mbarrier phase parity

    __device__ __forceinline__ int slot(int k) const { return (int)((g0 + (unsigned)k) % NS); }
    __device__ __forceinline__ unsigned phase(int k) const { return ((g0 + (unsigned)k) / NS) & 1u; }
    static constexpr size_t ring_stride = SM::stage_max;
    __device__ __forceinline__ const T* stage_base() const { return reinterpret_cast<const T*>(sm.stages + cs * ring_stride); }
    // element offset of node x of stage row er (pair of moments 0, 1)
    __device__ __forceinline__ int stage_off(int er, int x) const { return er * ROW + 2 * ((x + XOFF) - p0); }
    __device__ __forceinline__ void load_slot(int s, int k) const
    {
        mbar_expect_tx(&sm.bars[s], (unsigned)stage_bytes);
        // x runs over the interleaved pair elements: 2 per node
        tma_load_4d(sm.stages + s * ring_stride, map, 2 * p0, 0, Y0, z0 + k, &sm.bars[s]);
    }
    __device__ __forceinline__ void load(int k) const { load_slot(slot(k), k); }
    // CTA-wide timeout flag next to the ring barriers: a thread whose bounded
    // wait gave up raises it before the per-plane barrier, every thread reads
    // it after (a plain barrier measured 3 % faster than a reducing one)
    __device__ __forceinline__ void raise_timeout() const { *reinterpret_cast<volatile int*>(sm.bars + NSTAGE_MAX) = 1; }
    __device__ __forceinline__ bool timed_out() const { return *reinterpret_cast<volatile int*>(sm.bars + NSTAGE_MAX) != 0; }
    // after production k: reload its slot with production k + NS, then move
    // to the next slot
    __device__ __forceinline__ void advance(int k)
    {
        if (threadIdx.x == TMA_THREAD && k + NS < nprod) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            load_slot(cs, k + NS);
        }
        if (++cs == NS) {
            cs = 0;
            cph ^= 1u;
        }
    }
    // end of pipeline step k: barrier, timeout check, ring advance
    __device__ __forceinline__ bool end_step(int k, bool ok)
    {
        if (!ok) raise_timeout();
        __syncthreads();
        if (timed_out()) return false;
#ifdef MRLBM_BOUNDS_CHECK
        // the buffers consumption k-1 read are free until production k+1
        // writes them: NaN in every slot first
        poison((k + 1) & 1);
        __syncthreads();
#endif
        advance(k);
        return true;
    }
#ifdef MRLBM_BOUNDS_CHECK
    __device__ void poison(int par) const
    {
        const float nan = __int_as_float(0x7fc00000);
        const float4 n4 = make_float4(nan, nan, nan, nan);
        for (int i = threadIdx.x; i < EX::buf4; i += blockDim.x) sm.ex4[par * EX::buf4 + i] = n4;
        for (int i = threadIdx.x; i < EX::buf1; i += blockDim.x) sm.ex1[par * EX::buf1 + i] = nan;
        if constexpr (TH) {
            for (int i = threadIdx.x; i < EXG::buf4; i += blockDim.x) sm.exg4[par * EXG::buf4 + i] = n4;
            for (int i = threadIdx.x; i < EXG::buf1; i += blockDim.x) sm.exg1[par * EXG::buf1 + i] = nan;
        }
        for (int i = threadIdx.x; i < 2 * NR; i += blockDim.x) {
            const int side = i / NR, er = i % NR;
            sm.edge[(side * 2 + par) * NR + er] = n4;
            if constexpr (TH) sm.edgeg[(side * 2 + par) * NR + er] = n4;
        }
    }
#endif

    // ---- interior warps: row w, lane l = node (X0 + l, Y0 + w)
    struct Interior {
        float4* e4t[2];   // this thread's exchange slots, buffer 0 and 1
        float* e1t[2];
        const float4* eet[2];  // its edge-buffer float4 (used by lanes 0 and 31)
        float4* e4g[2];   // thermal
        float* e1g[2];
        const float4* eetg[2];
        int toff;         // its element offset in a stage
        int x, y;
        bool interior, xlo, xhi;
    };

    // pipeline step j (parity PAR = j & 1): production j into exchange
    // buffer PAR and consumption j-1 from buffer PAR ^ 1, one barrier.  The
    // node output by consumption j-1 lies in the plane of production j-2,
    // whose stored omega is in om_par (same parity as j) until production j
    // overwrites it.  Returns false when a bounded wait timed out somewhere
    // in the CTA.
    template <int PAR, bool LIGHT = false>
    __device__ __forceinline__ bool iter(const Interior& it, int j, float (&gsh_new)[Q], const float (&gsh_old)[Q],
                                         float (&up)[NUP], float (&mid)[NMID], float& om_par, float* sg_new = nullptr,
                                         const float* sg_old = nullptr, float* upg = nullptr, float* midg = nullptr)
    {
        const bool ok = mbar_wait(&sm.bars[cs], cph);
        const float om_out = om_par;
        // the two halves are independent; which comes first in the source
        // only steers the compiler's schedule (results are bit-identical):
        // consumption first measured 4 % faster on bulk and D3Q27 domains,
        // production first 4 % faster on D3Q19 domains with walls
        if constexpr (Q == 27 || (FLAGS & F_BC) == 0) {
            prod_b<Q, NM, NUP, NMID, T, FLAGS, TYI, BCP, LIGHT>(
                a, j - 1, z0 - 2 + j, it.e4t[PAR ^ 1], it.e1t[PAR ^ 1], it.eet[PAR ^ 1], it.xlo, it.xhi, it.interior,
                it.x, it.y, gsh_old, up, mid, om_out, it.e4g[PAR ^ 1], it.e1g[PAR ^ 1], it.eetg[PAR ^ 1], sg_old, upg,
                midg);
            prod_a<Q, NM, T, TYI, TH, NML>(a, stage_base() + it.toff, it.e4t[PAR], it.e1t[PAR], gsh_new, om_par,
                                      it.e4g[PAR], it.e1g[PAR], sg_new);
        } else {
            prod_a<Q, NM, T, TYI, TH, NML>(a, stage_base() + it.toff, it.e4t[PAR], it.e1t[PAR], gsh_new, om_par,
                                      it.e4g[PAR], it.e1g[PAR], sg_new);
            prod_b<Q, NM, NUP, NMID, T, FLAGS, TYI, BCP, LIGHT>(
                a, j - 1, z0 - 2 + j, it.e4t[PAR ^ 1], it.e1t[PAR ^ 1], it.eet[PAR ^ 1], it.xlo, it.xhi, it.interior,
                it.x, it.y, gsh_old, up, mid, om_out, it.e4g[PAR ^ 1], it.e1g[PAR ^ 1], it.eetg[PAR ^ 1], sg_old, upg,
                midg);
        }
        return end_step(j, ok);
    }

    // the interior pipeline; returns the production whose step timed out, or -1
    __device__ __forceinline__ int interior_loop(int lane, int warp)
    {
        const int er = warp + 1;
        const int ts = EX::slot(er, lane + 1);
        const int eside = lane >= TILE_X / 2 ? 1 : 0;
        Interior it;
        it.e4t[0] = sm.ex4 + ts; it.e4t[1] = sm.ex4 + EX::buf4 + ts;
        it.e1t[0] = sm.ex1 + ts; it.e1t[1] = sm.ex1 + EX::buf1 + ts;
        it.eet[0] = sm.edge + (eside * 2 + 0) * NR + er; it.eet[1] = sm.edge + (eside * 2 + 1) * NR + er;
        it.e4g[0] = sm.exg4 + ts; it.e4g[1] = sm.exg4 + EXG::buf4 + ts;
        it.e1g[0] = sm.exg1 + ts; it.e1g[1] = sm.exg1 + EXG::buf1 + ts;
        it.eetg[0] = sm.edgeg + (eside * 2 + 0) * NR + er; it.eetg[1] = sm.edgeg + (eside * 2 + 1) * NR + er;
        it.x = X0 + lane;
        it.y = Y0 + warp;
        it.toff = stage_off(er, it.x);
        it.interior = it.x < a.nx && it.y < a.ny;
        it.xlo = lane == 0;
        it.xhi = lane == TILE_X - 1;

        float upA[NUP], upB[NUP], mid[NMID], gA[Q], gB[Q];
#pragma unroll
        for (int s = 0; s < NUP; s++) upA[s] = upB[s] = 0.f;
#pragma unroll
        for (int s = 0; s < NMID; s++) mid[s] = 0.f;
        float omA = a.omega0, omB = a.omega0;
        // thermal populations: the same pipeline on the D3Q19 directions
        constexpr int NUPG = TH ? lat_num_cz(19, 1) : 1, NMIDG = TH ? lat_num_cz(19, 0) : 1;
        constexpr int NSG = TH ? 19 : 1;
        float ugA[NUPG], ugB[NUPG], mg[NMIDG], sgA[NSG], sgB[NSG];
#pragma unroll
        for (int s = 0; s < NUPG; s++) ugA[s] = ugB[s] = 0.f;
#pragma unroll
        for (int s = 0; s < NMIDG; s++) mg[s] = 0.f;

        {
            // prologue: production 0 only (exchange buffer 0)
            const bool ok = mbar_wait(&sm.bars[cs], cph);
            prod_a<Q, NM, T, TYI, TH, NML>(a, stage_base() + it.toff, it.e4t[0], it.e1t[0], gA, omA, it.e4g[0], it.e1g[0],
                                      sgA);
            if (!end_step(0, ok)) return 0;
        }
        // even productions use gA / upA and exchange buffer 0, odd ones gB / upB
        // and buffer 1: no register copies, no buffer selection at run time.
        // Consumptions 0 and 1 would complete planes z0 - 2 and z0 - 1, which
        // are not this column's: they only move the z pipeline (nprod >= 3, so
        // productions 1 and 2 exist).  The thermal variants keep them in the
        // loop: two more inlined pipeline steps raise their register spills.
        int j = 1;
        if constexpr (!TH) {
            if (!iter<1, true>(it, 1, gB, gA, upA, mid, omB, sgB, sgA, ugA, mg)) return 1;
            if (!iter<0, true>(it, 2, gA, gB, upB, mid, omA, sgA, sgB, ugB, mg)) return 2;
            j = 3;
        }
        for (;;) {
            // epilogues consume the last production j-1; its output plane is that
            // of production j-2, whose omega has the parity of j
            if (j >= nprod) {  // j odd: last production even
                prod_b<Q, NM, NUP, NMID, T, FLAGS, TYI, BCP>(a, j - 1, z0 - 2 + j, it.e4t[0], it.e1t[0], it.eet[0],
                                                            it.xlo, it.xhi, it.interior, it.x, it.y, gA, upA, mid, omB,
                                                            it.e4g[0], it.e1g[0], it.eetg[0], sgA, ugA, mg);
                return -1;
            }
            if (!iter<1>(it, j, gB, gA, upA, mid, omB, sgB, sgA, ugA, mg)) return j;
            j++;
            if (j >= nprod) {  // j even: last production odd
                prod_b<Q, NM, NUP, NMID, T, FLAGS, TYI, BCP>(a, j - 1, z0 - 2 + j, it.e4t[1], it.e1t[1], it.eet[1],
                                                            it.xlo, it.xhi, it.interior, it.x, it.y, gB, upB, mid, omA,
                                                            it.e4g[1], it.e1g[1], it.eetg[1], sgB, ugB, mg);
                return -1;
            }
            if (!iter<0>(it, j, gA, gB, upB, mid, omA, sgA, sgB, ugB, mg)) return j;
            j++;
        }
    }

    // the helper pipeline (SIDE -1: bottom row and left edge, +1: top row and
    // right edge); returns the production whose step timed out, or -1
    template <int SIDE>
    __device__ __forceinline__ int helper_loop(int lane)
    {
        constexpr int erh = SIDE < 0 ? 0 : TYI + 1;          // exchange row of the halo row
        constexpr int ece = SIDE < 0 ? 0 : EX_COLS - 1;      // exchange column of the edge nodes
        const int hoff = stage_off(erh, X0 + lane);
        const int eoff = stage_off(lane, SIDE < 0 ? X0 - 1 : X0 + TILE_X);
        const int sh = EX::slot(erh, lane + 1), se = EX::slot(lane, ece);
        const int side = SIDE < 0 ? 0 : 1;
        for (int j = 0; j < nprod; j++) {
            const bool ok = mbar_wait(&sm.bars[cs], cph);
            const int par = j & 1;
            const T* st = stage_base();
            float4* e4 = sm.ex4 + par * EX::buf4;
            float* e1 = sm.ex1 + par * EX::buf1;
            float4* g4 = sm.exg4 + par * EXG::buf4;
            float* g1 = sm.exg1 + par * EXG::buf1;
            prod_helper<Q, NM, T, TYI, SIDE, TH, NML>(a, lane, st + hoff, st + eoff, e4 + sh, e1 + sh, e4 + se, e1 + se,
                                                 sm.edge + (side * 2 + par) * NR, g4 + sh, g1 + sh, g4 + se, g1 + se,
                                                 sm.edgeg + (side * 2 + par) * NR);
            if (!end_step(j, ok)) return j;
        }
        return -1;
    }
};

// One column (X0, Y0) x planes [z0, zend) of one domain.  g0 is the CTA's
// running production count (advanced by the column's productions).  Returns
// false when a bounded wait timed out (the CTA must stop).
template <int Q, typename T, int FLAGS, int TYI, typename BCP = TableBC, int NPM, int RES, bool WC>
__device__ __forceinline__ bool zmarch_column(const StepArgs& a, const CUtensorMap* map, int X0, int Y0, int z0,
                                              int zend,
                                              const ZSmem<Q, T, TYI, NPM, (FLAGS & F_THERMAL) != 0, RES, WC>& sm,
                                              unsigned& g0)
{
    using ZM = ZMarch<Q, T, FLAGS, TYI, BCP, NPM, RES, WC>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // aligned box start (padded column): the TMA x coordinate, 2 elements a
    // node, must be a multiple of 16 bytes
    constexpr int NODE_ALIGN = 8 / (int)sizeof(T);
    const int p0 = (X0 - 1 + XOFF) & ~(NODE_ALIGN - 1);
    ZM zm{a, map, sm, g0, X0, Y0, z0, p0, zend - z0 + 2 /* planes z0-1 .. zend */, 0, 0u};
    zm.cs = zm.slot(0);
    zm.cph = zm.phase(0);
#ifdef MRLBM_BOUNDS_CHECK
    if (threadIdx.x == 0) {
        using SMT = ZSmem<Q, T, TYI, NPM, (FLAGS & F_THERMAL) != 0, RES, WC>;
        g_bounds.stage_lo = smem_u32(sm.stages);
        g_bounds.stage_hi = smem_u32(sm.stages) + (unsigned)(SMT::NS * SMT::stage_max);
        g_bounds.ex_lo = smem_u32(sm.ex4);
        g_bounds.ex_hi = smem_u32(sm.edge);
        g_bounds.edge_lo = smem_u32(sm.edge);
        g_bounds.edge_hi = smem_u32(sm.edge) + (unsigned)SMT::edge_bytes;
        g_bounds.err = a.err;
    }
    // no TMA load may land in the ring before the CTA's poison writes are done
    __syncthreads();
    zm.poison(0);
    zm.poison(1);
    __syncthreads();
#endif

    if (threadIdx.x == ZM::TMA_THREAD) {
        // the ring was last read through the generic proxy (previous column)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int s = 0; s < ZM::NS && s < zm.nprod; s++) zm.load(s);
    }
    int kfail;
    if (warp < TYI) kfail = zm.interior_loop(lane, warp);
    else if (warp == TYI) kfail = zm.template helper_loop<-1>(lane);
    else kfail = zm.template helper_loop<1>(lane);
    if (kfail >= 0) {
        // a bounded wait gave up: flag it, give the copies still in flight a
        // bounded time to land, and leave together
        if (threadIdx.x == ZM::TMA_THREAD) {
            atomicOr(a.err, 1);
            for (int q = kfail; q < zm.nprod && q < kfail + ZM::NS; q++) (void)mbar_wait(&sm.bars[zm.slot(q)], zm.phase(q));
        }
        __syncthreads();
        return false;
    }
    g0 += (unsigned)zm.nprod;
    // the last consumption read exchange buffers other warps may overwrite next
    __syncthreads();
    return true;
}

// Barriers, the timeout flag and, in wall kernels, the staged copy of the
// first ZSmem::CT classes of the table bc (nbc classes)
template <int Q, typename T, int TYI, int NPM, bool TH, int RES, bool WC>
__device__ __forceinline__ void zmarch_init_barriers(const ZSmem<Q, T, TYI, NPM, TH, RES, WC>& sm,
                                                     const BcClass* bc = nullptr, int nbc = 0)
{
    using SMT = ZSmem<Q, T, TYI, NPM, TH, RES, WC>;
    int staged = 0;
    if constexpr (SMT::CT > 0) {
        staged = nbc < SMT::CT ? nbc : SMT::CT;
        const float4* src = reinterpret_cast<const float4*>(bc);
        float4* dst = reinterpret_cast<float4*>(dyn_smem() + 128);
        const int n = staged * (int)(sizeof(BcClass) / 16);
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    if (threadIdx.x == 0) {
        *reinterpret_cast<int*>(sm.bars + NSTAGE_MAX) = 0;  // the timeout flag
        *reinterpret_cast<int*>(dyn_smem() + HDR_STAGED_CLASSES) = staged;
        for (int s = 0; s < SMT::NS; s++) mbar_init(&sm.bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// Tile-ordered steps.  Each launch of the single-domain step may begin while
// the launch before it is still finishing (programmatic dependent launch):
// instead of waiting for the whole previous grid, a tile waits only for the
// previous step's tiles it reads from or writes over, so the SMs that the
// previous step's last CTAs leave idle already run the next step.  State
// (sched): a 64-bit ticket counter, then one word per tile (x tile, y tile,
// z chunk) holding 1 + the last step that finished it.  A CTA takes ticket
// t: step s = t / tiles, work index w = t % tiles; tickets follow the CTAs'
// start order, and every CTA of a launch holds its ticket before the next
// launch starts.  Work index w is column w % columns (x tiles fastest, as the
// plain grid runs) of chunk (w / columns + s) % chunks: each step starts one
// chunk further on, so its first tiles need the previous step's first
// finished chunks (a periodic z axis makes chunk 0 read the last chunk's
// ghost plane).  A tile of step s reads planes z0 - 1 .. z1 and rows and
// columns one node beyond its own, and writes its nodes plus their ghost
// copies, so it waits for the 27 tiles around it (periodic wrap included,
// which also covers every ghost copy) to hold s; waiting for them to finish
// step s - 1 covers both their writes of the buffer it reads and their reads
// of the buffer it writes.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Takes the CTA's ticket and waits for the tiles around its tile; returns the
// step index and sets the tile.  Ends with no CTA barrier: the caller's next
// one orders the waits before the tile's first load.
__device__ __forceinline__ unsigned tile_order_begin(const StepArgs& a, int& tx, int& ty, int& kc)
{
    unsigned* hdr = reinterpret_cast<unsigned*>(dyn_smem() + HDR_TICKET);
    const unsigned ncol = gridDim.x * gridDim.y, ntile = ncol * gridDim.z;
    if (threadIdx.x == 0) {
        const unsigned long long t = atomicAdd(reinterpret_cast<unsigned long long*>(a.sched), 1ull);
        hdr[0] = (unsigned)(t % ntile);
        hdr[1] = (unsigned)(t / ntile);
    }
    __syncthreads();
    const unsigned w = hdr[0], s = hdr[1];
    // every CTA of this launch holds its ticket: the next launch may start
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned col = w % ncol;
    tx = (int)(col % gridDim.x);
    ty = (int)(col / gridDim.x);
    kc = (int)((w / ncol + s) % gridDim.z);
    if (threadIdx.x < 27) {
        const int dx = (int)threadIdx.x % 3 - 1, dy = (int)threadIdx.x / 3 % 3 - 1, dz = (int)threadIdx.x / 9 - 1;
        const int nx = (tx + dx + (int)gridDim.x) % (int)gridDim.x;
        const int ny = (ty + dy + (int)gridDim.y) % (int)gridDim.y;
        const int nz = (kc + dz + (int)gridDim.z) % (int)gridDim.z;
        const unsigned* f = a.sched + 2 + ((size_t)nz * gridDim.y + ny) * gridDim.x + nx;
        bool ok = false;
        for (unsigned it = 0; it < DEP_LIMIT; it++) {
            if ((int)(ld_acquire_u32(f) - s) >= 0) {
                ok = true;
                break;
            }
            // another tile gave up already: so does this one, at once
            if ((it & 1023u) == 1023u && (*reinterpret_cast<volatile int*>(a.err) & 4)) break;
            __nanosleep(64);
        }
        // on a timeout the step runs on (its result is flagged), so the
        // tiles waiting on this one do not time out in turn
        if (!ok) atomicOr(a.err, 4);
    }
    return s;
}

// Marks the CTA's tile done with step s; called after a CTA barrier that
// follows the tile's last global store.
__device__ __forceinline__ void tile_order_end(const StepArgs& a, int tx, int ty, int kc, unsigned s)
{
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned* f = a.sched + 2 + ((size_t)kc * gridDim.y + ty) * gridDim.x + tx;
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(f), "r"(s + 1u) : "memory");
    }
}

// Single-domain step: one CTA per (x tile, y tile, z chunk of lz planes).
// Launch order runs x tiles fastest, so the CTAs resident at one time march
// neighbouring columns through the same planes and their halo reads hit L2.
// With a.sched set, a CTA's tile comes from its ticket instead (tile_order_begin).
template <int Q, typename T, int FLAGS, int TYI, typename BCP = TableBC>
__global__ void __launch_bounds__(32 * (TYI + 2), ctas_per_sm(TYI))
    zmarch_step(const __grid_constant__ CUtensorMap map_in, const StepArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr bool WC = (FLAGS & F_BC) != 0 && stages_classes<BCP>::value;
    const ZSmem<Q, T, TYI, npairs_of(FLAGS), (FLAGS & F_THERMAL) != 0, 0, WC> sm(smem);
    int tx = blockIdx.x, ty = blockIdx.y, kc = blockIdx.z;
    unsigned s = 0;
    if (a.sched) s = tile_order_begin(a, tx, ty, kc);
    zmarch_init_barriers(sm, a.bc, a.nbc);  // ends with a CTA barrier
    // the tiles' stores of the previous step were made visible to this
    // thread through the generic proxy; the ring's loads use the async one
    if (a.sched) asm volatile("fence.proxy.async.global;" ::: "memory");
    unsigned g0 = 0;
    const int z0 = kc * a.lz;
    (void)zmarch_column<Q, T, FLAGS, TYI, BCP>(a, &map_in, tx * TILE_X, ty * TYI, z0, min(z0 + a.lz, a.nz), sm, g0);
    // zmarch_column ends with a CTA barrier on every path
    if (a.sched) tile_order_end(a, tx, ty, kc, s);
}

// Grid of the single-domain step.
__host__ __device__ inline dim3 zmarch_grid(int nx, int ny, int nz, int tyi, int lz)
{
    return dim3((nx + TILE_X - 1) / TILE_X, (ny + tyi - 1) / tyi, (nz + lz - 1) / lz);
}

template <int Q, typename T, int FLAGS, int TYI, typename BCP = TableBC>
constexpr size_t step_smem_bytes()
{
    return ZSmem<Q, T, TYI, npairs_of(FLAGS), (FLAGS & F_THERMAL) != 0, 0,
                 (FLAGS & F_BC) != 0 && stages_classes<BCP>::value>::bytes;
}

}  // namespace mrlbm
