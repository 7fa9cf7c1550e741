// kernels.cuh -- device code of the fused MR-LBM collide-stream step.
//
// One step of the moment-representation LBM (the reference's
// gpuMomCollisionStream, src/mlbm.cu:3-714) computes, for every fluid node x,
//   f_i*(x) = f_i^post(x - c_i)   with f^post reconstructed from the stored
//                                 post-collision moments of the source node,
// then the new moments (bulk sums, or the moment-space wall BC), and collides
// them in moment space.  Only the 10 (11) moments live in HBM.
//
// B200 design (z-marching, ping-pong moments):
//   * A CTA owns a column of 30 x TYI interior nodes in (x, y) and a chunk of
//     LZ planes in z.  Warp w holds row y = Y0 - 1 + w, lane l holds
//     x = X0 - 1 + l: the outer lanes / warps are the one-node halo.
//   * Each production step reads the moments of one (x, y) plane (coalesced,
//     prefetched one plane ahead) and reconstructs the post-collision
//     populations of every node of the plane in registers.
//   * Populations that move in x only are exchanged with warp shuffles,
//     populations that move in y go through a double-buffered shared-memory
//     row exchange (one __syncthreads per plane), populations that move in z
//     stay in registers: a plane's c_z=+1 populations are held until the next
//     plane, its c_z=0 ones until the output of the same plane is formed one
//     step later.  Output plane z is completed when plane z+1 is produced.
//   * Moments are read from one buffer and written to the other, so halo
//     moments are always the previous step's (no ghost-population arrays, no
//     per-step host sync).  DRAM traffic is the algorithmic 2*M*s bytes per
//     node plus halo re-reads that mostly hit L2.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>

#include "lattice.cuh"

namespace mrlbm {

enum : int {
    F_BC = 1,        // node classes present (walls, solids, velocity BCs)
    F_FORCE = 2,     // non-zero body force
    F_POWERLAW = 4,  // omega field, power-law viscosity
    F_BINGHAM = 8,   // omega field, Bingham viscosity
};

constexpr int TILE_X = 30;  // interior nodes per warp row
constexpr uint8_t CLS_BULK = 0;
constexpr uint8_t CLS_SOLID = 255;

// Moment-space wall BC data of one node class (octant mask + velocity index).
// The BC is the linear system
//   sum_I f_i          = sum_I f^reg_i(rho, u, (1-w) Pi + w u u)
//   sum_I f_i h_k(c_i) = sum_I h_k(c_i) f^reg_i(rho, u, Pi)
// in X = (rho, rho*Pi).  Its matrix is A(w) = A(w0) + (w - w0) e0 q^T, so the
// host stores Ainv = A(w0)^-1, v = Ainv e0, qa = q^T Ainv, s = q^T Ainv e0 and
// the device applies Sherman-Morrison for a per-node omega.
struct BcClass {
    float ainv[49];
    float v[7];
    float qa[7];
    float s;
    float u[3];        // prescribed wall velocity (unscaled)
    uint32_t known;    // bit i: population i is known (incoming from fluid)
    uint32_t valid;
};

struct StepArgs {
    const void* __restrict__ m_in;  // [nm][nz][ny][pitch] storage type
    void* __restrict__ m_out;
    const uint8_t* __restrict__ cls;  // [nz][ny][pitch]
    const BcClass* __restrict__ bc;
    int nx, ny, nz, pitch;
    long long plane, field;  // elements
    int periodic;            // bit a set: axis a periodic
    int lz;                  // planes per CTA
    float rho0, omega0;
    float fx, fy, fz;
    float nnf_n, nnf_k, nnf_yield, nnf_omega_p;
    float ext[11];     // stored-moment state of sources outside wall axes
    float scale[11];   // storage scale per moment (1 for fp32)
    float iscale[11];
};

// ------------------------------------------------------------------ storage

template <typename T>
struct Stor;
template <>
struct Stor<float> {
    static __device__ __forceinline__ float ld(const float* p) { return __ldg(p); }
    static __device__ __forceinline__ void st(float* p, float v) { *p = v; }
};
template <>
struct Stor<__half> {
    static __device__ __forceinline__ float ld(const __half* p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }
};
template <>
struct Stor<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }
    static __device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

template <typename T>
constexpr bool is_f32()
{
    return sizeof(T) == 4;
}

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

// Raw sums over the lattice, pairwise: rho, j, and sum f c_a c_b.
template <int Q>
__device__ __forceinline__ void lattice_sums(const float* p, float& r, float* j, float* P)
{
    r = p[0];
    j[0] = j[1] = j[2] = 0.f;
#pragma unroll
    for (int k = 0; k < 6; k++) P[k] = 0.f;
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const float s = p[i] + p[i + 1], d = p[i] - p[i + 1];
        const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        r += s;
        if (cx > 0) j[0] += d; else if (cx < 0) j[0] -= d;
        if (cy > 0) j[1] += d; else if (cy < 0) j[1] -= d;
        if (cz > 0) j[2] += d; else if (cz < 0) j[2] -= d;
        if (cx != 0) P[0] += s;
        if (cy != 0) P[3] += s;
        if (cz != 0) P[5] += s;
        if (cx * cy > 0) P[1] += s; else if (cx * cy < 0) P[1] -= s;
        if (cx * cz > 0) P[2] += s; else if (cx * cz < 0) P[2] -= s;
        if (cy * cz > 0) P[4] += s; else if (cy * cz < 0) P[4] -= s;
    }
}

// mac = rho, u (unscaled), Pi_hat (unscaled xx,xy,xz,yy,yz,zz) from the
// known-set moment system of class c (the wall-node closed forms of the
// reference's bc_definition.inc, e.g. src/cases/lidDrivenCavity_3D/
// bc_definition.inc:637-663, solved generically).
template <int Q>
__device__ __forceinline__ void bc_moments(const BcClass* __restrict__ c, const float* p, float omega,
                                           float omega0, float* mac)
{
    const uint32_t known = __ldg(&c->known);
    float b0 = 0.f, sxx = 0.f, sxy = 0.f, sxz = 0.f, syy = 0.f, syz = 0.f, szz = 0.f;
#pragma unroll
    for (int i = 0; i < Q; i++) {
        const float v = ((known >> i) & 1u) ? p[i] : 0.f;
        const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        b0 += v;
        if (cx != 0) sxx += v;
        if (cy != 0) syy += v;
        if (cz != 0) szz += v;
        if (cx * cy > 0) sxy += v; else if (cx * cy < 0) sxy -= v;
        if (cx * cz > 0) sxz += v; else if (cx * cz < 0) sxz -= v;
        if (cy * cz > 0) syz += v; else if (cy * cz < 0) syz -= v;
    }
    const float third = b0 * (1.0f / 3.0f);
    const float b[7] = {b0, sxx - third, sxy, sxz, syy - third, syz, szz - third};
    float X[7];
    float dot = 0.f;
#pragma unroll
    for (int r = 0; r < 7; r++) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 7; k++) acc = fmaf(__ldg(&c->ainv[r * 7 + k]), b[k], acc);
        X[r] = acc;
        dot = fmaf(__ldg(&c->qa[r]), b[r], dot);
    }
    const float dw = omega - omega0;
    if (dw != 0.f) {
        const float corr = dw * dot / (1.0f + dw * __ldg(&c->s));
#pragma unroll
        for (int r = 0; r < 7; r++) X[r] = fmaf(-corr, __ldg(&c->v[r]), X[r]);
    }
    const float rho = X[0], ir = 1.0f / rho;
    mac[0] = rho;
    mac[1] = __ldg(&c->u[0]);
    mac[2] = __ldg(&c->u[1]);
    mac[3] = __ldg(&c->u[2]);
#pragma unroll
    for (int k = 0; k < 6; k++) mac[4 + k] = X[1 + k] * ir;
}

// Power-law omega by Newton iteration (src/nnf.h:61-89 with its compile
// defects fixed) and Bingham (src/nnf.h:92-98).
__device__ __forceinline__ float nnf_powerlaw(float omega_old, float smag, float n, float K, float rho0)
{
    if (smag < 1e-6f) return 0.f;
    float omega = omega_old;
    const float a = K * powf(smag / (rho0 * (1.0f / 3.0f)), n);
    const float b = 0.5f * smag, c = -smag;
    for (int it = 0; it < 7; it++) {
        const float on = powf(omega, n);
        const float fx = a * on + b * omega + c;
        const float dfx = a * n * powf(omega, n - 1.0f) + b;
        if (fabsf(fx / dfx) < 1e-6f) break;
        omega = omega - fx / dfx;
    }
    return omega;
}

// Scale to the stored form, update omega (non-Newtonian), collide
// (src/colrec/MR_LBM/collision.inc:2-14), write the 10/11 stored moments.
template <int FLAGS>
__device__ __forceinline__ void collide(const StepArgs& a, const float* mac, float omega, float* out)
{
    const float rho = mac[0];
    float ux = 3.0f * mac[1], uy = 3.0f * mac[2], uz = 3.0f * mac[3];
    float mxx = 4.5f * mac[4], mxy = 9.0f * mac[5], mxz = 9.0f * mac[6];
    float myy = 4.5f * mac[7], myz = 9.0f * mac[8], mzz = 4.5f * mac[9];
    const float Fx = (FLAGS & F_FORCE) ? a.fx : 0.f;
    const float Fy = (FLAGS & F_FORCE) ? a.fy : 0.f;
    const float Fz = (FLAGS & F_FORCE) ? a.fz : 0.f;
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
    const float ir = 1.0f / rho;
    const float t_om = 1.0f - omega, tt_om = 1.0f - 0.5f * omega, om_d2 = 0.5f * omega;
    if constexpr ((FLAGS & F_FORCE) != 0) {
        ux += 3.0f * ir * Fx;
        uy += 3.0f * ir * Fy;
        uz += 3.0f * ir * Fz;
        const float c15 = 1.5f * ir * tt_om, c3 = 3.0f * tt_om * ir;
        mxx = t_om * mxx + om_d2 * ux * ux + c15 * (2.0f * Fx * ux);
        myy = t_om * myy + om_d2 * uy * uy + c15 * (2.0f * Fy * uy);
        mzz = t_om * mzz + om_d2 * uz * uz + c15 * (2.0f * Fz * uz);
        mxy = t_om * mxy + omega * ux * uy + c3 * (Fx * uy + Fy * ux);
        mxz = t_om * mxz + omega * ux * uz + c3 * (Fx * uz + Fz * ux);
        myz = t_om * myz + omega * uy * uz + c3 * (Fy * uz + Fz * uy);
    } else {
        mxx = t_om * mxx + om_d2 * ux * ux;
        myy = t_om * myy + om_d2 * uy * uy;
        mzz = t_om * mzz + om_d2 * uz * uz;
        mxy = t_om * mxy + omega * ux * uy;
        mxz = t_om * mxz + omega * ux * uz;
        myz = t_om * myz + omega * uy * uz;
    }
    out[0] = rho - a.rho0;
    out[1] = ux; out[2] = uy; out[3] = uz;
    out[4] = mxx; out[5] = mxy; out[6] = mxz; out[7] = myy; out[8] = myz; out[9] = mzz;
    out[10] = omega;
}

// ---------------------------------------------------------- the step kernel

template <typename T, int NM>
__device__ __forceinline__ void load_node(const StepArgs& a, bool outside, long long idx, float* m)
{
    const T* base = reinterpret_cast<const T*>(a.m_in);
    if (outside) {
#pragma unroll
        for (int k = 0; k < NM; k++) m[k] = a.ext[k];
    } else {
#pragma unroll
        for (int k = 0; k < NM; k++) {
            const float v = Stor<T>::ld(base + k * a.field + idx);
            m[k] = is_f32<T>() ? v : v * a.iscale[k];
        }
    }
}

template <int Q, typename T, int FLAGS, int TYI>
__global__ void __launch_bounds__(32 * (TYI + 2), 1) zmarch_step(const StepArgs a)
{
    constexpr int NW = TYI + 2;
    constexpr int NCY = lat_num_cy(Q);
    constexpr int NUP = lat_num_cz(Q, 1);
    constexpr int NMID = lat_num_cz(Q, 0);
    constexpr bool OMF = (FLAGS & (F_POWERLAW | F_BINGHAM)) != 0;
    constexpr int NM = OMF ? 11 : 10;
    extern __shared__ float s_rows[];  // [2][NCY][NW][32]

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int X0 = blockIdx.x * TILE_X, Y0 = blockIdx.y * TYI, z0 = blockIdx.z * a.lz;
    const int x = X0 - 1 + lane, y = Y0 - 1 + warp;
    bool out_xy = false;
    int xs = x, ys = y;
    if (x < 0 || x >= a.nx) {
        if (a.periodic & 1) xs = (x + a.nx) % a.nx; else out_xy = true;
    }
    if (y < 0 || y >= a.ny) {
        if (a.periodic & 2) ys = (y + a.ny) % a.ny; else out_xy = true;
    }
    const bool interior = lane >= 1 && lane <= TILE_X && x < a.nx && warp >= 1 && warp <= TYI && y < a.ny;
    const long long rowoff = out_xy ? 0 : (long long)ys * a.pitch + xs;
    const int zend = min(z0 + a.lz, a.nz);
    const int nprod = zend - z0 + 2;
    T* outp = reinterpret_cast<T*>(a.m_out);

    auto src_index = [&](int zp, bool& outside) -> long long {
        outside = out_xy;
        int zs = zp;
        if (zp < 0 || zp >= a.nz) {
            if (a.periodic & 4) zs = (zp + a.nz) % a.nz; else outside = true;
        }
        return (long long)zs * a.plane + rowoff;
    };

    float mc[NM], mn[NM];
    {
        bool o;
        const long long id = src_index(z0 - 1, o);
        load_node<T, NM>(a, o, id, mc);
    }
    float up1[NUP], up2[NUP], mid[NMID];
    float om_prev = a.omega0;

    for (int k = 0; k < nprod; k++) {
        const int zp = z0 - 1 + k;
        if (k + 1 < nprod) {
            bool o;
            const long long id = src_index(zp + 1, o);
            load_node<T, NM>(a, o, id, mn);
        }
        float f[Q];
        reconstruct<Q>(mc, a.rho0, f);

        float* buf = s_rows + (k & 1) * (NCY * NW * 32);
#pragma unroll
        for (int i = 1; i < Q; i++)
            if (lat_cy(i) != 0) buf[(lat_cy_slot(Q, i) * NW + warp) * 32 + lane] = f[i];
        float g[Q];
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (lat_cy(i) == 0) {
                if (lat_cx(i) > 0) g[i] = __shfl_up_sync(0xffffffffu, f[i], 1);
                else if (lat_cx(i) < 0) g[i] = __shfl_down_sync(0xffffffffu, f[i], 1);
                else g[i] = f[i];
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 1; i < Q; i++) {
            if (lat_cy(i) != 0) {
                const int w = min(max(warp - lat_cy(i), 0), NW - 1);
                const int l = (lane - lat_cx(i)) & 31;
                g[i] = buf[(lat_cy_slot(Q, i) * NW + w) * 32 + l];
            }
        }

        if (k >= 2 && interior) {
            const int zd = zp - 1;
            const long long oidx = (long long)zd * a.plane + (long long)y * a.pitch + x;
            uint8_t cls = CLS_BULK;
            if constexpr ((FLAGS & F_BC) != 0) cls = __ldg(a.cls + oidx);
            if (cls != CLS_SOLID) {
                float p[Q];
#pragma unroll
                for (int i = 0; i < Q; i++) {
                    if (lat_cz(i) > 0) p[i] = up2[lat_cz_slot(Q, i)];
                    else if (lat_cz(i) == 0) p[i] = mid[lat_cz_slot(Q, i)];
                    else p[i] = g[i];
                }
                const float omega = OMF ? om_prev : a.omega0;
                float mac[10];
                if (cls == CLS_BULK) {
                    float r, j[3], P[6];
                    lattice_sums<Q>(p, r, j, P);
                    const float ir = 1.0f / r;
                    mac[0] = r;
                    mac[1] = j[0] * ir; mac[2] = j[1] * ir; mac[3] = j[2] * ir;
                    mac[4] = P[0] * ir - (1.0f / 3.0f);
                    mac[5] = P[1] * ir;
                    mac[6] = P[2] * ir;
                    mac[7] = P[3] * ir - (1.0f / 3.0f);
                    mac[8] = P[4] * ir;
                    mac[9] = P[5] * ir - (1.0f / 3.0f);
                } else {
                    bc_moments<Q>(a.bc + cls, p, omega, a.omega0, mac);
                }
                float o[11];
                collide<FLAGS>(a, mac, omega, o);
#pragma unroll
                for (int m = 0; m < NM; m++) {
                    const float v = is_f32<T>() ? o[m] : o[m] * a.scale[m];
                    Stor<T>::st(outp + m * a.field + oidx, v);
                }
            }
        }
        // rotate the z pipeline
#pragma unroll
        for (int s = 0; s < NUP; s++) up2[s] = up1[s];
#pragma unroll
        for (int i = 0; i < Q; i++) {
            if (lat_cz(i) > 0) up1[lat_cz_slot(Q, i)] = g[i];
            else if (lat_cz(i) == 0) mid[lat_cz_slot(Q, i)] = g[i];
        }
        if constexpr (OMF) om_prev = mc[NM - 1];
#pragma unroll
        for (int m = 0; m < NM; m++) mc[m] = mn[m];
    }
}

}  // namespace mrlbm
