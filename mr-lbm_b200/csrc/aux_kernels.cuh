// aux_kernels.cuh -- initial state, layout conversion, FP64 reductions.
#pragma once
#include "kernels.cuh"

namespace mrlbm {

// Stored moments from physical rho, u exactly as the reference's
// gpuInitialization_mom (src/lbmInitialization.cu:28-131): an equilibrium
// with weight*RHO_0, second moments summed over the first `qs` velocities
// (19 reproduces the reference, which uses the D3Q19 sums also on D3Q27).
template <int Q>
__device__ __forceinline__ void init_moments(float rho, float ux, float uy, float uz, float rho0, int qs,
                                             float* m)
{
    const float uu = ux * ux + uy * uy + uz * uz;
    const float p1muu = 1.0f - 1.5f * uu;
    float pxx = 0.f, pxy = 0.f, pxz = 0.f, pyy = 0.f, pyz = 0.f, pzz = 0.f;
#pragma unroll
    for (int i = 0; i < Q; i++) {
        if (i >= qs) break;
        const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        const float uc3 = 3.0f * (ux * cx + uy * cy + uz * cz);
        const float f = ((float)lat_w(Q, i) * rho0) * (p1muu + uc3 * (1.0f + uc3 * 0.5f));
        pxx += f * (cx * cx); pxy += f * (cx * cy); pxz += f * (cx * cz);
        pyy += f * (cy * cy); pyz += f * (cy * cz); pzz += f * (cz * cz);
    }
    const float ir = 1.0f / rho;
    m[0] = rho - rho0;
    m[1] = 3.0f * ux; m[2] = 3.0f * uy; m[3] = 3.0f * uz;
    m[4] = 4.5f * (pxx * ir - (1.0f / 3.0f));
    m[5] = 9.0f * (pxy * ir);
    m[6] = 9.0f * (pxz * ir);
    m[7] = 4.5f * (pyy * ir - (1.0f / 3.0f));
    m[8] = 9.0f * (pyz * ir);
    m[9] = 4.5f * (pzz * ir - (1.0f / 3.0f));
}

struct InitArgs {
    void* m0;
    void* m1;
    int nx, ny, nz, pitch;
    long long plane, field;
    int nm, qs;
    float rho0, omega0;
    int kind;  // 0: host fields, 1: uniform, 2: Taylor-Green
    const float *rho, *ux, *uy, *uz;  // device copies of x-fastest fields (kind 0)
    float u0[3];
    float tg_u0, tg_L;
    int thermal;  // moments 10..13 are C and its flux: C = c0, no flux
    float c0;     // (the thermal cases' flow_initialization.inc: cVar = T_REFERENCE, q = 0)
    int lo0;      // split storage: stored word of the low part of 3u_x (-1: none)
    int lom;      // split storage: stored word of the low part of omega (-1: none)
    float scale[NM_MAX];
};

// Split velocity: the part of 3u that its fp16 high word (storage scale s)
// rounds away, stored in the low word.
__device__ __forceinline__ float split_low(float u3, float s)
{
    return u3 - __half2float(__float2half_rn(u3 * s)) / s;
}

template <int Q, typename T>
__global__ void init_kernel(const InitArgs a)
{
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n;
         g += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(g % a.nx);
        const int y = (int)((g / a.nx) % a.ny);
        const int z = (int)(g / ((long long)a.nx * a.ny));
        float rho, ux, uy, uz;
        if (a.kind == 0) {
            rho = a.rho[g]; ux = a.ux[g]; uy = a.uy[g]; uz = a.uz[g];
        } else if (a.kind == 1) {
            rho = a.rho0; ux = a.u0[0]; uy = a.u0[1]; uz = a.u0[2];
        } else {
            // src/cases/taylorGreen/flow_initialization.inc:1-4 (cs2 = 1/3)
            const float L = a.tg_L, U = a.tg_u0;
            rho = a.rho0 + (1.0f / (16.0f * (1.0f / 3.0f))) * a.rho0 * U * U *
                               (cosf(2.0f * x / L) + cosf(2.0f * y / L)) * (cosf(2.0f * z / L) + 2.0f);
            ux = U * sinf(x / L) * cosf(y / L) * cosf(z / L);
            uy = -U * cosf(x / L) * sinf(y / L) * cosf(z / L);
            uz = 0.0f;
        }
        float m[NM_MAX];
        init_moments<Q>(rho, ux, uy, uz, a.rho0, a.qs, m);
        if (a.thermal) {
            m[10] = a.c0;
            m[11] = m[12] = m[13] = 0.f;
        } else {
            m[10] = a.omega0;
        }
        if (a.lo0 >= 0)
            for (int c = 0; c < 3; c++) m[a.lo0 + c] = split_low(m[1 + c], a.scale[1 + c]);
        if (a.lom >= 0) m[a.lom] = split_low(m[10], a.scale[10]);
        const long long idx = pidx(x, y, z, a.pitch, a.plane);
        T* p0 = reinterpret_cast<T*>(a.m0);
        T* p1 = reinterpret_cast<T*>(a.m1);
        for (int k = 0; k < a.nm; k++) {
            const float v = is_f32<T>() ? m[k] : m[k] * a.scale[k];
            Stor<T>::st(p0 + mphys(k, idx, a.field), v);
            Stor<T>::st(p1 + mphys(k, idx, a.field), v);
        }
    }
}

// Conversion between the planar storage and float views:
//   mode 0: planar -> float [m][z][y][x]      mode 1: float [m][z][y][x] -> planar (both buffers)
//   mode 2: planar -> reference idxMom layout mode 3: reference idxMom -> planar (both buffers)
struct ConvArgs {
    void* m0;
    void* m1;
    float* f;
    int nx, ny, nz, pitch;
    long long plane, field;
    int nm, mode;
    int lo0;  // split storage: stored word of the low part of 3u_x (-1: none)
    int lom;  // split storage: stored word of the low part of omega (-1: none)
    float scale[NM_MAX], iscale[NM_MAX];
};

template <typename T>
__global__ void convert_kernel(const ConvArgs a)
{
    const long long n = (long long)a.nx * a.ny * a.nz;
    const int nbx = a.nx / 8, nby = a.ny / 8;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n * a.nm;
         g += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(g / n);
        const long long node = g % n;
        const int x = (int)(node % a.nx);
        const int y = (int)((node / a.nx) % a.ny);
        const int z = (int)(node / ((long long)a.nx * a.ny));
        const long long idx = mphys(k, pidx(x, y, z, a.pitch, a.plane), a.field);
        long long fi;
        if (a.mode < 2) {
            fi = g;
        } else {
            // idxMom: tx + 8*(ty + 8*(tz + 8*(mom + NM*(bx + NBX*(by + NBY*bz)))))
            const long long blk = (x >> 3) + (long long)nbx * ((y >> 3) + (long long)nby * (z >> 3));
            fi = (x & 7) + 8 * ((y & 7) + 8 * ((z & 7) + 8 * (k + (long long)a.nm * blk)));
        }
        // split storage: 3u (and omega) = high word + low word
        const int lw = (a.lo0 >= 0 && k >= 1 && k <= 3) ? a.lo0 + k - 1 : (a.lom >= 0 && k == 10 ? a.lom : -1);
        const bool split = lw >= 0;
        const long long lidx = split ? mphys(lw, pidx(x, y, z, a.pitch, a.plane), a.field) : 0;
        if (a.mode == 0 || a.mode == 2) {
            const float v = Stor<T>::ld(reinterpret_cast<const T*>(a.m0) + idx);
            float r = is_f32<T>() ? v : v * a.iscale[k];
            if (split) r += Stor<T>::ld(reinterpret_cast<const T*>(a.m0) + lidx) * a.iscale[lw];
            a.f[fi] = r;
        } else {
            const float v = is_f32<T>() ? a.f[fi] : a.f[fi] * a.scale[k];
            Stor<T>::st(reinterpret_cast<T*>(a.m0) + idx, v);
            Stor<T>::st(reinterpret_cast<T*>(a.m1) + idx, v);
            if (split) {
                const float lo = split_low(a.f[fi], a.scale[k]) * a.scale[lw];
                Stor<T>::st(reinterpret_cast<T*>(a.m0) + lidx, lo);
                Stor<T>::st(reinterpret_cast<T*>(a.m1) + lidx, lo);
            }
        }
    }
}

// Ghost shell of the padded layout: periodic axes copy the wrapped interior,
// wall axes hold the exterior state (the reference's stale initial ghost
// populations at walls, src/includeFiles/interface.h:6-19).  Applied to both
// ping-pong buffers after any host-side change of the moments.
struct GhostArgs {
    void* m0;
    void* m1;
    int nx, ny, nz, pitch;
    long long plane, field;
    int nm, periodic;
    float ext[NM_MAX];
    float scale[NM_MAX];
};

template <typename T>
__global__ void ghost_fill_kernel(const GhostArgs a)
{
    const long long ex = a.nx + 2, ey = a.ny + 2, ez = a.nz + 2;
    const long long n = ex * ey * ez;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(g % ex) - 1;
        const int y = (int)((g / ex) % ey) - 1;
        const int z = (int)(g / (ex * ey)) - 1;
        const bool in_x = x >= 0 && x < a.nx, in_y = y >= 0 && y < a.ny, in_z = z >= 0 && z < a.nz;
        if (in_x && in_y && in_z) continue;
        bool wall = false;
        int sx = x, sy = y, sz = z;
        if (!in_x) { if (a.periodic & 1) sx = (x + a.nx) % a.nx; else wall = true; }
        if (!in_y) { if (a.periodic & 2) sy = (y + a.ny) % a.ny; else wall = true; }
        if (!in_z) { if (a.periodic & 4) sz = (z + a.nz) % a.nz; else wall = true; }
        const long long di = pidx(x, y, z, a.pitch, a.plane);
        T* p0 = reinterpret_cast<T*>(a.m0);
        T* p1 = reinterpret_cast<T*>(a.m1);
        if (wall) {
            for (int k = 0; k < a.nm; k++) {
                const float v = is_f32<T>() ? a.ext[k] : a.ext[k] * a.scale[k];
                Stor<T>::st(p0 + mphys(k, di, a.field), v);
                Stor<T>::st(p1 + mphys(k, di, a.field), v);
            }
        } else {
            const long long si = pidx(sx, sy, sz, a.pitch, a.plane);
            for (int k = 0; k < a.nm; k++) {
                p0[mphys(k, di, a.field)] = p0[mphys(k, si, a.field)];
                p1[mphys(k, di, a.field)] = p0[mphys(k, si, a.field)];
            }
        }
    }
}

// FP64 block partial sums over non-solid nodes:
//   [0] rho, [1..3] rho u, [4] rho |u|^2 / 2, [5] fluid nodes, [6] max |u|,
//   [7] non-finite moments.  (src/reduction.cu:100-155 in double.)
// Partials go to a scratch array of gridDim.x * 8 doubles; reduce_finish sums
// them in a fixed order, so results are deterministic.
constexpr int RED_THREADS = 256;

struct RedArgs {
    const void* m;
    const uint8_t* cls;
    int has_cls;
    int nx, ny, nz, pitch;
    long long plane, field;
    int nm;
    int lo0;  // split velocity: stored word of the low part of 3u_x (-1: none)
    float rho0;
    float iscale[NM_MAX];
    double* partial;
    double* out;
    int nblocks;
    // residual: ||u - usnap||^2 and ||u||^2, snapshot update
    float* usnap;
    int residual_mode;  // 0 none, 1 accumulate residual sums, 2 snapshot only
};

template <typename T>
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(const RedArgs a)
{
    __shared__ double sh[RED_THREADS / 32][8];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long long n = (long long)a.nx * a.ny * a.nz;
    const T* mp = reinterpret_cast<const T*>(a.m);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(g % a.nx);
        const int y = (int)((g / a.nx) % a.ny);
        const int z = (int)(g / ((long long)a.nx * a.ny));
        const long long idx = pidx(x, y, z, a.pitch, a.plane);
        if (a.has_cls && a.cls[idx] == CLS_SOLID) continue;
        float v[4];
        bool finite = true;
        for (int k = 0; k < 4; k++) {
            const float s = Stor<T>::ld(mp + mphys(k, idx, a.field));
            v[k] = is_f32<T>() ? s : s * a.iscale[k];
            if (k >= 1 && a.lo0 >= 0) v[k] += Stor<T>::ld(mp + mphys(a.lo0 + k - 1, idx, a.field)) * a.iscale[a.lo0 + k - 1];
            finite = finite && isfinite(v[k]);
        }
        const double rho = (double)a.rho0 + (double)v[0];
        const double ux = v[1] / 3.0, uy = v[2] / 3.0, uz = v[3] / 3.0;
        const double u2 = ux * ux + uy * uy + uz * uz;
        if (a.residual_mode == 0) {
            acc[0] += rho;
            acc[1] += rho * ux; acc[2] += rho * uy; acc[3] += rho * uz;
            acc[4] += 0.5 * rho * u2;
            acc[5] += 1.0;
            acc[6] = fmax(acc[6], finite ? sqrt(u2) : INFINITY);
            acc[7] += finite ? 0.0 : 1.0;
        } else {
            float* us = a.usnap + 3 * g;
            if (a.residual_mode == 1) {
                const double dx = ux - us[0], dy = uy - us[1], dz = uz - us[2];
                acc[0] += dx * dx + dy * dy + dz * dz;
                acc[1] += u2;
            }
            us[0] = (float)ux; us[1] = (float)uy; us[2] = (float)uz;
        }
    }
    // warp then block reduction, fixed order
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 8; k++) {
        double v = acc[k];
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, v, off);
            v = (k == 6) ? fmax(v, o) : v + o;
        }
        if (lane == 0) sh[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int k = threadIdx.x;
        double v = sh[0][k];
        for (int i = 1; i < RED_THREADS / 32; i++) v = (k == 6) ? fmax(v, sh[i][k]) : v + sh[i][k];
        a.partial[blockIdx.x * 8 + k] = v;
    }
}

__global__ void reduce_finish(const double* partial, int nblocks, double* out)
{
    const int k = threadIdx.x;
    if (k >= 8) return;
    double v = (k == 6) ? 0.0 : 0.0;
    for (int b = 0; b < nblocks; b++) v = (k == 6) ? fmax(v, partial[b * 8 + k]) : v + partial[b * 8 + k];
    out[k] = v;
}

}  // namespace mrlbm
