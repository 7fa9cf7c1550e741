// lattice.cuh -- compile-time D3Q19 / D3Q27 velocity sets.
//
// Velocity ordering and weights follow the reference's velocity-set files
// (src/includeFiles/velocitySets/D3Q19.inc:8-19, D3Q27.inc:9-22): index i and
// i+1 are opposite for every odd i, D3Q19 is the first 19 entries of D3Q27.
// The ordering is part of the case API (bc_definition snippets index pop[i]),
// so it is kept identical.
#pragma once
#include <cstdint>
#include <utility>

namespace mrlbm {

__host__ __device__ constexpr int lat_cx(int i)
{
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int lat_cy(int i)
{
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int lat_cz(int i)
{
    constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int lat_norm2(int i)
{
    return lat_cx(i) * lat_cx(i) + lat_cy(i) * lat_cy(i) + lat_cz(i) * lat_cz(i);
}
// weight class: 0 rest, 1 axis, 2 face diagonal, 3 corner
__host__ __device__ constexpr double lat_w(int Q, int i)
{
    return Q == 19 ? (lat_norm2(i) == 0 ? 1.0 / 3.0 : lat_norm2(i) == 1 ? 1.0 / 18.0 : 1.0 / 36.0)
                   : (lat_norm2(i) == 0 ? 8.0 / 27.0
                      : lat_norm2(i) == 1 ? 2.0 / 27.0
                      : lat_norm2(i) == 2 ? 1.0 / 54.0
                                          : 1.0 / 216.0);
}

// Number of directions with c_y != 0 (exchanged between warps through shared
// memory in the z-marching kernel) and the slot of direction i among them.
__host__ __device__ constexpr int lat_num_cy(int Q)
{
    int n = 0;
    for (int i = 0; i < Q; i++) n += lat_cy(i) != 0;
    return n;
}
__host__ __device__ constexpr int lat_cy_slot(int Q, int i)
{
    int n = 0;
    for (int j = 0; j < i && j < Q; j++) n += lat_cy(j) != 0;
    return n;
}
// Number of directions with c_z == +1 (or -1), i.e. populations that cross
// from one z plane to the next.
__host__ __device__ constexpr int lat_num_cz(int Q, int s)
{
    int n = 0;
    for (int i = 0; i < Q; i++) n += lat_cz(i) == s;
    return n;
}
__host__ __device__ constexpr int lat_cz_slot(int Q, int i)
{
    int n = 0;
    for (int j = 0; j < i; j++) n += lat_cz(j) == lat_cz(i);
    return n;
}

// Index of the direction (cx, cy, cz) in the first Q entries, -1 if absent.
__host__ __device__ constexpr int lat_find(int Q, int cx, int cy, int cz)
{
    for (int i = 0; i < Q; i++)
        if (lat_cx(i) == cx && lat_cy(i) == cy && lat_cz(i) == cz) return i;
    return -1;
}

// Compile-time loop: f(std::integral_constant<int, I>) for I = B .. E-1, so
// every lattice index (and everything computed from it) is a constant
// expression and register arrays indexed by it never spill to local memory.
template <int B, typename F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>)
{
    (f(std::integral_constant<int, B + Is>{}), ...);
}
template <int B, int E, typename F>
__host__ __device__ __forceinline__ void static_for(F&& f)
{
    static_for_impl<B>(f, std::make_integer_sequence<int, E - B>{});
}

}  // namespace mrlbm
