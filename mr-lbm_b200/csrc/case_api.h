// case_api.h -- the environment a reference case directory's snippets expect
// (the names they read from the reference's var.h, definitions.h,
// nodeTypeMap.h and velocity-set files), so an existing
// src/cases/<case>/*.inc compiles unchanged into this library's kernels.
//
// Include order in a case driver (see casebuild.py):
//   case_api.h (CASE_API_PRE) -> model.inc -> case_api.h (CASE_API_LATTICE)
//   -> constants.inc -> output.inc -> case_api.h (CASE_API_POST)
#if defined(CASE_API_PRE)
#undef CASE_API_PRE
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <limits>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef float dfloat;  // the reference's SINGLE_PRECISION build

#define STR_IMPL(A) #A
#define STR(A) STR_IMPL(A)
#ifndef myMax
#define myMax(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef myMin
#define myMin(a, b) (((a) < (b)) ? (a) : (b))
#endif

// compile-time square roots used by some constants.inc files
constexpr double case_api_sqrt_iter(double x, double cur, double prev)
{
    return cur == prev ? cur : case_api_sqrt_iter(x, 0.5 * (cur + x / cur), cur);
}
constexpr dfloat sqrtt(dfloat x)
{
    return (x >= 0 && x < std::numeric_limits<dfloat>::infinity()) ? (dfloat)case_api_sqrt_iter(x, x > 1 ? x : 1, 0)
                                                                    : std::numeric_limits<dfloat>::quiet_NaN();
}
constexpr dfloat invSqrtt(dfloat x) { return (dfloat)(1.0 / (double)sqrtt(x)); }

// node-type words: octant mask o = ox + 2 oy + 4 oz (o_a = 1 on the + side)
// of solid neighbours, BC kind in bits 8-10, velocity index in bits 11-12
constexpr unsigned int BULK = 0x00u;
constexpr unsigned int WEST = 0x55u, EAST = 0xAAu, SOUTH = 0x33u, NORTH = 0xCCu, BACK = 0x0Fu, FRONT = 0xF0u;
constexpr unsigned int NORTH_WEST = NORTH | WEST, NORTH_EAST = NORTH | EAST, NORTH_FRONT = NORTH | FRONT,
                       NORTH_BACK = NORTH | BACK, SOUTH_WEST = SOUTH | WEST, SOUTH_EAST = SOUTH | EAST,
                       SOUTH_FRONT = SOUTH | FRONT, SOUTH_BACK = SOUTH | BACK, WEST_FRONT = WEST | FRONT,
                       WEST_BACK = WEST | BACK, EAST_FRONT = EAST | FRONT, EAST_BACK = EAST | BACK;
constexpr unsigned int NORTH_WEST_FRONT = NORTH | WEST | FRONT, NORTH_WEST_BACK = NORTH | WEST | BACK,
                       NORTH_EAST_FRONT = NORTH | EAST | FRONT, NORTH_EAST_BACK = NORTH | EAST | BACK,
                       SOUTH_WEST_FRONT = SOUTH | WEST | FRONT, SOUTH_WEST_BACK = SOUTH | WEST | BACK,
                       SOUTH_EAST_FRONT = SOUTH | EAST | FRONT, SOUTH_EAST_BACK = SOUTH | EAST | BACK;
constexpr unsigned int SOLID_NODE = 0xFFu;
constexpr unsigned int BC_ZERO_VELOCITY_WALL = 0u << 8, BC_VELOCITY_WALL = 1u << 8, BC_OUTFLOW = 2u << 8,
                       BC_SYMMETRY = 3u << 8, BC_FREESLIP = 4u << 8;
constexpr unsigned int BC_VELOCITY_INDEX_0 = 0u << 11, BC_VELOCITY_INDEX_1 = 1u << 11, BC_VELOCITY_INDEX_2 = 2u << 11,
                       BC_VELOCITY_INDEX_3 = 3u << 11;
constexpr unsigned int MISSING_DEFINITION = 0xFFFFFFFFu;

#elif defined(CASE_API_LATTICE)
#undef CASE_API_LATTICE
// velocity set selected by the case's model.inc (D3Q19 or D3Q27); ordering
// as the case API's pop[i] expects
#if defined(D3Q19)
constexpr unsigned char Q = 19;
constexpr unsigned char QF = 5;
constexpr dfloat W0 = 1.0 / 3, W1 = 1.0 / 18, W2 = 1.0 / 36;
__device__ const dfloat w[Q] = {W0, W1, W1, W1, W1, W1, W1, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2};
#elif defined(D3Q27)
constexpr unsigned char Q = 27;
constexpr unsigned char QF = 9;
constexpr dfloat W0 = 8.0 / 27, W1 = 2.0 / 27, W2 = 1.0 / 54, W3 = 1.0 / 216;
__device__ const dfloat w[Q] = {W0, W1, W1, W1, W1, W1, W1, W2, W2, W2, W2, W2, W2, W2,
                                W2, W2, W2, W2, W2, W3, W3, W3, W3, W3, W3, W3, W3};
#else
#error "case model.inc must define D3Q19 or D3Q27"
#endif
__device__ const char cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
__device__ const char cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
__device__ const char cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
constexpr dfloat as2 = 3.0;
constexpr dfloat cs2 = 1.0 / as2;
constexpr dfloat F_M_0_SCALE = 1.0, F_M_I_SCALE = as2, F_M_II_SCALE = as2 * as2 / 2, F_M_IJ_SCALE = as2 * as2;

#elif defined(CASE_API_POST)
#undef CASE_API_POST
// relaxation constants every case may read
constexpr dfloat OMEGA = 1.0 / TAU;
constexpr dfloat OMEGAd2 = OMEGA / 2.0, OMEGAd9 = OMEGA / 9.0, T_OMEGA = 1.0 - OMEGA, TT_OMEGA = 1.0 - 0.5 * OMEGA;
constexpr dfloat OMEGA_P1 = 1.0 + OMEGA, TT_OMEGA_T3 = TT_OMEGA * 3.0;
constexpr dfloat ONESIXTH = 1.0 / 6.0, ONETHIRD = 1.0 / 3.0;
// non-Newtonian model parameters (the reference's defaults when a case
// selects the model without setting them)
#if defined(POWERLAW)
#ifndef CASE_N_INDEX
constexpr dfloat N_INDEX = 0.5;
#else
constexpr dfloat N_INDEX = CASE_N_INDEX;
#endif
constexpr dfloat K_CONSISTENCY = RHO_0 * (TAU - 0.5) / 3;
constexpr dfloat GAMMA_0 = 0;
#define OMEGA_FIELD
#endif
#if defined(BINGHAM)
constexpr dfloat OMEGA_P = (dfloat)(1.0) / (3.0 * VISC + 0.5);
#define OMEGA_FIELD
#endif
#ifndef COLLISION_TYPE
#error "case model.inc must define COLLISION_TYPE"
#endif
#define CASE_API_COLLISION_MR_LBM 1
// moment indices of fMom (src/arrayIndex.h:8-50): the flow's, omega, then the
// thermal scalar's
constexpr int M_RHO_INDEX = 0, M_UX_INDEX = 1, M_UY_INDEX = 2, M_UZ_INDEX = 3, M_MXX_INDEX = 4, M_MXY_INDEX = 5,
              M_MXZ_INDEX = 6, M_MYY_INDEX = 7, M_MYZ_INDEX = 8, M_MZZ_INDEX = 9;
#if defined(OMEGA_FIELD)
constexpr int M_OMEGA_INDEX = 10;
constexpr int CASE_API_M_NEXT = 11;
#else
constexpr int CASE_API_M_NEXT = 10;
#endif
#if defined(SECOND_DIST)
constexpr int M2_C_INDEX = CASE_API_M_NEXT, M2_CX_INDEX = CASE_API_M_NEXT + 1, M2_CY_INDEX = CASE_API_M_NEXT + 2,
              M2_CZ_INDEX = CASE_API_M_NEXT + 3;
// D3G19 weights (src/includeFiles/velocitySets/D3G19.inc)
constexpr unsigned char GQ = 19;
constexpr dfloat gW0 = 1.0 / 3, gW1 = 1.0 / 18, gW2 = 1.0 / 36;
#endif
#endif
