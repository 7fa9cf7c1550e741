// ref_kat.cpp -- TEST INFRASTRUCTURE ONLY (builds oracle/_ref/libref_kat.so).
//
// Compiles the reference's own per-node arithmetic on the host, in FP64, so the
// oracle's restatement can be pinned against it (known-answer tests).  The
// reference snippets are #included from the reference tree at build time
// (-I <reference>/src); nothing from the reference is stored in this repository.
// Snippets used:
//   src/includeFiles/velocitySets/D3Q19.inc, D3Q27.inc     lattice constants
//   src/colrec/MR_LBM/reconstruction.inc                   population reconstruction
//   src/colrec/MR_LBM/collision.inc                        moment-space collision
//   src/nodeTypeMap.h                                      node type words
//   src/cases/lidDrivenCavity_3D/bc_definition.inc         26 wall cases + moving lid
//   src/cases/voxel/bc_definition.inc                      254 octant masks
//   src/cases/parallelPlates_D3Q27/bc_definition.inc       D3Q27 plate walls
//   src/includeFiles/velocitySets/D3G19.inc                thermal lattice weights
//   src/colrec/G_SCALAR/reconstruction.inc                 thermal population reconstruction
//   src/cases/rayleighBenard_Periodic/constants.inc        thermal case constants
//   src/cases/rayleighBenard_Periodic/bc_definition.inc    its wall closed forms
#include <cmath>
#include <cstdint>

#define __device__
typedef double dfloat;

#include "nodeTypeMap.h"

namespace q19 {
#include "includeFiles/velocitySets/D3Q19.inc"
}
namespace q27 {
#include "includeFiles/velocitySets/D3Q27.inc"
}

extern "C" {

// stored scaled moments m[10] -> populations f[Q]
void ref_reconstruct_q19(const double* m, double rho0, double* pop)
{
    using namespace q19;
    dfloat rhoVar = rho0 + m[0];
    dfloat ux_t30 = m[1], uy_t30 = m[2], uz_t30 = m[3];
    dfloat m_xx_t45 = m[4], m_xy_t90 = m[5], m_xz_t90 = m[6], m_yy_t45 = m[7], m_yz_t90 = m[8], m_zz_t45 = m[9];
    dfloat multiplyTerm, pics2;
#include "colrec/MR_LBM/reconstruction.inc"
}

#define D3Q27
void ref_reconstruct_q27(const double* m, double rho0, double* pop)
{
    using namespace q27;
    dfloat rhoVar = rho0 + m[0];
    dfloat ux_t30 = m[1], uy_t30 = m[2], uz_t30 = m[3];
    dfloat m_xx_t45 = m[4], m_xy_t90 = m[5], m_xz_t90 = m[6], m_yy_t45 = m[7], m_yz_t90 = m[8], m_zz_t45 = m[9];
    dfloat multiplyTerm, pics2;
#include "colrec/MR_LBM/reconstruction.inc"
}
#undef D3Q27

namespace g19 {
#include "includeFiles/velocitySets/D3G19.inc"
}

// thermal populations from C, the stored flow velocity 3u and the diffusive
// correction ud (src/mlbm.cu:165-169 computes ud = G_DIFF_FLUC_COEF (q/C - u))
void ref_reconstruct_g19(double cVar, const double* u3, const double* ud3, double* gNode)
{
    using namespace g19;
    dfloat ux_t30 = u3[0], uy_t30 = u3[1], uz_t30 = u3[2];
    dfloat udx_t30 = ud3[0], udy_t30 = ud3[1], udz_t30 = ud3[2];
    dfloat multiplyTerm, pics2;
#include "colrec/G_SCALAR/reconstruction.inc"
}

namespace rbp {
#include "cases/rayleighBenard_Periodic/constants.inc"
}

// [0] G_DIFF_FLUC_COEF, [1] T_DIFFUSIVITY, [2] T_gravity_t_beta, [3] VISC,
// [4] T_REFERENCE, [5] T_HOT, [6] T_COLD, [7..9] gravity_vector
void ref_rb_periodic_constants(double* out)
{
    out[0] = rbp::G_DIFF_FLUC_COEF;
    out[1] = rbp::T_DIFFUSIVITY;
    out[2] = rbp::T_gravity_t_beta;
    out[3] = rbp::VISC;
    out[4] = rbp::T_REFERENCE;
    out[5] = rbp::T_HOT;
    out[6] = rbp::T_COLD;
    for (int a = 0; a < 3; a++) out[7 + a] = rbp::gravity_vector[a];
}

// scaled pre-collision moments m[1..9], rho, force, omega -> post-collision m[1..9]
void ref_collide(double* m, double rho, const double* F, double omegaVar)
{
    dfloat ux_t30 = m[1], uy_t30 = m[2], uz_t30 = m[3];
    dfloat m_xx_t45 = m[4], m_xy_t90 = m[5], m_xz_t90 = m[6], m_yy_t45 = m[7], m_yz_t90 = m[8], m_zz_t45 = m[9];
    dfloat invRho = 1.0 / rho;
    dfloat L_Fx = F[0], L_Fy = F[1], L_Fz = F[2];
    dfloat t_omegaVar = 1 - omegaVar;
    dfloat tt_omegaVar = 1 - omegaVar / 2;
    dfloat omegaVar_d2 = omegaVar / 2;
    dfloat tt_omega_t3 = tt_omegaVar * 3;
#include "colrec/MR_LBM/collision.inc"
    m[1] = ux_t30; m[2] = uy_t30; m[3] = uz_t30;
    m[4] = m_xx_t45; m[5] = m_xy_t90; m[6] = m_xz_t90; m[7] = m_yy_t45; m[8] = m_yz_t90; m[9] = m_zz_t45;
}

// Output layout for the BC functions: out[0]=rho, out[1..3]=u (unscaled),
// out[4..9]=Pi_hat xx,xy,xz,yy,yz,zz (unscaled).  Returns 1 when the case
// label exists in the snippet (nodeType matched), 0 otherwise.
#define BC_PROLOGUE                                                              \
    dfloat rhoVar = -12345.0;                                                    \
    dfloat ux_t30 = 0, uy_t30 = 0, uz_t30 = 0;                                   \
    dfloat m_xx_t45 = 0, m_xy_t90 = 0, m_xz_t90 = 0, m_yy_t45 = 0, m_yz_t90 = 0, \
           m_zz_t45 = 0;                                                         \
    (void)rhoVar;
#define BC_EPILOGUE                                                              \
    out[0] = rhoVar; out[1] = ux_t30; out[2] = uy_t30; out[3] = uz_t30;          \
    out[4] = m_xx_t45; out[5] = m_xy_t90; out[6] = m_xz_t90;                     \
    out[7] = m_yy_t45; out[8] = m_yz_t90; out[9] = m_zz_t45;                     \
    return rhoVar != -12345.0;

int ref_bc_lid_q19(unsigned int nodeType, const double* pop, double omegaVar, double U_MAX, double* out)
{
    BC_PROLOGUE
#include "cases/lidDrivenCavity_3D/bc_definition.inc"
    BC_EPILOGUE
}

#define VOXEL_FILENAME "unused.csv"
int ref_bc_voxel_q19(unsigned int nodeType, const double* pop, double omegaVar, double RHO_0, double* out)
{
    BC_PROLOGUE
#include "cases/voxel/bc_definition.inc"
    BC_EPILOGUE
}
#undef VOXEL_FILENAME

int ref_bc_plates_q27(unsigned int nodeType, const double* pop, double omegaVar, double* out)
{
    BC_PROLOGUE
#include "cases/parallelPlates_D3Q27/bc_definition.inc"
    BC_EPILOGUE
}

int ref_bc_plates_q19(unsigned int nodeType, const double* pop, double omegaVar, double* out)
{
    BC_PROLOGUE
#include "cases/parallelPlates_D3Q19/bc_definition.inc"
    BC_EPILOGUE
}

// the thermal Rayleigh-Benard case's walls (its own closed forms, written in
// the wall normal l and the wall velocity)
int ref_bc_rb_q19(unsigned int nodeType, const double* pop, double omegaVar, double* out)
{
    BC_PROLOGUE
    using namespace q19;
#include "cases/rayleighBenard_Periodic/bc_definition.inc"
    BC_EPILOGUE
}

}  // extern "C"
