/*
 * mrlbm_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the moment-representation LBM (MR-LBM) step of the
 * reference solver, written from the method's equations.  The CUDA library's
 * results are compared against it (tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it); it is never linked into or called by the product.
 *
 * What it restates (reference file:line it follows):
 *   - lattice ordering / weights      src/includeFiles/velocitySets/D3Q19.inc:8-24,
 *                                     src/includeFiles/velocitySets/D3Q27.inc:9-28
 *   - stored scaled moments           src/arrayIndex.h:8-17,186-187
 *   - reconstruction                  src/colrec/MR_LBM/reconstruction.inc:1-35
 *   - pull streaming (ghost exchange) src/mlbm.cu:388-454, src/includeFiles/popLoad.inc:1-86
 *   - bulk moments + scaling          src/mlbm.cu:462-509
 *   - moment-space BC (known set I)   src/cases/lidDrivenCavity_3D/bc_definition.inc:14-717,
 *                                     src/cases/voxel/bc_definition.inc:16-7891
 *     solved here as the linear system those closed forms come from:
 *       sum_{i in I} f_i          = sum_{i in I} f^reg_i(rho, u, (1-w)Pi + w uu)
 *       sum_{i in I} f_i h_k(c_i) = sum_{i in I} h_k(c_i) f^reg_i(rho, u, Pi)
 *   - octant-mask known-set rule      src/lbmInitialization.cu:1080-1227, src/nodeTypeMap.h:10-80
 *   - outflow walls (BC_OUTFLOW)      src/cases/mountedCube/bc_definition.inc:18-33, 55-67
 *   - collision (with force terms)    src/colrec/MR_LBM/collision.inc:2-14
 *   - shear magnitude + nnf omega     src/mlbm.cu:526-563, src/nnf.h:61-98
 *     (power law with the reference's three compile defects fixed: the
 *      POWERLAW/POWER_LAW guard, the undeclared `omega`, POW_FUNCTION = pow)
 *   - initial moments                 src/lbmInitialization.cu:28-131
 *   - kinetic energy                  src/reduction.cu:128-155, src/treatData.cu:105-165
 *   - thermal scalar (D3G19)          src/mlbm.cu:157-191 (pull + sums), 515-522 (Boussinesq
 *                                     force), 603-616 (stored C, q); G_SCALAR reconstruction
 *                                     src/colrec/G_SCALAR/reconstruction.inc:1-25; weights
 *                                     src/includeFiles/velocitySets/D3G19.inc:1-19; diffusivity
 *                                     coefficient src/cases/rayleighBenard_Periodic/constants.inc:54-65;
 *                                     wall kinds as in src/cases/thermal_2D/g_bc_definition.inc,
 *                                     src/cases/rayleighBenard_Closed/g_bc_definition.inc
 *
 * Parity pins: per-node functions are checked against the reference's own
 * snippets compiled on the host (oracle/ref_kat.cpp -> oracle/_ref); full runs
 * are checked against analytic solutions and against the reference CUDA build.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXQ 27
#define ORC_SLAB 16   /* z planes per slab of the step (bounds the population scratch) */

/* Arithmetic type of the step.  FP64 by default (liboracle.so, the oracle);
 * `-DORC_REAL=float -fsingle-precision-constant` builds liboracle_f32.so, the
 * same restatement in FP32 arithmetic and FP32 storage.  The FP32 build is the
 * yardstick for how far any FP32 implementation of this algorithm drifts from
 * FP64 on a given case (driven flows accumulate round-off); the exported
 * interface takes and returns double in both builds. */
#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL real;

/* D3Q27 ordering; the first 19 entries are D3Q19 (same order as the reference). */
static const int CX[27] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 0, 0, 1,-1, 1,-1, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1};
static const int CY[27] = {0, 0, 0, 1,-1, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1, 1,-1};
static const int CZ[27] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 1,-1, 1,-1, 0, 0,-1, 1,-1, 1, 1,-1,-1, 1, 1,-1, 1,-1};

static real weight(int q, int i)
{
    int n = CX[i] * CX[i] + CY[i] * CY[i] + CZ[i] * CZ[i];
    if (q == 19) {
        static const real w19[3] = {1.0 / 3.0, 1.0 / 18.0, 1.0 / 36.0};
        return w19[n];
    }
    static const real w27[4] = {8.0 / 27.0, 2.0 / 27.0, 1.0 / 54.0, 1.0 / 216.0};
    return w27[n];
}

enum { ORC_NEWTONIAN = 0, ORC_POWERLAW = 1, ORC_BINGHAM = 2 };

typedef struct {
    int nx, ny, nz, q;
    int periodic[3];
    double tau, rho0;
    double force[3];
    double bc_velocity[4][3];
    int rheology;          /* ORC_* */
    double n_index, k_consistency, yield_stress, omega_p;
    double exterior[10];   /* stored-moment state used for sources outside wall axes */
    int bc_matrix_q;       /* lattice of the BC system matrix (19 or q) */
    /* thermal scalar C on D3G19 (THERMAL_MODEL): 4 more stored moments
     * C, 3 sum g c_x, 3 sum g c_y, 3 sum g c_z after the flow's */
    int thermal;
    double t_alpha;        /* T_DIFFUSIVITY */
    double t_reference;    /* T_REFERENCE: buoyancy reference, exterior C */
    double t_gbeta[3];     /* gravity_vector * T_gravity_t_beta */
    double t_source;       /* T_Q_INTERNAL_D_Cp, added at bulk nodes */
    double t_wall[4];      /* wall values by thermal value index */
} orc_desc;

typedef struct {
    orc_desc d;
    int nm;                /* 10, or 11 with an omega field, or 14 with the thermal scalar */
    int nmf;               /* flow moments (10 or 11) */
    real tcoef;            /* G_DIFF_FLUC_COEF */
    size_t n;
    real *m, *m2;        /* [node][nm], node = x + nx*(y + ny*z) */
    uint32_t *type;        /* reference nodeTypeMap words, same node order */
    real *pop;           /* [slab + 2][plane][q] post-collision populations of a slab of planes */
    real *gpop;          /* [slab + 2][plane][19] thermal populations (thermal only) */
    int slab;              /* output planes per slab */
} orc_domain;

/* ----------------------------------------------------------------- per node */

/* f_i = rho w_i [1 - cs2 tr(m2) + c.u3 + sum c_a^2 m_aa + sum c_a c_b m_ab]
 * with m in the stored scaled form (reconstruction.inc:1-35). */
void orc_reconstruct(int q, real rho0, const real *m, real *f)
{
    real rho = rho0 + m[0];
    real ux = m[1], uy = m[2], uz = m[3];
    real mxx = m[4], mxy = m[5], mxz = m[6], myy = m[7], myz = m[8], mzz = m[9];
    real pics2 = 1.0 - (mxx + myy + mzz) / 3.0;
    for (int i = 0; i < q; i++) {
        real cx = CX[i], cy = CY[i], cz = CZ[i];
        real t = pics2 + cx * ux + cy * uy + cz * uz + cx * cx * mxx + cy * cy * myy + cz * cz * mzz
                 + cx * cy * mxy + cx * cz * mxz + cy * cz * myz;
        f[i] = rho * weight(q, i) * t;
    }
}

/* Bulk macroscopics, unscaled: rho, u, Pi_hat = sum f cc / rho - cs2 delta (mlbm.cu:462-497). */
void orc_bulk_moments(int q, const real *f, real *out /* rho,ux,uy,uz,pxx,pxy,pxz,pyy,pyz,pzz */)
{
    real r = 0, jx = 0, jy = 0, jz = 0, pxx = 0, pxy = 0, pxz = 0, pyy = 0, pyz = 0, pzz = 0;
    for (int i = 0; i < q; i++) {
        real cx = CX[i], cy = CY[i], cz = CZ[i], v = f[i];
        r += v;
        jx += v * cx; jy += v * cy; jz += v * cz;
        pxx += v * cx * cx; pxy += v * cx * cy; pxz += v * cx * cz;
        pyy += v * cy * cy; pyz += v * cy * cz; pzz += v * cz * cz;
    }
    real ir = 1.0 / r;
    out[0] = r;
    out[1] = jx * ir; out[2] = jy * ir; out[3] = jz * ir;
    out[4] = pxx * ir - 1.0 / 3.0; out[5] = pxy * ir; out[6] = pxz * ir;
    out[7] = pyy * ir - 1.0 / 3.0; out[8] = pyz * ir; out[9] = pzz * ir - 1.0 / 3.0;
}

/* Known-set rule for the octant mask (low 8 bits of the node type):
 * octant o = ox + 2*oy + 4*oz (o_a = 1 is the + side).  The source x - c_i is
 * treated as solid when every octant consistent with the offset -c_i is marked
 * (this is how bc_id marks a solid neighbour, lbmInitialization.cu:1080-1227). */
uint32_t orc_known_mask(int q, uint32_t octants)
{
    uint32_t known = 0;
    for (int i = 0; i < q; i++) {
        int d[3] = {-CX[i], -CY[i], -CZ[i]};
        int all = 1;
        for (int o = 0; o < 8; o++) {
            int s[3] = {(o & 1) ? 1 : -1, (o & 2) ? 1 : -1, (o & 4) ? 1 : -1};
            int consistent = 1;
            for (int a = 0; a < 3; a++)
                if (d[a] != 0 && d[a] != s[a]) consistent = 0;
            if (consistent && !((octants >> o) & 1u)) { all = 0; break; }
        }
        if (!all) known |= (1u << i);
    }
    return known;
}

static void h_vec(int i, real *h)
{
    real cx = CX[i], cy = CY[i], cz = CZ[i];
    h[0] = cx * cx - 1.0 / 3.0; h[1] = cx * cy; h[2] = cx * cz;
    h[3] = cy * cy - 1.0 / 3.0; h[4] = cy * cz; h[5] = cz * cz - 1.0 / 3.0;
}

/* coefficient of Pi_k inside 4.5 * H_i : Pi  (off-diagonals counted twice) */
static void g_vec(int i, real *g)
{
    real cx = CX[i], cy = CY[i], cz = CZ[i];
    g[0] = 4.5 * (cx * cx - 1.0 / 3.0); g[1] = 9.0 * cx * cy; g[2] = 9.0 * cx * cz;
    g[3] = 4.5 * (cy * cy - 1.0 / 3.0); g[4] = 9.0 * cy * cz; g[5] = 4.5 * (cz * cz - 1.0 / 3.0);
}

static int solve7(real A[7][7], real *b, real *x)
{
    int p[7];
    for (int i = 0; i < 7; i++) p[i] = i;
    for (int c = 0; c < 7; c++) {
        int best = c;
        for (int r = c + 1; r < 7; r++)
            if (fabs(A[p[r]][c]) > fabs(A[p[best]][c])) best = r;
        int t = p[c]; p[c] = p[best]; p[best] = t;
        real piv = A[p[c]][c];
        if (piv == 0) return -1;
        for (int r = c + 1; r < 7; r++) {
            real f = A[p[r]][c] / piv;
            if (f == 0.0) continue;
            for (int k = c; k < 7; k++) A[p[r]][k] -= f * A[p[c]][k];
            b[p[r]] -= f * b[p[c]];
        }
    }
    for (int c = 6; c >= 0; c--) {
        real s = b[p[c]];
        for (int k = c + 1; k < 7; k++) s -= A[p[c]][k] * x[k];
        x[c] = s / A[p[c]][c];
    }
    return 0;
}

/* Moment-based wall BC.  Inputs: post-stream pops f (only `known` entries are
 * read), prescribed velocity u (unscaled), omega.  Output: rho and the
 * unscaled Pi_hat (xx,xy,xz,yy,yz,zz) -> out[0], out[4..9]; out[1..3] = u.
 * The right-hand side sums the known pops of the q-velocity lattice; the
 * system matrix is assembled over the first mq velocities (mq = 19 on a
 * D3Q27 lattice reproduces the reference's D3Q27 wall formulas, which are the
 * D3Q19 closed forms fed with D3Q27 known-set moments,
 * src/cases/parallelPlates_D3Q27/bc_definition.inc:18-44). */
int orc_bc_solve(int q, int mq, uint32_t known, const real *u, real omega, const real *f, real *out)
{
    real A[7][7], b[7], x[7];
    memset(A, 0, sizeof(A));
    memset(b, 0, sizeof(b));
    real uu[6] = {u[0] * u[0], u[0] * u[1], u[0] * u[2], u[1] * u[1], u[1] * u[2], u[2] * u[2]};
    for (int i = 0; i < q; i++) {
        if (!((known >> i) & 1u)) continue;
        real h[6], g[6];
        h_vec(i, h);
        b[0] += f[i];
        for (int r = 0; r < 6; r++) b[1 + r] += f[i] * h[r];
    }
    for (int i = 0; i < mq; i++) {
        if (!((known >> i) & 1u)) continue;
        real w = weight(mq, i), h[6], g[6];
        h_vec(i, h);
        g_vec(i, g);
        real cu = 3.0 * (CX[i] * u[0] + CY[i] * u[1] + CZ[i] * u[2]);
        real guu = 0.0;
        for (int k = 0; k < 6; k++) guu += g[k] * uu[k];
        /* row 0: sum_I f^reg(rho, u, (1-w)Pi + w uu) */
        A[0][0] += w * (1.0 + cu + omega * guu);
        for (int k = 0; k < 6; k++) A[0][1 + k] += (1.0 - omega) * w * g[k];
        /* rows 1..6: sum_I h_k f^reg(rho, u, Pi) */
        for (int r = 0; r < 6; r++) {
            A[1 + r][0] += w * h[r] * (1.0 + cu);
            for (int k = 0; k < 6; k++) A[1 + r][1 + k] += w * h[r] * g[k];
        }
    }
    if (solve7(A, b, x) != 0) return -1;
    out[0] = x[0];
    out[1] = u[0]; out[2] = u[1]; out[3] = u[2];
    for (int k = 0; k < 6; k++) out[4 + k] = x[1 + k] / x[0];
    return 0;
}

/* Power-law omega by Newton iteration (nnf.h:61-89), defects fixed. */
real orc_nnf_powerlaw(real omega_old, real smag, real n_index, real k_cons, real rho0)
{
    real omega = omega_old;
    real a = k_cons * pow(smag / (rho0 / 3.0), n_index);
    real b = 0.5 * smag, c = -smag;
    if (smag < 1e-6) return 0.0;
    for (int it = 0; it < 7; it++) {
        real fx = a * pow(omega, n_index) + b * omega + c;
        real dfx = a * n_index * pow(omega, n_index - 1.0) + b;
        if (fabs(fx / dfx) < 1e-6) break;
        omega = omega - fx / dfx;
    }
    return omega;
}

real orc_nnf_bingham(real smag, real omega_p, real yield_stress)
{
    real v = 1.0 - yield_stress / smag;
    return omega_p * (v > 0.0 ? v : 0.0);
}

/* Scale, (shear, nnf), collide.  mac = rho,u,Pi unscaled in/out; m = stored
 * scaled moments out (nm entries).  Follows mlbm.cu:500-591 + collision.inc. */
static void collide_store(const orc_desc *d, int nm, const real *mac, real omega_in, real *m, const real *F)
{
    real rho = mac[0];
    real ux = 3.0 * mac[1], uy = 3.0 * mac[2], uz = 3.0 * mac[3];
    real mxx = 4.5 * mac[4], mxy = 9.0 * mac[5], mxz = 9.0 * mac[6];
    real myy = 4.5 * mac[7], myz = 9.0 * mac[8], mzz = 4.5 * mac[9];
    real Fx = F[0], Fy = F[1], Fz = F[2];
    real omega = omega_in;
    if (d->rheology != ORC_NEWTONIAN) {
        real sxx = rho * (mxx / 4.5 - ux * ux / 9.0), syy = rho * (myy / 4.5 - uy * uy / 9.0);
        real szz = rho * (mzz / 4.5 - uz * uz / 9.0), sxy = rho * (mxy / 9.0 - ux * uy / 9.0);
        real sxz = rho * (mxz / 9.0 - ux * uz / 9.0), syz = rho * (myz / 9.0 - uy * uz / 9.0);
        real fxx = ux * Fx / 3.0, fyy = uy * Fy / 3.0, fzz = uz * Fz / 3.0;
        real fxy = (ux * Fy + uy * Fx) / 6.0, fxz = (ux * Fz + uz * Fx) / 6.0, fyz = (uy * Fz + uz * Fy) / 6.0;
        real smag = sqrt(0.5 * ((sxx + fxx) * (sxx + fxx) + (syy + fyy) * (syy + fyy) + (szz + fzz) * (szz + fzz)
                                  + 2.0 * ((sxy + fxy) * (sxy + fxy) + (sxz + fxz) * (sxz + fxz) + (syz + fyz) * (syz + fyz))));
        if (d->rheology == ORC_POWERLAW)
            omega = orc_nnf_powerlaw(omega_in, smag, d->n_index, d->k_consistency, d->rho0);
        else
            omega = orc_nnf_bingham(smag, d->omega_p, d->yield_stress);
    }
    real ir = 1.0 / rho;
    real t_om = 1.0 - omega, tt_om = 1.0 - 0.5 * omega, om_d2 = 0.5 * omega, tt_om_t3 = 3.0 * tt_om;
    ux += 3.0 * ir * Fx; uy += 3.0 * ir * Fy; uz += 3.0 * ir * Fz;
    real ir15 = 1.5 * ir;
    mxx = t_om * mxx + om_d2 * ux * ux + ir15 * tt_om * (2.0 * Fx * ux);
    myy = t_om * myy + om_d2 * uy * uy + ir15 * tt_om * (2.0 * Fy * uy);
    mzz = t_om * mzz + om_d2 * uz * uz + ir15 * tt_om * (2.0 * Fz * uz);
    mxy = t_om * mxy + omega * ux * uy + tt_om_t3 * ir * (Fx * uy + Fy * ux);
    mxz = t_om * mxz + omega * ux * uz + tt_om_t3 * ir * (Fx * uz + Fz * ux);
    myz = t_om * myz + omega * uy * uz + tt_om_t3 * ir * (Fy * uz + Fz * uy);
    m[0] = rho - d->rho0;
    m[1] = ux; m[2] = uy; m[3] = uz;
    m[4] = mxx; m[5] = mxy; m[6] = mxz; m[7] = myy; m[8] = myz; m[9] = mzz;
    if (nm > 10) m[10] = omega;
}

/* exposed for KATs: unscaled macroscopics + omega -> stored post-collision moments */
void orc_collide(const orc_desc *d, const real *mac, real omega, real *m_out, int nm)
{
    real F[3] = {d->force[0], d->force[1], d->force[2]};
    collide_store(d, nm, mac, omega, m_out, F);
}

/* --------------------------------------------------------- thermal scalar */

/* G_DIFF_FLUC_COEF from the thermal diffusivity, with the reference's fixed
 * T_DIFF_REF = 1/6 and G_TAU = 3 T_DIFF_REF + 1/2
 * (src/cases/rayleighBenard_Periodic/constants.inc:58-65). */
double orc_thermal_coef(double alpha)
{
    double diff_ref = 1.0 / 6.0, g_tau = diff_ref * 3.0 + 0.5, g_omega = 1.0 / g_tau;
    double aaa = 3.0 * (alpha - diff_ref) * g_omega;
    return aaa / (1.0 + aaa);
}

/* g_i = C w_i (1 + c_i . (u3 + ud3)), ud3 = coef (q3 / C - u3), on the first
 * 19 directions with the D3Q19 weights (G_SCALAR/reconstruction.inc:1-25,
 * mlbm.cu:159-167). u3, q3: stored 3u and 3 sum g c. */
void orc_reconstruct_g(real coef, real c, const real *u3, const real *q3, real *g)
{
    real ic = 1.0 / c, v[3];
    for (int a = 0; a < 3; a++) v[a] = u3[a] + coef * (q3[a] * ic - u3[a]);
    for (int i = 0; i < 19; i++)
        g[i] = c * weight(19, i) * (1.0 + CX[i] * v[0] + CY[i] * v[1] + CZ[i] * v[2]);
}

/* C = sum g + source, q3 = 3 sum g c (mlbm.cu:180-188). */
void orc_sums_g(const real *g, real source, real *cq)
{
    real c = 0, qx = 0, qy = 0, qz = 0;
    for (int i = 0; i < 19; i++) {
        c += g[i];
        qx += g[i] * CX[i]; qy += g[i] * CY[i]; qz += g[i] * CZ[i];
    }
    cq[0] = c + source;
    cq[1] = 3.0 * qx; cq[2] = 3.0 * qy; cq[3] = 3.0 * qz;
}

/* The wall of a face class: the axis whose whole + or - half of the octant
 * mask is solid, when exactly one such (axis, side) exists.  Returns the axis
 * (0..2) and *side (+1: solid on the + side), or -1. */
int orc_face_normal(uint32_t octants, int *side)
{
    int found = -1, n = 0;
    for (int a = 0; a < 3; a++)
        for (int sd = 0; sd < 2; sd++) {
            int all = 1;
            for (int o = 0; o < 8; o++)
                if ((((o >> a) & 1) == sd) && !((octants >> o) & 1u)) all = 0;
            if (all) { found = a; *side = sd ? 1 : -1; n++; }
        }
    return n == 1 ? found : -1;
}

/* ------------------------------------------------------------------ domain */

void *orc_create(const orc_desc *d)
{
    orc_domain *o = (orc_domain *)calloc(1, sizeof(orc_domain));
    if (!o) return NULL;
    o->d = *d;
    o->nmf = (d->rheology != ORC_NEWTONIAN) ? 11 : 10;
    o->nm = o->nmf + (d->thermal ? 4 : 0);
    o->tcoef = (real)orc_thermal_coef(d->t_alpha);
    o->n = (size_t)d->nx * d->ny * d->nz;
    o->m = (real *)calloc(o->n * o->nm, sizeof(real));
    o->m2 = (real *)calloc(o->n * o->nm, sizeof(real));
    o->type = (uint32_t *)calloc(o->n, sizeof(uint32_t));
    o->slab = d->nz < ORC_SLAB ? d->nz : ORC_SLAB;
    o->pop = (real *)malloc((size_t)(o->slab + 2) * d->nx * d->ny * d->q * sizeof(real));
    o->gpop = d->thermal ? (real *)malloc((size_t)(o->slab + 2) * d->nx * d->ny * 19 * sizeof(real)) : NULL;
    if (!o->m || !o->m2 || !o->type || !o->pop || (d->thermal && !o->gpop)) {
        free(o->m); free(o->m2); free(o->type); free(o->pop); free(o->gpop); free(o);
        return NULL;
    }
    return o;
}

void orc_destroy(void *h)
{
    orc_domain *o = (orc_domain *)h;
    if (!o) return;
    free(o->m); free(o->m2); free(o->type); free(o->pop); free(o->gpop); free(o);
}

int orc_num_moments(void *h) { return ((orc_domain *)h)->nm; }

void orc_set_node_types(void *h, const uint32_t *t)
{
    orc_domain *o = (orc_domain *)h;
    memcpy(o->type, t, o->n * sizeof(uint32_t));
}

void orc_set_moments(void *h, const double *m)
{
    orc_domain *o = (orc_domain *)h;
    for (size_t k = 0; k < o->n * o->nm; k++) o->m[k] = o->m2[k] = (real)m[k];
}

void orc_get_moments(void *h, double *m)
{
    orc_domain *o = (orc_domain *)h;
    for (size_t k = 0; k < o->n * o->nm; k++) m[k] = o->m[k];
}

/* Initial moments from physical rho,u (x-fastest) exactly as
 * gpuInitialization_mom (lbmInitialization.cu:28-131): the second moments are
 * built from an equilibrium with weight*RHO_0 and the D3Q19 index sums even for
 * D3Q27 (when d3q19_sums != 0; 0 uses the full lattice sums). */
void orc_init_from_macro(void *h, const double *rho, const double *ux, const double *uy, const double *uz,
                         int d3q19_sums)
{
    orc_domain *o = (orc_domain *)h;
    int q = o->d.q, qs = d3q19_sums ? 19 : q;
    real omega = 1.0 / o->d.tau;
    for (size_t k = 0; k < o->n; k++) {
        real f[ORC_MAXQ];
        real u[3] = {ux[k], uy[k], uz[k]};
        real uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        for (int i = 0; i < q; i++) {
            real uc3 = 3.0 * (u[0] * CX[i] + u[1] * CY[i] + u[2] * CZ[i]);
            f[i] = weight(q, i) * o->d.rho0 * ((1.0 - 1.5 * uu) + uc3 * (1.0 + 0.5 * uc3));
        }
        real ir = 1.0 / rho[k], p[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < qs; i++) {
            real cx = CX[i], cy = CY[i], cz = CZ[i];
            p[0] += f[i] * cx * cx; p[1] += f[i] * cx * cy; p[2] += f[i] * cx * cz;
            p[3] += f[i] * cy * cy; p[4] += f[i] * cy * cz; p[5] += f[i] * cz * cz;
        }
        real *m = o->m + k * o->nm;
        m[0] = rho[k] - o->d.rho0;
        m[1] = 3.0 * u[0]; m[2] = 3.0 * u[1]; m[3] = 3.0 * u[2];
        m[4] = 4.5 * (p[0] * ir - 1.0 / 3.0);
        m[5] = 9.0 * (p[1] * ir);
        m[6] = 9.0 * (p[2] * ir);
        m[7] = 4.5 * (p[3] * ir - 1.0 / 3.0);
        m[8] = 9.0 * (p[4] * ir);
        m[9] = 4.5 * (p[5] * ir - 1.0 / 3.0);
        if (o->nmf > 10) m[10] = omega;
        if (o->d.thermal) {
            m[o->nmf] = o->d.t_reference;
            m[o->nmf + 1] = m[o->nmf + 2] = m[o->nmf + 3] = 0.0;
        }
    }
    memcpy(o->m2, o->m, o->n * o->nm * sizeof(real));
}

static inline int resolve(int v, int n, int periodic, int *outside)
{
    if (v >= 0 && v < n) return v;
    if (periodic) return (v + n) % n;
    *outside = 1;
    return 0;
}

void orc_step(void *h, int nsteps)
{
    orc_domain *o = (orc_domain *)h;
    const orc_desc *d = &o->d;
    const int q = d->q, nm = o->nm, nmf = o->nmf, nx = d->nx, ny = d->ny, nz = d->nz;
    const int th = d->thermal;
    const size_t pl = (size_t)nx * ny;
    const real omega0 = 1.0 / d->tau;
    real fext[ORC_MAXQ], gext[19];
    real ext[10];
    for (int k = 0; k < 10; k++) ext[k] = (real)d->exterior[k];
    orc_reconstruct(q, d->rho0, ext, fext);
    if (th) {
        const real q0[3] = {0, 0, 0};
        orc_reconstruct_g(o->tcoef, (real)d->t_reference, ext + 1, q0, gext);
    }
    for (int s = 0; s < nsteps; s++) {
        /* output planes [z0, z1) pull from planes z0-1 .. z1: their
         * post-collision populations (from the stored moments) are built
         * for one slab at a time, so the scratch is slab + 2 planes */
        for (int z0 = 0; z0 < nz; z0 += o->slab) {
            const int z1 = (z0 + o->slab < nz) ? z0 + o->slab : nz;
            const int nsl = z1 - z0 + 2;
            int src[ORC_SLAB + 2];
            for (int k = 0; k < nsl; k++) {
                int out = 0;
                const int sz = resolve(z0 - 1 + k, nz, d->periodic[2], &out);
                src[k] = out ? -1 : sz;
            }
#pragma omp parallel for collapse(2) schedule(static)
            for (int k = 0; k < nsl; k++)
                for (long c = 0; c < (long)pl; c++)
                    if (src[k] >= 0) {
                        const real *ms = o->m + ((size_t)src[k] * pl + c) * nm;
                        orc_reconstruct(q, d->rho0, ms, o->pop + ((size_t)k * pl + c) * q);
                        if (th)
                            orc_reconstruct_g(o->tcoef, ms[nmf], ms + 1, ms + nmf + 1, o->gpop + ((size_t)k * pl + c) * 19);
                    }
#pragma omp parallel for collapse(2) schedule(static)
            for (int z = z0; z < z1; z++)
                for (int y = 0; y < ny; y++)
                    for (int x = 0; x < nx; x++) {
                        size_t k = (size_t)x + (size_t)nx * (y + (size_t)ny * z);
                        uint32_t t = o->type[k];
                        real *mo = o->m2 + k * nm;
                        const real *mi = o->m + k * nm;
                        if ((t & 0xFFu) == 0xFFu) { memcpy(mo, mi, nm * sizeof(real)); continue; }
                        real f[ORC_MAXQ], g[19];
                        for (int i = 0; i < q; i++) {
                            int out = 0;
                            int sx = resolve(x - CX[i], nx, d->periodic[0], &out);
                            int sy = resolve(y - CY[i], ny, d->periodic[1], &out);
                            const int ks = z - CZ[i] - (z0 - 1);
                            const int ext_src = out || src[ks] < 0;
                            const size_t ps = (size_t)ks * pl + (size_t)sx + (size_t)nx * sy;
                            f[i] = ext_src ? fext[i] : o->pop[ps * q + i];
                            if (th && i < 19) g[i] = ext_src ? gext[i] : o->gpop[ps * 19 + i];
                        }
                        real omega = (nmf > 10) ? mi[10] : omega0;
                        real F[3] = {d->force[0], d->force[1], d->force[2]};
                        real cq[4];
                        if (th) {
                            const int tkind = (t >> 13) & 3u;
                            if ((t & 0xFFu) == 0) {
                                orc_sums_g(g, (real)d->t_source, cq);
                                /* Boussinesq force at bulk nodes (mlbm.cu:515-522) */
                                for (int a = 0; a < 3; a++) F[a] += (real)d->t_gbeta[a] * d->rho0 * (cq[0] - d->t_reference);
                            } else if (tkind == 0) {
                                /* no thermal rule for this node type: C, q keep the stored values */
                                for (int c = 0; c < 4; c++) cq[c] = mi[nmf + c];
                            } else {
                                const real tw = (real)d->t_wall[(t >> 15) & 3u];
                                int side = 0;
                                const int ax = orc_face_normal(t & 0xFFu, &side);
                                if (tkind == 1 || ax < 0) {
                                    cq[0] = tw; cq[1] = cq[2] = cq[3] = 0.0;
                                } else if (tkind == 2) {
                                    /* normal flux of the inward neighbour, previous step */
                                    int nb[3] = {x, y, z};
                                    const int dim[3] = {nx, ny, nz};
                                    nb[ax] -= side;
                                    cq[0] = tw; cq[1] = cq[2] = cq[3] = 0.0;
                                    if (nb[ax] >= 0 && nb[ax] < dim[ax]) {
                                        const size_t kn = (size_t)nb[0] + (size_t)nx * (nb[1] + (size_t)ny * nb[2]);
                                        cq[1 + ax] = o->m[kn * nm + nmf + 1 + ax];
                                    }
                                } else {
                                    /* adiabatic: populations arriving from the solid side
                                     * mirrored across the wall plane */
                                    real gm[19];
                                    for (int i = 0; i < 19; i++) {
                                        const int c[3] = {CX[i], CY[i], CZ[i]};
                                        if (c[ax] == -side) {
                                            int mc[3] = {c[0], c[1], c[2]};
                                            mc[ax] = -mc[ax];
                                            int j = 0;
                                            while (CX[j] != mc[0] || CY[j] != mc[1] || CZ[j] != mc[2]) j++;
                                            gm[i] = g[j];
                                        } else {
                                            gm[i] = g[i];
                                        }
                                    }
                                    orc_sums_g(gm, 0.0, cq);
                                }
                            }
                        }
                        real mac[10];
                        if ((t & 0xFFu) == 0) {
                            orc_bulk_moments(q, f, mac);
                        } else if (((t >> 8) & 7u) == 2) {
                            /* outflow (BC_OUTFLOW, mountedCube/bc_definition.inc:18-33): the
                             * inward neighbour's stored moments of the previous step, unscaled */
                            int side = 0;
                            const int ax = orc_face_normal(t & 0xFFu, &side);
                            int nb[3] = {x, y, z};
                            if (ax >= 0) nb[ax] -= side;
                            const real *mn = o->m + ((size_t)nb[0] + (size_t)nx * (nb[1] + (size_t)ny * nb[2])) * nm;
                            mac[0] = d->rho0 + mn[0];
                            mac[1] = mn[1] / 3.0; mac[2] = mn[2] / 3.0; mac[3] = mn[3] / 3.0;
                            mac[4] = mn[4] / 4.5; mac[5] = mn[5] / 9.0; mac[6] = mn[6] / 9.0;
                            mac[7] = mn[7] / 4.5; mac[8] = mn[8] / 9.0; mac[9] = mn[9] / 4.5;
                        } else {
                            int vidx = (t >> 11) & 3u;
                            int kind = (t >> 8) & 7u;
                            real u[3] = {0, 0, 0};
                            if (kind == 1) { u[0] = d->bc_velocity[vidx][0]; u[1] = d->bc_velocity[vidx][1]; u[2] = d->bc_velocity[vidx][2]; }
                            orc_bc_solve(q, d->bc_matrix_q ? d->bc_matrix_q : q, orc_known_mask(q, t & 0xFFu), u, omega, f, mac);
                        }
                        collide_store(d, nmf, mac, omega, mo, F);
                        if (th)
                            for (int c = 0; c < 4; c++) mo[nmf + c] = cq[c];
                    }
        }
        real *tmp = o->m; o->m = o->m2; o->m2 = tmp;
    }
}

/* FP64 sums over non-solid nodes: [0] sum rho, [1..3] sum rho u, [4] sum KE
 * where KE per node = rho |u|^2 / 2 (reduction.cu:145 uses (rho0+m0)|3u|^2/18),
 * [5] fluid node count. */
void orc_sums(void *h, double *out)
{
    orc_domain *o = (orc_domain *)h;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (size_t k = 0; k < o->n; k++) {
        if ((o->type[k] & 0xFFu) == 0xFFu) continue;
        const real *m = o->m + k * o->nm;
        double rho = o->d.rho0 + (double)m[0];
        double ux = m[1] / 3.0, uy = m[2] / 3.0, uz = m[3] / 3.0;
        s[0] += rho; s[1] += rho * ux; s[2] += rho * uy; s[3] += rho * uz;
        s[4] += 0.5 * rho * (ux * ux + uy * uy + uz * uz);
        s[5] += 1.0;
    }
    memcpy(out, s, sizeof(s));
}

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
