// io.cu -- the reference's on-disk formats: checkpoints, macroscopic .bin
// files and the _info.txt summary.
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mrlbm.h"
#include "domain.h"

using namespace mrlbm;

static mrlbm_status mkdirs(const std::string& path)
{
    std::string cur;
    size_t pos = 0;
    while (pos != std::string::npos) {
        pos = path.find('/', pos + 1);
        cur = path.substr(0, pos);
        if (cur.empty()) continue;
        if (mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST)
            return fail(MRLBM_EIO, "cannot create folder '%s': %s", cur.c_str(), strerror(errno));
    }
    return MRLBM_OK;
}

static mrlbm_status write_file(const std::string& name, const void* p, size_t bytes)
{
    FILE* f = fopen(name.c_str(), "wb");
    if (!f) return fail(MRLBM_EIO, "cannot open '%s' for writing", name.c_str());
    const size_t w = bytes ? fwrite(p, bytes, 1, f) : 1;
    fclose(f);
    if (w != 1) return fail(MRLBM_EIO, "short write to '%s'", name.c_str());
    return MRLBM_OK;
}

static mrlbm_status read_file(const std::string& name, void* p, size_t bytes)
{
    FILE* f = fopen(name.c_str(), "rb");
    if (!f) return fail(MRLBM_EIO, "cannot open '%s'", name.c_str());
    fseek(f, 0, SEEK_END);
    const long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz < 0 || (size_t)sz != bytes) {
        fclose(f);
        return fail(MRLBM_EIO, "'%s' has %ld bytes, expected %zu", name.c_str(), sz, bytes);
    }
    const size_t r = fread(p, bytes, 1, f);
    fclose(f);
    if (r != 1) return fail(MRLBM_EIO, "short read from '%s'", name.c_str());
    return MRLBM_OK;
}

// Host reconstruction (same arithmetic as the device's) for the ghost files.
static void host_reconstruct(int q, float rho0, const float* m, float* f)
{
    const float rho = rho0 + m[0];
    const float pics2 = 1.0f - (m[4] + m[7] + m[9]) * (1.0f / 3.0f);
    for (int i = 0; i < q; i++) {
        const float cx = (float)lat_cx(i), cy = (float)lat_cy(i), cz = (float)lat_cz(i);
        const float t = pics2 + cx * m[1] + cy * m[2] + cz * m[3] + cx * cx * m[4] + cy * cy * m[7] + cz * cz * m[9] +
                        cx * cy * m[5] + cx * cz * m[6] + cy * cz * m[8];
        f[i] = rho * (float)lat_w(q, i) * t;
    }
}

// Host reconstruction of the thermal populations (same formula as the
// device's): g_i = C w_i (1 + c_i . (u3 + coef (q3 / C - u3))), D3G19.
static void host_reconstruct_g(float coef, const float* m, float* g)
{
    const float C = m[10], iC = 1.0f / C;
    float v[3];
    for (int a = 0; a < 3; a++) v[a] = m[1 + a] + coef * (m[11 + a] * iC - m[1 + a]);
    for (int i = 0; i < 19; i++)
        g[i] = C * (float)lat_w(19, i) * (1.0f + lat_cx(i) * v[0] + lat_cy(i) * v[1] + lat_cz(i) * v[2]);
}

// Ghost-face files of the reference (fGhost.{X,Y,Z}_{0,1}, layout idxPopX/Y/Z,
// src/globalFunctions.h:45-124): the populations leaving each 8^3 block through
// each face, face pops in increasing velocity index.  On a wall axis the faces
// on the domain boundary hold the initial rest state, as in the reference
// (they are never rewritten there, src/includeFiles/interface.h:6-19).  With
// the thermal scalar the D3G19 populations go to g_fGhost.* the same way
// (src/checkpoint.cu:188-194, GF = 5 per face).
static mrlbm_status write_ghosts(mrlbm_domain* dom, const std::vector<float>& m, const std::string& base)
{
    const mrlbm_desc& d = dom->d;
    const int nbx = d.nx / 8, nby = d.ny / 8, nbz = d.nz / 8;
    const size_t n = (size_t)d.nx * d.ny * d.nz;
    const int nm = dom->nm;
    static const char* names[6] = {"X_0", "X_1", "Y_0", "Y_1", "Z_0", "Z_1"};
    float coef = 0.f;
    if (d.thermal) {
        const double diff_ref = 1.0 / 6.0, aaa = 3.0 * (d.t_diffusivity - diff_ref) / (diff_ref * 3.0 + 0.5);
        coef = (float)(aaa / (1.0 + aaa));
    }
    for (int dist = 0; dist < (d.thermal ? 2 : 1); dist++) {
        const int q = dist ? 19 : dom->q, qf = q == 19 ? 5 : 9;
        float mext[NM_MAX];
        memcpy(mext, dom->ext, sizeof(mext));
        float fext[27];
        if (dist) host_reconstruct_g(coef, mext, fext); else host_reconstruct(q, (float)d.rho0, mext, fext);
        for (int face = 0; face < 6; face++) {
            const int axis = face / 2, side = face % 2;  // side 0: the -face (pops with c_axis = -1)
            const int sgn = side ? 1 : -1;
            std::vector<int> pops;
            for (int i = 0; i < q; i++) {
                const int c = axis == 0 ? lat_cx(i) : axis == 1 ? lat_cy(i) : lat_cz(i);
                if (c == sgn) pops.push_back(i);
            }
            std::vector<float> buf((size_t)64 * qf * nbx * nby * nbz);
            for (int bz = 0; bz < nbz; bz++)
                for (int by = 0; by < nby; by++)
                    for (int bx = 0; bx < nbx; bx++)
                        for (int b = 0; b < 8; b++)
                            for (int a = 0; a < 8; a++) {
                                int tx, ty, tz;
                                const int t = side ? 7 : 0;
                                if (axis == 0) { tx = t; ty = a; tz = b; }
                                else if (axis == 1) { tx = a; ty = t; tz = b; }
                                else { tx = a; ty = b; tz = t; }
                                const int x = bx * 8 + tx, y = by * 8 + ty, z = bz * 8 + tz;
                                const int coord = axis == 0 ? x : axis == 1 ? y : z;
                                const int ncoord = axis == 0 ? d.nx : axis == 1 ? d.ny : d.nz;
                                const bool wall_face = !d.periodic[axis] && coord == (side ? ncoord - 1 : 0);
                                float f[27];
                                if (wall_face) {
                                    memcpy(f, fext, sizeof(f));
                                } else {
                                    float mm[NM_MAX];
                                    const size_t node = (size_t)x + (size_t)d.nx * (y + (size_t)d.ny * z);
                                    for (int k = 0; k < nm; k++) mm[k] = m[k * n + node];
                                    if (dist) host_reconstruct_g(coef, mm, f); else host_reconstruct(q, (float)d.rho0, mm, f);
                                }
                                const size_t blk = bx + (size_t)nbx * (by + (size_t)nby * bz);
                                for (int p = 0; p < qf; p++)
                                    buf[a + 8 * (b + 8 * (p + (size_t)qf * blk))] = f[pops[p]];
                            }
            mrlbm_status st = write_file(base + (dist ? "g_fGhost." : "fGhost.") + names[face] + ".bin", buf.data(),
                                         buf.size() * sizeof(float));
            if (st) return st;
        }
    }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_save_checkpoint(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step)
{
    if (!dom || !path_files || !id_sim) return fail(MRLBM_EINVAL, "null argument");
    const mrlbm_desc& d = dom->d;
    if (d.nx % 8 || d.ny % 8 || d.nz % 8) return fail(MRLBM_EINVAL, "checkpoint format needs multiples of 8");
    const std::string dir = std::string(path_files) + "/" + id_sim + "/checkpoint";
    mrlbm_status st = mkdirs(dir);
    if (st) return st;
    const std::string base = dir + "/_";
    const size_t n = (size_t)d.nx * d.ny * d.nz;
    std::vector<float> ref(n * dom->nm), plain(n * dom->nm);
    if ((st = mrlbm_get_moments_ref_layout(dom, ref.data()))) return st;
    if ((st = mrlbm_get_moments(dom, plain.data()))) return st;
    int32_t s32 = step;
    if ((st = write_file(base + "curr_step.bin", &s32, sizeof(s32)))) return st;
    if ((st = write_file(base + "fMom.bin", ref.data(), ref.size() * sizeof(float)))) return st;
    return write_ghosts(dom, plain, base);
}

extern "C" mrlbm_status mrlbm_load_checkpoint(mrlbm_domain* dom, const char* path_files, const char* id_sim, int* step)
{
    if (!dom || !path_files || !id_sim || !step) return fail(MRLBM_EINVAL, "null argument");
    const mrlbm_desc& d = dom->d;
    const std::string base = std::string(path_files) + "/" + id_sim + "/checkpoint/_";
    int32_t s32 = 0;
    mrlbm_status st = read_file(base + "curr_step.bin", &s32, sizeof(s32));
    if (st) return st;
    std::vector<float> ref((size_t)d.nx * d.ny * d.nz * dom->nm);
    if ((st = read_file(base + "fMom.bin", ref.data(), ref.size() * sizeof(float)))) return st;
    if ((st = mrlbm_set_moments_ref_layout(dom, ref.data()))) return st;
    // the ghost files hold populations this solver reconstructs from the
    // moments; their presence is checked for format compatibility only
    static const char* names[6] = {"X_0", "X_1", "Y_0", "Y_1", "Z_0", "Z_1"};
    for (int dist = 0; dist < (d.thermal ? 2 : 1); dist++)
        for (int f = 0; f < 6; f++) {
            const std::string g = base + (dist ? "g_fGhost." : "fGhost.") + names[f] + ".bin";
            struct stat sb;
            if (stat(g.c_str(), &sb) != 0) return fail(MRLBM_EIO, "missing ghost file '%s'", g.c_str());
        }
    *step = s32 + 1;
    dom->step = s32 + 1;
    return MRLBM_OK;
}

// PATH/ID/ID_<var><6-digit step>.bin; step 0 gets seven zeros, like
// getVarFilename (src/saveData.cu:439-467).
static std::string var_filename(const char* path, const char* id, const char* var, unsigned step, const char* ext)
{
    unsigned nz = 0, pot = 10;
    const unsigned aux = 1000000;
    if (step != 0)
        for (nz = 0; step * pot < aux; pot *= 10) nz++;
    else
        nz = 6;
    std::string s = std::string(path) + "/" + id + "/" + id + "_" + var;
    for (unsigned i = 0; i < nz; i++) s += "0";
    return s + std::to_string(step) + ext;
}

// the thermal scalar C (moment 10 of a thermal domain), x-fastest
static mrlbm_status thermal_scalar(mrlbm_domain* dom, std::vector<float>& c)
{
    const size_t n = (size_t)dom->d.nx * dom->d.ny * dom->d.nz;
    std::vector<float> all(n * dom->nm);
    mrlbm_status st = mrlbm_get_moments(dom, all.data());
    if (st) return st;
    c.assign(all.begin() + 10 * n, all.begin() + 11 * n);
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_save_macr_bin(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step)
{
    if (!dom || !path_files || !id_sim) return fail(MRLBM_EINVAL, "null argument");
    const mrlbm_desc& d = dom->d;
    const size_t n = (size_t)d.nx * d.ny * d.nz;
    mrlbm_status st = mkdirs(std::string(path_files) + "/" + id_sim);
    if (st) return st;
    const bool has_om = d.rheology != MRLBM_NEWTONIAN;
    std::vector<float> rho(n), ux(n), uy(n), uz(n), om, cv;
    if (has_om) om.resize(n);
    if ((st = mrlbm_get_macr(dom, rho.data(), ux.data(), uy.data(), uz.data(), has_om ? om.data() : nullptr)))
        return st;
    if (d.thermal && (st = thermal_scalar(dom, cv))) return st;
    const unsigned s = (unsigned)step;
    if ((st = write_file(var_filename(path_files, id_sim, "rho", s, ".bin"), rho.data(), n * 4))) return st;
    if ((st = write_file(var_filename(path_files, id_sim, "ux", s, ".bin"), ux.data(), n * 4))) return st;
    if ((st = write_file(var_filename(path_files, id_sim, "uy", s, ".bin"), uy.data(), n * 4))) return st;
    if ((st = write_file(var_filename(path_files, id_sim, "uz", s, ".bin"), uz.data(), n * 4))) return st;
    if (has_om)
        if ((st = write_file(var_filename(path_files, id_sim, "omega", s, ".bin"), om.data(), n * 4))) return st;
    // SECOND_DIST: <id>_C<step>.bin (src/saveData.cu:192-193, 229-230)
    if (d.thermal)
        if ((st = write_file(var_filename(path_files, id_sim, "C", s, ".bin"), cv.data(), n * 4))) return st;
    return MRLBM_OK;
}

// Legacy VTK structured-points file, binary (big-endian floats), as
// saveVarVTK writes it (src/saveData.cu:303-400): SCALARS rho (rho0 + m0),
// VECTORS velocity (physical u, the stored 3u divided by 3), SCALARS omega
// when the domain carries an omega field and SCALARS C with the thermal scalar.  File <path>/<id>/<id>_vtk<step>.vtk
// (src/saveData.cu:153).  The reference's optional node-type and BC-force
// sections (NODE_TYPE_SAVE, SAVE_BC_FORCES) are not written.
static void put_be(std::string& out, const float* v, size_t n)
{
    const size_t at = out.size();
    out.resize(at + 4 * n);
    for (size_t i = 0; i < n; i++) {
        uint32_t w;
        memcpy(&w, &v[i], 4);
        w = __builtin_bswap32(w);
        memcpy(&out[at + 4 * i], &w, 4);
    }
}

extern "C" mrlbm_status mrlbm_save_vtk(mrlbm_domain* dom, const char* path_files, const char* id_sim, int step)
{
    if (!dom || !path_files || !id_sim) return fail(MRLBM_EINVAL, "null argument");
    const mrlbm_desc& d = dom->d;
    const size_t n = (size_t)d.nx * d.ny * d.nz;
    mrlbm_status st = mkdirs(std::string(path_files) + "/" + id_sim);
    if (st) return st;
    const bool has_om = d.rheology != MRLBM_NEWTONIAN;
    std::vector<float> rho(n), ux(n), uy(n), uz(n), om, cv;
    if (has_om) om.resize(n);
    if ((st = mrlbm_get_macr(dom, rho.data(), ux.data(), uy.data(), uz.data(), has_om ? om.data() : nullptr)))
        return st;
    if (d.thermal && (st = thermal_scalar(dom, cv))) return st;
    std::string out;
    out.reserve(n * 16 + 512);
    char head[512];
    snprintf(head, sizeof(head),
             "# vtk DataFile Version 3.0\nLBM output (binary)\nBINARY\nDATASET STRUCTURED_POINTS\n"
             "DIMENSIONS %d %d %d\nORIGIN 0 0 0\nSPACING 1 1 1\nPOINT_DATA %zu\n",
             d.nx, d.ny, d.nz, n);
    out += head;
    out += "SCALARS rho float 1\nLOOKUP_TABLE default\n";
    put_be(out, rho.data(), n);
    out += "VECTORS velocity float\n";
    {
        std::vector<float> v(3 * n);
        for (size_t i = 0; i < n; i++) {
            v[3 * i] = ux[i] / 3.0f;
            v[3 * i + 1] = uy[i] / 3.0f;
            v[3 * i + 2] = uz[i] / 3.0f;
        }
        put_be(out, v.data(), 3 * n);
    }
    if (has_om) {
        out += "SCALARS omega float 1\nLOOKUP_TABLE default\n";
        put_be(out, om.data(), n);
    }
    if (d.thermal) {  // src/saveData.cu:371-376
        out += "SCALARS C float 1\nLOOKUP_TABLE default\n";
        put_be(out, cv.data(), n);
    }
    return write_file(var_filename(path_files, id_sim, "vtk", (unsigned)step, ".vtk"), out.data(), out.size());
}

// Same keys and number formatting as getSimInfoString (src/saveData.cu:469-613),
// which the reference's reader parses (post/fileTreat.py:61-150).  by / bz:
// the step's rows per CTA and z planes per CTA (the reference's BLOCK_NY / NZ).
static std::string info_text(const mrlbm_desc& d, const char* id_sim, const char* case_name, int nsteps, double mlups,
                             int by, int bz)
{
    std::string t;
    char line[256];
    auto put = [&](const char* fmt, auto... v) {
        snprintf(line, sizeof(line), fmt, v...);
        t += line;
    };
    put("---------------------------- SIMULATION INFORMATION ----------------------------\n");
    put("      Simulation ID: %s\n", id_sim);
    put("       Velocity set: D3Q%d\n", d.lattice);
    put("          Precision: %s\n", d.storage == MRLBM_F32    ? "float"
                                    : d.storage == MRLBM_F16  ? "half"
                                    : d.storage == MRLBM_F16U ? "half-split-velocity"
                                                              : "bfloat16");
    put("                 NX: %d\n", d.nx);
    put("                 NY: %d\n", d.ny);
    put("                 NZ: %d\n", d.nz);
    put("           NZ_TOTAL: %d\n", d.nz);
    put("                Tau: %.6e\n", d.tau);
    double umax = 0.0;
    for (int k = 0; k < 4; k++)
        for (int a = 0; a < 3; a++) umax = std::max(umax, std::fabs(d.bc_velocity[k][a]));
    put("               Umax: %.6e\n", umax);
    put("                 FX: %.6e\n", d.force[0]);
    put("                 FY: %.6e\n", d.force[1]);
    put("                 FZ: %.6e\n", d.force[2]);
    put("         Save steps: %.6e\n", 0.0);
    put("             Nsteps: %d\n", nsteps);
    put("              MLUPS: %.6e\n", mlups);
    put("                 BX: %d\n", TILE_X);
    put("                 BY: %d\n", by);
    put("                 BZ: %d\n", bz);
    put("--------------------------------------------------------------------------------\n");
    put("\n------------------------------ BOUNDARY CONDITIONS -----------------------------\n");
    put("            BC mode: Moment Based \n");
    put("            BC type: %s\n", case_name ? case_name : "runtime");
    put("--------------------------------------------------------------------------------\n");
    if (d.rheology != MRLBM_NEWTONIAN) {
        put("\n------------------------------ NON NEWTONIAN FLUID -----------------------------\n");
        if (d.rheology == MRLBM_POWERLAW) {
            put("              Model: Power-Law\n");
            put("        Power index: %.6e\n", d.nnf_n);
            put(" Consistency factor: %.6e\n", d.nnf_k);
            put("            Gamma 0: %.6e\n", 0.0);
        } else {
            put("              Model: Bingham\n");
            put("  Plastic viscosity: %.6e\n", (1.0 / d.nnf_omega_p - 0.5) / 3.0);
            put("       Yield stress: %.6e\n", d.nnf_yield);
            put("      Plastic omega: %.6e\n", d.nnf_omega_p);
        }
        put("--------------------------------------------------------------------------------\n");
    }
    return t;
}

extern "C" mrlbm_status mrlbm_save_info(mrlbm_domain* dom, const char* path_files, const char* id_sim,
                                         const char* case_name, int nsteps, double mlups)
{
    if (!dom || !path_files || !id_sim) return fail(MRLBM_EINVAL, "null argument");
    mrlbm_status st = mkdirs(std::string(path_files) + "/" + id_sim);
    if (st) return st;
    StepArgs sa;
    int flags = 0;
    fill_step_args(dom, sa, dom->cur, flags);
    const std::string t = info_text(dom->d, id_sim, case_name, nsteps, mlups, tile_rows(flags), sa.lz);
    return write_file(std::string(path_files) + "/" + id_sim + "/" + id_sim + "_info.txt", t.data(), t.size());
}

// The same text for a description alone, on the host (no device work): the
// step's geometry is that of a domain without wall classes on a 148-SM B200,
// stepped tile-ordered (the default).
extern "C" mrlbm_status mrlbm_info_text(const mrlbm_desc* d, const char* id_sim, const char* case_name, int nsteps,
                                        double mlups, char* buf, size_t cap, size_t* len)
{
    if (!d || !id_sim || !len) return fail(MRLBM_EINVAL, "null argument");
    mrlbm_domain tmp;
    tmp.d = *d;
    tmp.nsm = 148;
    const int flags = (d->rheology != MRLBM_NEWTONIAN ? F_POWERLAW | F_BC : 0) | (d->thermal ? F_THERMAL : 0);
    const int by = tile_rows(flags);
    const int lz = tile_ordered(&tmp, flags) ? choose_lz_overlap(&tmp, by) : choose_lz(&tmp, by);
    const std::string t = info_text(*d, id_sim, case_name, nsteps, mlups, by, lz);
    *len = t.size();
    if (buf) {
        if (cap < t.size() + 1) return fail(MRLBM_EINVAL, "buffer of %zu bytes, the text needs %zu", cap, t.size() + 1);
        memcpy(buf, t.c_str(), t.size() + 1);
    }
    return MRLBM_OK;
}
