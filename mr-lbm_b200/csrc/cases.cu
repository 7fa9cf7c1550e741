// cases.cu -- host-side node-type builders for the run-time case mode
// (the reference does this in each case's bc_initialization.inc and, for voxel
// geometries, in bc_id / define_voxel_bc).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/mrlbm.h"
#include "domain.h"

using namespace mrlbm;

// Octant bits touched by a solid neighbour at offset (dx,dy,dz): every octant
// whose signs agree with the non-zero components (src/lbmInitialization.cu:1080-1227).
static uint32_t octants_of(int dx, int dy, int dz)
{
    uint32_t m = 0;
    for (int o = 0; o < 8; o++) {
        const int s[3] = {(o & 1) ? 1 : -1, (o & 2) ? 1 : -1, (o & 4) ? 1 : -1};
        const int d[3] = {dx, dy, dz};
        bool ok = true;
        for (int a = 0; a < 3; a++)
            if (d[a] != 0 && d[a] != s[a]) ok = false;
        if (ok) m |= 1u << o;
    }
    return m;
}

extern "C" mrlbm_status mrlbm_voxel_node_types(int nx, int ny, int nz, const uint8_t* solid, const int periodic[3],
                                                uint32_t* out)
{
    if (nx < 1 || ny < 1 || nz < 1 || !solid || !periodic || !out) return fail(MRLBM_EINVAL, "bad argument");
    const int n[3] = {nx, ny, nz};
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const size_t k = (size_t)x + (size_t)nx * (y + (size_t)ny * z);
                if (solid[k]) { out[k] = MRLBM_NODE_SOLID; continue; }
                uint32_t m = 0;
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dx = -1; dx <= 1; dx++) {
                            if (!dx && !dy && !dz) continue;
                            int c[3] = {x + dx, y + dy, z + dz};
                            bool is_solid = false, outside = false;
                            for (int a = 0; a < 3; a++) {
                                if (c[a] < 0 || c[a] >= n[a]) {
                                    if (periodic[a]) c[a] = (c[a] + n[a]) % n[a];
                                    else outside = true;
                                }
                            }
                            if (outside) is_solid = true;
                            else is_solid = solid[(size_t)c[0] + (size_t)nx * (c[1] + (size_t)ny * c[2])] != 0;
                            if (is_solid) m |= octants_of(dx, dy, dz);
                        }
                // a fluid node whose every octant is blocked keeps a valid wall type
                out[k] = (m == 0xFFu) ? 0xFEu : m;
            }
    return MRLBM_OK;
}

// The reference's 3-D lid-driven cavity typing
// (src/cases/lidDrivenCavity_3D/bc_initialization.inc:1-100): the y = NY-1 face
// including its edges and corners is the moving lid (NORTH octants), the other
// boundary nodes get the face/edge/corner octant masks of no-slip walls.
extern "C" mrlbm_status mrlbm_lid_cavity_node_types(int nx, int ny, int nz, int lid_velocity_index, uint32_t* out)
{
    if (nx < 2 || ny < 2 || nz < 2 || !out || lid_velocity_index < 0 || lid_velocity_index > 3)
        return fail(MRLBM_EINVAL, "bad argument");
    const uint32_t W = 0x55u, E = 0xAAu, S = 0x33u, N = 0xCCu, B = 0x0Fu, F = 0xF0u;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const size_t k = (size_t)x + (size_t)nx * (y + (size_t)ny * z);
                uint32_t t = 0;
                if (y == ny - 1) {
                    t = N | MRLBM_BC_VELOCITY_WALL | MRLBM_BC_VELOCITY_INDEX(lid_velocity_index);
                } else {
                    if (y == 0) t |= S;
                    if (x == 0) t |= W;
                    if (x == nx - 1) t |= E;
                    if (z == 0) t |= B;
                    if (z == nz - 1) t |= F;
                }
                out[k] = t;
            }
    return MRLBM_OK;
}

extern "C" mrlbm_status mrlbm_bc_class_info(int lattice, int bc_matrix_q, uint32_t node_type,
                                            const double bc_velocity[4][3], double omega0, float* out, uint32_t* known)
{
    if ((lattice != 19 && lattice != 27) || !bc_velocity || !out || !known) return fail(MRLBM_EINVAL, "bad argument");
    const int mq = bc_matrix_q ? bc_matrix_q : 19;
    BcClass c;
    mrlbm_status st = build_bc_class(lattice, mq, node_type, bc_velocity, omega0, &c);
    if (st) return st;
    memcpy(out, c.ainv, 49 * sizeof(float));
    memcpy(out + 49, c.v, 7 * sizeof(float));
    memcpy(out + 56, c.qa, 7 * sizeof(float));
    out[63] = c.s;
    memcpy(out + 64, c.u, 3 * sizeof(float));
    *known = c.known;
    return MRLBM_OK;
}

// The reference's voxel-file loading (read_xyz_file, src/lbmInitialization.cu:
// 978-1039): every line "x,y,z" of the CSV marks node (x, y, z) solid (0xFF)
// and its 26 neighbours (each axis wrapped periodically) unresolved
// (0xFFFFFFFF) unless they are solid already; lines outside the grid are
// skipped.  node_types is x-fastest and keeps its other values.
extern "C" mrlbm_status mrlbm_voxel_mark_csv(const char* path, int nx, int ny, int nz, uint32_t* node_types,
                                             long long* voxels)
{
    if (!path || !node_types || nx < 1 || ny < 1 || nz < 1) return fail(MRLBM_EINVAL, "bad argument");
    FILE* f = fopen(path, "r");
    if (!f) return fail(MRLBM_EIO, "cannot open voxel file %s", path);
    long long count = 0;
    char line[256];
    auto idx = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); };
    while (fgets(line, sizeof(line), f)) {
        char* p = line;
        char* e = nullptr;
        long v[3];
        bool ok = true;
        for (int k = 0; k < 3 && ok; k++) {
            v[k] = strtol(p, &e, 10);
            if (e == p) ok = false;
            p = e;
            if (k < 2) {
                if (*p != ',') ok = false;
                else p++;
            }
        }
        if (!ok) continue;   // blank or malformed line
        if (v[0] < 0 || v[1] < 0 || v[2] < 0 || v[0] >= nx || v[1] >= ny || v[2] >= nz) continue;
        const int x = (int)v[0], y = (int)v[1], z = (int)v[2];
        const size_t c = idx(x, y, z);
        node_types[c] = MRLBM_NODE_SOLID;
        count++;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const size_t k = idx((x + dx + nx) % nx, (y + dy + ny) % ny, (z + dz + nz) % nz);
                    if (k == c || node_types[k] == MRLBM_NODE_SOLID) continue;
                    node_types[k] = MRLBM_NODE_UNRESOLVED;
                }
    }
    fclose(f);
    if (voxels) *voxels = count;
    return MRLBM_OK;
}

// The reference's define_voxel_bc + bc_id (src/lbmInitialization.cu:1058-1227):
// every unresolved node (0xFFFFFFFF) takes the octant mask of its solid
// neighbours, each axis wrapped periodically (a mask of all eight octants is
// the solid word 0xFF, as in the reference).
extern "C" mrlbm_status mrlbm_voxel_resolve(int nx, int ny, int nz, uint32_t* node_types)
{
    if (!node_types || nx < 1 || ny < 1 || nz < 1) return fail(MRLBM_EINVAL, "bad argument");
    auto idx = [&](int x, int y, int z) { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * z); };
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const size_t c = idx(x, y, z);
                if (node_types[c] != MRLBM_NODE_UNRESOLVED) continue;
                uint32_t m = 0;
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dx = -1; dx <= 1; dx++) {
                            if (!dx && !dy && !dz) continue;
                            const size_t k = idx((x + dx + nx) % nx, (y + dy + ny) % ny, (z + dz + nz) % nz);
                            if (node_types[k] == MRLBM_NODE_SOLID) m |= octants_of(dx, dy, dz);
                        }
                node_types[c] = m;
            }
    return MRLBM_OK;
}
