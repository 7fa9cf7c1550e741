// domain.h -- internal state of one MR-LBM domain (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/mrlbm.h"
#include "kernels.cuh"

namespace mrlbm {

constexpr int GRAPH_STEPS = 16;  // launches per captured graph (even: parities chain)

}  // namespace mrlbm

// HBM layout: the nm moments are stored in pairs (moments 2p, 2p + 1); each
// pair is a plane stack [z+1][y+1][x+XOFF][2] with a one-node ghost shell
// (z = -1..nz, y = -1..ny, x = -1..nx; pitch = nx + XOFF + 1 rounded up to 8
// nodes, so rows are 16-byte aligned for TMA), in the domain's storage type;
// an odd moment count is padded to a full pair (mphys() gives the element of
// moment m at node offset pidx()).  Two such buffers ping-pong (step n reads
// m[cur] and writes m[cur^1]).  Node classes are one byte per node in the
// padded node layout.
struct mrlbm_domain {
    mrlbm_desc d{};
    int q = 19, nm = 10;
    int nms = 10;                    // stored words per node: nm, + 3 low words of 3u with split-velocity storage
    size_t esize = 4;
    int pitch = 0;
    long long plane = 0, field = 0;
    double omega0 = 1.0;
    void* m[2] = {nullptr, nullptr};
    int cur = 0;
    int step = 0;
    uint8_t* cls = nullptr;
    int* err = nullptr;              // device flag: a bounded wait timed out
    CUtensorMap tmap[2][2];          // TMA maps [moment buffer][tile kind: TYI_BULK, TYI_WALL rows]
    mrlbm::BcClass* bc = nullptr;
    int nclasses = 0;
    bool has_bc = false;
    bool has_outflow = false;        // some class is an outflow wall (not taken by batches)
    float ext[mrlbm::NM_MAX] = {};
    float scale[mrlbm::NM_MAX] = {}, iscale[mrlbm::NM_MAX] = {};
    int lz = 0;                      // z planes per work item when a batch has set it (0: single-domain choice)
    int lz_t[2] = {16, 16};          // single-domain z planes per CTA, per tile kind
    int lz_o[2] = {16, 16};          // the same for tile-ordered (overlapping) steps
    int nsm = 148;                   // SMs of the device the domain lives on
    cudaStream_t stream = nullptr;      // where the domain's work is queued
    cudaStream_t own_stream = nullptr;  // the stream the domain created (stream unless mrlbm_set_stream)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t xev = nullptr;          // stream ordering (set_stream, z-slab copies)
    int device = 0;
    double* red_scratch = nullptr;  // block partials + 8 results
    double* red_host = nullptr;     // pinned
    int red_blocks = 0;
    float* usnap = nullptr;         // residual snapshot (3 floats per node)
    float* stage = nullptr;         // float staging buffer for layout conversions
    bool have_snap = false;
    cudaGraphExec_t graph_exec = nullptr;
    // tile-ordered steps (zmarch_step): ticket counter + a word per tile
    bool tile_order = true;
    unsigned* sched = nullptr;
    size_t sched_words = 0;
    long long sched_key = -1;  // grid the state belongs to (x, y, z tiles)
};

namespace mrlbm {

mrlbm_status fail(mrlbm_status st, const char* fmt, ...);
uint32_t known_mask(int q, uint32_t octants);
mrlbm_status build_bc_class(int q, int mq, uint32_t word, const double uvel[4][3], double omega0, BcClass* out);
mrlbm_status classify_nodes(int q, int mq, const uint32_t* nt, long long n, const double uvel[4][3], double omega0,
                            std::vector<uint8_t>& cls, std::vector<BcClass>& table, bool& any_bc,
                            bool case_mode = false, const double* t_wall = nullptr);
void storage_scales(int storage, int nm, float* scale, float* iscale);
// storages kept as fp16 words (plain, or with split velocity)
inline bool is_half_storage(int storage) { return storage == MRLBM_F16 || storage == MRLBM_F16U; }
mrlbm_status domain_alloc(mrlbm_domain* dom);
int choose_lz(const mrlbm_domain* dom, int tyi);
int choose_lz_overlap(const mrlbm_domain* dom, int tyi);
// whether a step with these flags is tile-ordered (overlapping launches)
bool tile_ordered(const mrlbm_domain* dom, int flags);
void fill_step_args(const mrlbm_domain* dom, StepArgs& a, int parity, int& flags);
// chained: the launch before this one on s is this domain's step
mrlbm_status enqueue_step(mrlbm_domain* dom, int parity, cudaStream_t s, bool chained);
mrlbm_status prepare_tile_order(mrlbm_domain* dom, cudaStream_t s);
// maps: the read buffer's two tensor maps (tile kinds TYI_BULK, TYI_WALL)
template <int Q, typename T>
mrlbm_status dispatch_step(const CUtensorMap* maps, const StepArgs& a, int flags, cudaStream_t s, bool pdl);
mrlbm_status make_tensor_maps(mrlbm_domain* dom);
mrlbm_status fill_ghosts(mrlbm_domain* dom);
mrlbm_status check_device_error(mrlbm_domain* dom);
mrlbm_status enqueue_reduce(mrlbm_domain* dom, double* partial, double* out, int residual_mode, cudaStream_t s);

}  // namespace mrlbm
