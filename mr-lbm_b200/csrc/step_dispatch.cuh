// step_dispatch.cuh -- launch of the z-marching step kernel for one
// (lattice, storage) pair; instantiated in step_q*_*.cu so the 36 kernel
// variants compile in parallel translation units.
#pragma once
#include <cuda_runtime.h>

#include "domain.h"
#include "kernels.cuh"

namespace mrlbm {

// pdl: the launch before this one on stream s is a tile-ordered step of the
// same domain (a.sched set in both), so this one may start while it finishes
template <int Q, typename T, int FLAGS, typename BCP = table_policy_t<Q, FLAGS>>
static mrlbm_status launch_step_t(const CUtensorMap* maps, const StepArgs& a, cudaStream_t s, bool pdl)
{
    constexpr int TYI = tile_rows(FLAGS);
    constexpr int NW = TYI + 2;
    const CUtensorMap& map = maps[tile_kind(TYI)];
    constexpr size_t smem = step_smem_bytes<Q, T, FLAGS, TYI, BCP>();
    static_assert(smem <= smem_budget(TYI), "shared memory over the sm_100 limit");
    auto kern = zmarch_step<Q, T, FLAGS, TYI, BCP>;
    int dev = 0;
    cudaGetDevice(&dev);
    static int attr_done_mask = 0;  // one bit per device (up to 32)
    if (!(attr_done_mask & (1 << (dev & 31)))) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return fail(MRLBM_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        attr_done_mask |= 1 << (dev & 31);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = zmarch_grid(a.nx, a.ny, a.nz, TYI, a.lz);
    cfg.blockDim = dim3(32 * NW);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, map, a);
    if (e != cudaSuccess) return fail(MRLBM_ECUDA, "step launch: %s", cudaGetErrorString(e));
    return MRLBM_OK;
}

template <int Q, typename T>
mrlbm_status dispatch_step(const CUtensorMap* maps, const StepArgs& a, int flags, cudaStream_t s, bool pdl)
{
    switch (flags) {
        case 0: return launch_step_t<Q, T, 0>(maps, a, s, pdl);
        case F_BC: return launch_step_t<Q, T, F_BC>(maps, a, s, pdl);
        case F_FORCE: return launch_step_t<Q, T, F_FORCE>(maps, a, s, pdl);
        case F_BC | F_FORCE: return launch_step_t<Q, T, F_BC | F_FORCE>(maps, a, s, pdl);
        case F_BC | F_POWERLAW: return launch_step_t<Q, T, F_BC | F_POWERLAW>(maps, a, s, pdl);
        case F_BC | F_FORCE | F_POWERLAW: return launch_step_t<Q, T, F_BC | F_FORCE | F_POWERLAW>(maps, a, s, pdl);
        case F_BC | F_BINGHAM: return launch_step_t<Q, T, F_BC | F_BINGHAM>(maps, a, s, pdl);
        case F_BC | F_FORCE | F_BINGHAM: return launch_step_t<Q, T, F_BC | F_FORCE | F_BINGHAM>(maps, a, s, pdl);
        // outflow walls (Newtonian domains, as the reference's outflow cases)
        case F_BC | F_OUTFLOW: return launch_step_t<Q, T, F_BC, OutflowBC>(maps, a, s, pdl);
        case F_BC | F_FORCE | F_OUTFLOW: return launch_step_t<Q, T, F_BC | F_FORCE, OutflowBC>(maps, a, s, pdl);
        default: break;
    }
    // split-velocity 16-bit storage (no thermal scalar, no outflow walls)
    if constexpr (std::is_same<T, __half>::value) {
        switch (flags) {
            case F_SPLITU: return launch_step_t<Q, T, F_SPLITU>(maps, a, s, pdl);
            case F_SPLITU | F_BC: return launch_step_t<Q, T, F_SPLITU | F_BC>(maps, a, s, pdl);
            case F_SPLITU | F_FORCE: return launch_step_t<Q, T, F_SPLITU | F_FORCE>(maps, a, s, pdl);
            case F_SPLITU | F_BC | F_FORCE: return launch_step_t<Q, T, F_SPLITU | F_BC | F_FORCE>(maps, a, s, pdl);
            case F_SPLITU | F_BC | F_POWERLAW: return launch_step_t<Q, T, F_SPLITU | F_BC | F_POWERLAW>(maps, a, s, pdl);
            case F_SPLITU | F_BC | F_FORCE | F_POWERLAW:
                return launch_step_t<Q, T, F_SPLITU | F_BC | F_FORCE | F_POWERLAW>(maps, a, s, pdl);
            case F_SPLITU | F_BC | F_BINGHAM: return launch_step_t<Q, T, F_SPLITU | F_BC | F_BINGHAM>(maps, a, s, pdl);
            case F_SPLITU | F_BC | F_FORCE | F_BINGHAM:
                return launch_step_t<Q, T, F_SPLITU | F_BC | F_FORCE | F_BINGHAM>(maps, a, s, pdl);
            default: break;
        }
    }
    // thermal scalar: D3Q19 with FP32 storage only (its second row exchange
    // fits next to the D3Q19 flow's in shared memory)
    if constexpr (Q == 19 && is_f32<T>()) {
        if (flags == (F_THERMAL | F_FORCE)) return launch_step_t<Q, T, F_THERMAL | F_FORCE>(maps, a, s, pdl);
        if (flags == (F_THERMAL | F_FORCE | F_BC)) return launch_step_t<Q, T, F_THERMAL | F_FORCE | F_BC>(maps, a, s, pdl);
    }
    return fail(MRLBM_EINVAL, "unsupported step flag combination %d", flags);
}

}  // namespace mrlbm
