// batch_kernel.cuh -- persistent z-march over many independent domains.
//
// A batch packs the columns of many domains of uneven sizes into one work list.
// Each persistent CTA (one per SM) takes the next column from a global ticket
// counter and runs the same z-march as the single-domain kernel on it; the
// last CTA to finish resets the counter and advances the batch step, so the
// launch can be replayed from a CUDA graph with no host work between steps.
#pragma once
#include "kernels.cuh"

namespace mrlbm {

// rows per CTA: either tile height of the single-domain kernels (members
// share their tensor maps), 8 with two CTAs per SM or 14 with one; the batch
// starts at this one (8, except D3Q27 split-velocity fp16 batches, whose 15
// stored words of a power-law member spill at 8 rows) and its autotuner
// measures both
__host__ __device__ constexpr int batch_tyi(int q, int s) { return (q == 27 && s != 0) ? TYI_WALL : TYI_BULK; }
// static shared memory of the batch kernel (the work item and its step
// arguments), kept out of the ring's share
constexpr int BATCH_STATIC_SMEM = 512;
// moment pairs a ring slot holds: the largest flag set's (power law, with
// the split storage's low words when S = F_SPLITU)
template <typename T, int S>
__host__ __device__ constexpr int batch_npm()
{
    return npairs_of(F_BC | F_POWERLAW | S);
}

// Per-domain data the batched kernel needs; both parities are precomputed so
// the kernel only selects.  64-byte aligned for the tensor maps.
struct alignas(64) BatchDomain {
    CUtensorMap map[2];  // TMA maps over moment buffers 0 and 1
    StepArgs args[2];    // args[p]: read buffer p, write buffer p^1
    int flags;           // F_* set of this domain
    int parity_offset;   // parity of buffer read at batch step s: (s + offset) & 1
    int pad[14];
};

struct BatchItem {
    int dom;
    int X0, Y0, z0;
};

// Device-side queue control (one per batch).
struct BatchCtl {
    int next;    // ticket counter
    int done;    // CTAs finished in this launch
    int step;    // batch step count (parity source)
    int nitems;  // active work items
};

// D3Q19 batches stage the class table of the member a work item belongs to
// (each member has its own), as the single-domain wall kernels do
__host__ __device__ constexpr bool batch_stages(int q) { return q == 19; }

template <int Q, typename T, int FLAGS, int TYI>
__device__ __forceinline__ bool batch_column(
    const StepArgs& a, const CUtensorMap* map, const BatchItem& it,
    const ZSmem<Q, T, TYI, batch_npm<T, FLAGS & F_SPLITU>(), false, BATCH_STATIC_SMEM, batch_stages(Q)>& sm,
    unsigned& g0)
{
    // one generic-pointer solve for every flag set: the batch kernel holds
    // them all, and two inlined solves per set spill
    using BCP = std::conditional_t<batch_stages(Q), TableBCGeneric, TableBC>;
    return zmarch_column<Q, T, FLAGS, TYI, BCP>(a, map, it.X0, it.Y0, it.z0, min(it.z0 + a.lz, a.nz), sm, g0);
}

// S = F_SPLITU for split-storage fp16 batches (their members' flag sets carry
// it), else 0: one kernel per storage kind keeps each kernel's code and
// register demand to the flag sets it can meet.
template <int Q, typename T, int S, int TYI>
__global__ void __launch_bounds__(32 * (TYI + 2), ctas_per_sm(TYI))
    batch_step(const BatchDomain* __restrict__ doms, const BatchItem* __restrict__ items, BatchCtl* ctl)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item;
    __shared__ __align__(16) StepArgs s_args;
    static_assert(sizeof(StepArgs) + 16 <= BATCH_STATIC_SMEM, "batch static shared memory");
    // ring slots for the largest flag set
    using SMT = ZSmem<Q, T, TYI, batch_npm<T, S>(), false, BATCH_STATIC_SMEM, batch_stages(Q)>;
    const SMT sm(smem);
    zmarch_init_barriers(sm);  // nothing staged yet
    int staged_dom = -1;
    const int step = *((volatile int*)&ctl->step);
    const int nitems = *((volatile int*)&ctl->nitems);
    unsigned g0 = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&ctl->next, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) break;
        const BatchItem item = items[it];
        const BatchDomain& D = doms[item.dom];
        const int par = (step + D.parity_offset) & 1;
        constexpr int NW = (int)(sizeof(StepArgs) / 4);
        if (threadIdx.x < NW)
            reinterpret_cast<int*>(&s_args)[threadIdx.x] = reinterpret_cast<const int*>(&D.args[par])[threadIdx.x];
        if constexpr (SMT::CT > 0) {
            // another member: its classes (the previous column's reads of the
            // staged table ended at that column's last barrier)
            if (item.dom != staged_dom) {
                const int nbc = D.args[par].nbc;
                const int n = nbc < SMT::CT ? nbc : SMT::CT;
                const float4* src = reinterpret_cast<const float4*>(D.args[par].bc);
                float4* dst = reinterpret_cast<float4*>(dyn_smem() + 128);
                for (int i = threadIdx.x; i < n * (int)(sizeof(BcClass) / 16); i += blockDim.x) dst[i] = __ldg(src + i);
                if (threadIdx.x == 0) *reinterpret_cast<int*>(dyn_smem() + HDR_STAGED_CLASSES) = n;
                staged_dom = item.dom;
            }
        }
        __syncthreads();
        bool ok = true;
        switch (D.flags) {
            case S: ok = batch_column<Q, T, S, TYI>(s_args, &D.map[par], item, sm, g0); break;
            case S | F_BC: ok = batch_column<Q, T, S | F_BC, TYI>(s_args, &D.map[par], item, sm, g0); break;
            case S | F_BC | F_FORCE: ok = batch_column<Q, T, S | F_BC | F_FORCE, TYI>(s_args, &D.map[par], item, sm, g0); break;
            case S | F_BC | F_FORCE | F_POWERLAW:
                ok = batch_column<Q, T, S | F_BC | F_FORCE | F_POWERLAW, TYI>(s_args, &D.map[par], item, sm, g0);
                break;
            default: break;  // rejected on the host when the domain joins
        }
        if (!ok) break;
    }
    // the last CTA out resets the ticket counter and advances the step; every
    // CTA has taken its last ticket before it counts itself done
    if (threadIdx.x == 0) {
        __threadfence();
        const int d = atomicAdd(&ctl->done, 1);
        if (d == (int)gridDim.x - 1) {
            ctl->next = 0;
            ctl->done = 0;
            ctl->step = step + 1;
            __threadfence();
        }
    }
}

}  // namespace mrlbm
