// Step-kernel variants for D3Q19 with __nv_bfloat16 moment storage.
#include "step_dispatch.cuh"
template mrlbm_status mrlbm::dispatch_step<19, __nv_bfloat16>(const CUtensorMap*, const mrlbm::StepArgs&, int, cudaStream_t, bool);
