// Step-kernel variants for D3Q27 with __nv_bfloat16 moment storage.
#include "step_dispatch.cuh"
template mrlbm_status mrlbm::dispatch_step<27, __nv_bfloat16>(const CUtensorMap*, const mrlbm::StepArgs&, int, cudaStream_t, bool);
