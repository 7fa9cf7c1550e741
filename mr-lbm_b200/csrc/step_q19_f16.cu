// Step-kernel variants for D3Q19 with __half moment storage.
#include "step_dispatch.cuh"
template mrlbm_status mrlbm::dispatch_step<19, __half>(const CUtensorMap*, const mrlbm::StepArgs&, int, cudaStream_t, bool);
