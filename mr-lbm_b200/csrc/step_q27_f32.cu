// Step-kernel variants for D3Q27 with float moment storage.
#include "step_dispatch.cuh"
template mrlbm_status mrlbm::dispatch_step<27, float>(const CUtensorMap*, const mrlbm::StepArgs&, int, cudaStream_t, bool);
