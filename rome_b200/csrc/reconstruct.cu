// M-step reconstruction (MyBackProjector::reconstruct) - being implemented.
#include "common.cuh"

using namespace rome;

extern "C" int rome_gpu_reconstruct(RomeGpuCtx* ctx, const RomeReconIn* in, RomeReconOut* out) {
    if (!ctx || !in || !out) return ROME_ERR_ARG;
    return guarded(ctx, [&] { fail(ROME_ERR_UNSUPPORTED, "rome_gpu_reconstruct is not available in this build"); });
}
