// passes_f32_3.cu -- FFT pass launchers and kernels for float fields of 3 components.
#include "passes.cuh"

PMGPU_INSTANTIATE_PASSES(float, 3, f32_3)
PMGPU_INSTANTIATE_BATCH(float, 3)
