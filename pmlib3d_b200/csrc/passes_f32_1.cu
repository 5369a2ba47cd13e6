// passes_f32_1.cu -- FFT pass launchers and kernels for float fields of 1 component.
#include "passes.cuh"

PMGPU_INSTANTIATE_PASSES(float, 1, f32_1)
