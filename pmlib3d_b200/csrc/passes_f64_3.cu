// passes_f64_3.cu -- FFT pass launchers and kernels for double fields of 3 components.
#include "passes.cuh"

PMGPU_INSTANTIATE_PASSES(double, 3, f64_3)
PMGPU_INSTANTIATE_BATCH(double, 3)
