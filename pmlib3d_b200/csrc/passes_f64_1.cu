// passes_f64_1.cu -- FFT pass launchers and kernels for double fields of 1 component.
#include "passes.cuh"

PMGPU_INSTANTIATE_PASSES(double, 1, f64_1)
