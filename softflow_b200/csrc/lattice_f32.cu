// lattice_f32.cu -- FP32 arithmetic lattice kernels for FP32 and
// FP16-shifted population storage.
#include "lattice_launch.cuh"
namespace sfg {
SFG_LATTICE_INST(float, float)
SFG_LATTICE_INST(__half, float)
}
