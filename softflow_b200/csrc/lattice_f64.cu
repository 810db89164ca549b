// lattice_f64.cu -- FP64 lattice kernels.  Built with --fmad=false so that,
// with the reference's evaluation order, results match the reference engine
// bit for bit.
#include "lattice_launch.cuh"
namespace sfg {
SFG_LATTICE_INST(double, double)
}
