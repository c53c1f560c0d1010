// FP64 instantiation of the step.  Built with --fmad=false (no contraction of
// products into FMA) and IEEE division / square root, so every operation is a
// separately rounded IEEE-754 binary64 operation in the written order.
#include "imhd_launch.cuh"
IMHD_INSTANTIATE(double)
