// FP32 instantiation of the step (bulk arithmetic in binary32 with FMA; the
// dt reduction, the forcing and diagnostic sums and near-degenerate
// eigenvector normalisations stay in FP64).
#include "imhd_launch.cuh"
IMHD_INSTANTIATE(float)
