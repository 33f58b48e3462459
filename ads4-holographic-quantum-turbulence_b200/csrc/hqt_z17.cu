// Column kernels for columns of up to 17 Chebyshev points.
#define HQT_ZN 17
#include "hqt_z_impl.cuh"
