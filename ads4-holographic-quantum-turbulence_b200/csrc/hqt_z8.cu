// Column kernels for columns of up to 8 Chebyshev points.
#define HQT_ZN 8
#include "hqt_z_impl.cuh"
