// Column kernels for columns of up to 25 Chebyshev points.
#define HQT_ZN 25
#include "hqt_z_impl.cuh"
