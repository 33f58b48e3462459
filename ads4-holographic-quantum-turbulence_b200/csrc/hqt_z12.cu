// Column kernels for columns of up to 12 Chebyshev points.
#define HQT_ZN 12
#include "hqt_z_impl.cuh"
