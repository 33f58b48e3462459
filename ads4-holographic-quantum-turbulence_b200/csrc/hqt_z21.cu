// Column kernels for columns of up to 21 Chebyshev points.
#define HQT_ZN 21
#include "hqt_z_impl.cuh"
