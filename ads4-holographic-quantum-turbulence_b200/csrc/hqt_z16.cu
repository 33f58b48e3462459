// Column kernels for columns of up to 16 Chebyshev points.
#define HQT_ZN 16
#include "hqt_z_impl.cuh"
