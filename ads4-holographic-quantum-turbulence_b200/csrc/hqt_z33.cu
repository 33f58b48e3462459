// Column kernels for columns of up to 33 Chebyshev points.
#define HQT_ZN 33
#include "hqt_z_impl.cuh"
