// Line transforms of compile-time length 256.
#define HQT_CN 256
#include "hqt_c_impl.cuh"
