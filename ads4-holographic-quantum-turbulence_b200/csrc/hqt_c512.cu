// Line transforms of compile-time length 512.
#define HQT_CN 512
#include "hqt_c_impl.cuh"
