// Line transforms of compile-time length 64.
#define HQT_CN 64
#include "hqt_c_impl.cuh"
