// Line transforms of compile-time length 33.
#define HQT_CN 33
#include "hqt_c_impl.cuh"
