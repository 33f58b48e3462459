// Line transforms of compile-time length 128.
#define HQT_CN 128
#include "hqt_c_impl.cuh"
