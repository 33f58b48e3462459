// Line transforms of compile-time length 192.
#define HQT_CN 192
#include "hqt_c_impl.cuh"
