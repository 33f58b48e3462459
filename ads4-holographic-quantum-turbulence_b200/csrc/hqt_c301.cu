// Line transforms of compile-time length 301.
#define HQT_CN 301
#include "hqt_c_impl.cuh"
