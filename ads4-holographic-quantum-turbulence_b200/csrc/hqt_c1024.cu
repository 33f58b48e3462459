// Line transforms of compile-time length 1024.
#define HQT_CN 1024
#include "hqt_c_impl.cuh"
