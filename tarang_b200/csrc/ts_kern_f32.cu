// FP32 instantiation of the kernel launchers.
#define TS_REAL float
#include "ts_kern_impl.cuh"
