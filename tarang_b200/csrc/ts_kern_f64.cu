// FP64 instantiation of the kernel launchers.
#define TS_REAL double
#include "ts_kern_impl.cuh"
