#define VF_ID 8
#include "vol_impl.cuh"
