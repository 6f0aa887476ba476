#define VF_ID 1
#include "vol_impl.cuh"
