#define VF_ID 0
#include "vol_impl.cuh"
