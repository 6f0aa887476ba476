#define VF_ID 3
#include "vol_impl.cuh"
