#define VF_ID 2
#include "vol_impl.cuh"
