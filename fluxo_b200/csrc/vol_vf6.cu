#define VF_ID 6
#include "vol_impl.cuh"
