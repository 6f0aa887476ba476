#define VF_ID 10
#include "vol_impl.cuh"
