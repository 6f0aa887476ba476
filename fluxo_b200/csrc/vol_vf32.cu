#define VF_ID 32
#include "vol_impl.cuh"
