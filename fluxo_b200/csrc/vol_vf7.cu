#define VF_ID 7
#include "vol_impl.cuh"
