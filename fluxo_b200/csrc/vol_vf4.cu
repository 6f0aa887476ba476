#define VF_ID 4
#include "vol_impl.cuh"
