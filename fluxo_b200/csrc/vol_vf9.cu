#define VF_ID 9
#include "vol_impl.cuh"
