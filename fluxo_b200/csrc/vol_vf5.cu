#define VF_ID 5
#include "vol_impl.cuh"
