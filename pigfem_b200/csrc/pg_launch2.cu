// pg_launch2.cu -- the 2D (tri3) kernels and their launches.
#define PG_LAUNCH_IMPL
#include "pg_launch.cuh"

namespace pgl {
PG_INSTANTIATE_LAUNCHES(2)
}
