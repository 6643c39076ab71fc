// pg_launch3.cu -- the 3D (tet4) kernels and their launches.
#define PG_LAUNCH_IMPL
#include "pg_launch.cuh"

namespace pgl {
PG_INSTANTIATE_LAUNCHES(3)
}
