// bvh/sdf_rebuild.hpp -- the reference's include path for the level-set functions
// (serial/bvh/sdf_rebuild.hpp); they are declared in ssdf.hpp with the rest of the drop-in API.
#ifndef SSDF_B200_BVH_SDF_REBUILD_HPP
#define SSDF_B200_BVH_SDF_REBUILD_HPP
#include "../ssdf.hpp"
#endif
