// bvh/bvh.hpp -- the reference's include path for the BVH entry points (serial/bvh/bvh.hpp); they
// are declared in ssdf.hpp with the rest of the drop-in API.
#ifndef SSDF_B200_BVH_BVH_HPP
#define SSDF_B200_BVH_BVH_HPP
#include "../ssdf.hpp"
#endif
