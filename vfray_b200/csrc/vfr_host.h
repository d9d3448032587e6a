// Host-only helpers of the render library shared by its .cc and .cu files.
#pragma once
#include <cstdint>
#include <string>

namespace vfr {

// Ids in range, adjacency that points back, external faces that are boundary
// faces (vfr_validate.cc).
bool validate_mesh(const uint32_t* tet4, const uint32_t* con4, uint32_t nV, uint32_t nT,
                   const uint32_t* extf2, uint32_t nExt, std::string& why);

// Walk records: per tet 8 words (4 neighbour ids, 4 packed opposite-vertex
// words); nV must be below 2^27 (vfr_validate.cc).
bool build_walk(const uint32_t* tet4, const uint32_t* con4, uint32_t nV, uint32_t nT,
                uint32_t* walk8, std::string& why);

}  // namespace vfr
