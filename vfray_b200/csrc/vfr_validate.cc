// Mesh validation at upload.  The reference trusts its inputs: an id out of
// range reads past its arrays, and a neighbour that does not point back makes
// vfRay abandon the rest of the face (vfRayKernelCPU.cc:359-365).  Here such
// meshes are refused with VFR_ERR_MESH before anything reaches the device.
#include <cstdio>
#include <string>

#include "vfr_host.h"

namespace vfr {

bool validate_mesh(const uint32_t* tet, const uint32_t* con, uint32_t nV, uint32_t nT,
                   const uint32_t* extf, uint32_t nExt, std::string& why) {
  char buf[160];
  for (size_t i = 0; i < 4 * (size_t)nT; ++i) {
    if (tet[i] >= nV) {
      std::snprintf(buf, sizeof buf, "tet %zu has vertex id %u >= nV %u", i / 4, tet[i], nV);
      why = buf;
      return false;
    }
    if (con[i] >= nT) {
      std::snprintf(buf, sizeof buf, "tet %zu has neighbour id %u >= nT %u", i / 4, con[i], nT);
      why = buf;
      return false;
    }
  }
  for (size_t t = 0; t < nT; ++t)
    for (int f = 0; f < 4; ++f) {
      const uint32_t n = con[4 * t + f];
      if (n == t) continue;
      const uint32_t* b = con + 4 * (size_t)n;
      if (b[0] != t && b[1] != t && b[2] != t && b[3] != t) {
        std::snprintf(buf, sizeof buf,
                      "adjacency does not point back: tet %zu face %d -> tet %u", t, f, n);
        why = buf;
        return false;
      }
    }
  for (size_t e = 0; e < nExt; ++e) {
    const uint32_t t = extf[2 * e], f = extf[2 * e + 1];
    if (t >= nT || f > 3) {
      std::snprintf(buf, sizeof buf, "external face %zu = (%u, %u) out of range", e, t, f);
      why = buf;
      return false;
    }
    if (con[4 * (size_t)t + f] != t) {
      std::snprintf(buf, sizeof buf, "external face %zu = (%u, %u) is not a boundary face", e, t,
                    f);
      why = buf;
      return false;
    }
  }
  return true;
}

}  // namespace vfr
