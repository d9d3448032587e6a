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

namespace vfr {

// The walk record of a tet (see vfr_device.cuh): per face f, the neighbour
// across f, and packed into one word the neighbour's vertex opposite the
// shared face, the face the neighbour is entered through (the first k with
// con[n][k] == t, as vfRayKernelCPU.cc:361-364 searches) and how the
// neighbour orders the shared face's vertices relative to this tet.
bool build_walk(const uint32_t* tet, const uint32_t* con, uint32_t nV, uint32_t nT,
                uint32_t* walk8, std::string& why) {
  static const int P[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  if (nV > (1u << 27)) {
    why = "more than 2^27 vertices";
    return false;
  }
  for (size_t t = 0; t < nT; ++t) {
    uint32_t* w = walk8 + 8 * t;
    for (int f = 0; f < 4; ++f) {
      const uint32_t n = con[4 * t + f];
      w[f] = n;
      if (n == t) {
        w[4 + f] = 7u << 29;
        continue;
      }
      const uint32_t* cn = con + 4 * (size_t)n;
      uint32_t fn = cn[0] == t ? 0 : cn[1] == t ? 1 : cn[2] == t ? 2 : cn[3] == t ? 3 : 4;
      if (fn == 4) {
        why = "adjacency does not point back";
        return false;
      }
      const uint32_t* tt = tet + 4 * t;
      const uint32_t* tn = tet + 4 * (size_t)n;
      int m[3];
      bool ok = true;
      for (int j = 0; j < 3; ++j) {
        const uint32_t id = tn[(fn + j) & 3];
        m[j] = -1;
        for (int k = 0; k < 3; ++k)
          if (tt[(f + k) & 3] == id) m[j] = k;
        ok = ok && m[j] >= 0;
      }
      uint32_t code = 6;  // shared face not matched by ids: the walk reloads the tet
      if (ok)
        for (uint32_t k = 0; k < 6; ++k)
          if (P[k][0] == m[0] && P[k][1] == m[1] && P[k][2] == m[2]) code = k;
      w[4 + f] = tn[(fn + 3) & 3] | (fn << 27) | (code << 29);
    }
  }
  return true;
}

}  // namespace vfr
