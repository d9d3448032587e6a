// Test infrastructure: drives the library's host-side precomputation, file
// I/O and mesh validation (vfray_b200/csrc/precomp.cc, vfr_validate.cc)
// through their C ABI in a build with AddressSanitizer and
// UndefinedBehaviorSanitizer, which abort on the first invalid access.
//
//   sanitize_host <mesh.off> <workdir>
//
// mesh.off: a mesh in the reference's .off layout (large enough that the
// reader takes its chunk-parallel path).  Reads it, precomputes adjacency,
// external faces and limits (all threads), validates the mesh and builds the
// walk records, writes and reads back every file format, the binary cache,
// the psi table source reader and cleanTF.  Prints "ok" and exits 0.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vfr_host.h"
#include "vfray.h"

#define CHECK(x)                                                   \
  do {                                                             \
    const int rc_ = (x);                                           \
    if (rc_ != VFR_OK) {                                           \
      std::fprintf(stderr, "%s:%d %s -> %d\n", __FILE__, __LINE__, #x, rc_); \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  const std::string off = argv[1], dir = argv[2];
  uint32_t nV = 0, nT = 0;
  CHECK(vfr_read_off(off.c_str(), nullptr, &nV, nullptr, &nT));
  std::vector<float> v(4 * (size_t)nV);
  std::vector<uint32_t> t(4 * (size_t)nT);
  CHECK(vfr_read_off(off.c_str(), v.data(), &nV, t.data(), &nT));
  CHECK(vfr_normalize(v.data(), nV));
  std::vector<uint32_t> con(4 * (size_t)nT);
  uint32_t next = 0;
  CHECK(vfr_build_con(t.data(), nT, nV, con.data(), &next, 0));
  std::vector<uint32_t> extf(2 * (size_t)next);
  uint32_t n2 = 0;
  CHECK(vfr_build_extf(con.data(), nT, extf.data(), next, &n2));
  if (n2 != next) return 3;
  float lmt[3];
  CHECK(vfr_build_lmt(v.data(), nV, t.data(), nT, lmt));
  std::string why;
  if (!vfr::validate_mesh(t.data(), con.data(), nV, nT, extf.data(), next, why)) {
    std::fprintf(stderr, "validate: %s\n", why.c_str());
    return 4;
  }
  std::vector<uint32_t> walk(8 * (size_t)nT);
  if (!vfr::build_walk(t.data(), con.data(), nV, nT, walk.data(), why)) return 5;
  float mv[16] = {0, 0, 1, 0, 0, 1, 0, 0, -1, 0, 0, 0, 0, 0, 0, 1};
  std::vector<float> r(v);
  CHECK(vfr_rotate(r.data(), nV, mv));
  CHECK(vfr_normalize(r.data(), nV));
  // every file format, written and read back
  std::vector<float> tf(1024);
  CHECK(vfr_default_tf(tf.data()));
  const std::string b = dir + "/m";
  CHECK(vfr_write_off((b + ".off").c_str(), v.data(), nV, t.data(), nT));
  CHECK(vfr_write_con((b + ".con").c_str(), con.data(), nT, next));
  CHECK(vfr_write_extf((b + ".extf").c_str(), extf.data(), next));
  CHECK(vfr_write_lmt((b + ".lmt").c_str(), lmt));
  CHECK(vfr_write_tf((b + ".tf").c_str(), tf.data()));
  std::vector<uint32_t> con2(4 * (size_t)nT), extf2(2 * (size_t)next);
  uint32_t nT2 = nT, ne2 = 0, ne3 = next;  // in: capacities
  CHECK(vfr_read_con((b + ".con").c_str(), con2.data(), &nT2, &ne2));
  CHECK(vfr_read_extf((b + ".extf").c_str(), extf2.data(), &ne3));
  float lmt2[3];
  std::vector<float> tf2(1024);
  CHECK(vfr_read_lmt((b + ".lmt").c_str(), lmt2));
  CHECK(vfr_read_tf((b + ".tf").c_str(), tf2.data()));
  if (con2 != con || extf2 != extf || tf2 != tf) return 6;
  CHECK(vfr_write_mesh_cache((b + ".vfrb").c_str(), v.data(), nV, t.data(), con.data(), nT,
                             extf.data(), next, lmt));
  uint32_t cV = 0, cT = 0, cE = 0;
  CHECK(vfr_read_mesh_cache((b + ".vfrb").c_str(), nullptr, &cV, nullptr, nullptr, &cT, nullptr, &cE,
                            nullptr));
  std::vector<float> cv(4 * (size_t)cV), clmt(3);
  std::vector<uint32_t> ct(4 * (size_t)cT), cc(4 * (size_t)cT), ce(2 * (size_t)cE);
  CHECK(vfr_read_mesh_cache((b + ".vfrb").c_str(), cv.data(), &cV, ct.data(), cc.data(), &cT,
                            ce.data(), &cE, clmt.data()));
  if (cv != v || ct != t || cc != con || ce != extf) return 7;
  // the psi table: generated, written as a C source, parsed back
  std::vector<float> psi(512 * 512), psi2(512 * 512);
  CHECK(vfr_psi_table(psi.data()));
  {
    FILE* f = std::fopen((b + "_psi.h").c_str(), "w");
    if (!f) return 8;
    std::fprintf(f, "/* notice */\nfloat psiGammaTable[512][512] = {\n");
    for (size_t i = 0; i < psi.size(); ++i) std::fprintf(f, "%.9gf,%s", psi[i], (i % 8 == 7) ? "\n" : " ");
    std::fprintf(f, "};\n");
    std::fclose(f);
  }
  CHECK(vfr_read_psi_source((b + "_psi.h").c_str(), psi2.data()));
  if (psi2 != psi) return 9;
  // cleanTF on the old layout
  {
    FILE* f = std::fopen((b + "_old.tf").c_str(), "w");
    if (!f) return 10;
    for (int i = 0; i < 7; ++i) std::fprintf(f, "header %d\n", i);
    for (int i = 0; i < 256; ++i) std::fprintf(f, "%d %g %g %g %g\n", i, i / 255.0, 0.5, 1 - i / 255.0, 0.25);
    std::fclose(f);
  }
  CHECK(vfr_clean_tf((b + "_old.tf").c_str(), (b + "_clean.tf").c_str()));
  // bad inputs are refused, not read past
  if (vfr_read_off((dir + "/missing.off").c_str(), nullptr, &nV, nullptr, &nT) == VFR_OK) return 11;
  std::printf("ok %u verts %u tets %u ext\n", nV, nT, next);
  return 0;
}
