// vfRay: the command-line driver of the VF-Ray render path, rewritten over
// the vfray_b200 C ABI (include/vfray.h).  Same command line and files as
// the reference's vfRay.cu:737-936:
//
//   vfRay <volume>       reads ../tet_offs/<volume>.off, normalises it, reads
//                        or computes (and then writes) .con .tf .extf .lmt
//                        next to it, renders 512x512 and writes
//                        <volume>_gpu_img.ppm in the working directory.
//
// Options (all optional, before the volume name): --dir DIR (dataset
// directory, default ../tet_offs/), --size WxH, --psi FILE (a
// psiGammaTable512.h-style table, or "generated" for the table this library
// computes; default: the reference's own table, vfr_psi_table_reference),
// --mode ref|composited, --device N, --out FILE.ppm, --rgba FILE (raw
// float32 RGBA), --steps FILE (raw uint32 steps per pixel), --cache (read
// the normalised mesh, conTet, external faces and limits from <volume>.vfrb
// when present, else read the text files as above and write that cache).
//
// Host-only code: the GPU work happens behind the C ABI.  Unlike the
// reference there is no GLUT viewer (display needs a graphics stack); the
// image goes to the PPM file.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "vfray.h"

namespace {

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

int die(const char* what, int rc, vfr_ctx* ctx = nullptr) {
  std::fprintf(stderr, "%s failed: %s%s%s\n", what, vfr_status_string(rc), ctx ? " - " : "",
               ctx ? vfr_last_error(ctx) : "");
  return 1;
}

bool write_raw(const std::string& path, const void* p, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(p, 1, n, f) == n;
  return (std::fclose(f) == 0) && ok;
}

}  // namespace

int main(int argc, char** argv) {
  std::string dir = "../tet_offs/", psi_path, out_path, rgba_path, steps_path;
  uint32_t W = 512, H = 512;
  int mode = VFR_MODE_REF, device = 0;
  bool use_cache = false;
  const char* volume = nullptr;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto need = [&](const char* opt) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "%s needs a value\n", opt);
        std::exit(1);
      }
      return argv[++i];
    };
    if (a == "--dir") {
      dir = need("--dir");
      if (!dir.empty() && dir.back() != '/') dir += '/';
    } else if (a == "--size") {
      if (std::sscanf(need("--size"), "%ux%u", &W, &H) != 2) return die("--size WxH", VFR_ERR_INVALID);
    } else if (a == "--psi") {
      psi_path = need("--psi");
    } else if (a == "--mode") {
      std::string m = need("--mode");
      mode = (m == "composited") ? VFR_MODE_COMPOSITED : VFR_MODE_REF;
    } else if (a == "--device") {
      device = std::atoi(need("--device"));
    } else if (a == "--out") {
      out_path = need("--out");
    } else if (a == "--rgba") {
      rgba_path = need("--rgba");
    } else if (a == "--steps") {
      steps_path = need("--steps");
    } else if (a == "--cache") {
      use_cache = true;
    } else if (!volume && a[0] != '-') {
      volume = argv[i];
    } else {
      volume = nullptr;
      break;
    }
  }
  if (!volume) {
    std::printf("use: %s [--dir D] [--size WxH] [--psi F] [--mode ref|composited] model\n"
                "Where model can be: spx, blunt, ...\n", argv[0]);
    return 1;
  }
  const std::string base = dir + volume;
  int rc;

  // --- mesh and precomputed files (vfRay.cu:746-842), or the binary cache ---
  std::vector<float> vert;
  std::vector<uint32_t> tet, con, extf;
  uint32_t nV = 0, nT = 0, numExt = 0;
  float lmt[3];
  std::string fn;
  bool from_cache = false;
  const std::string cache = base + ".vfrb";
  std::vector<float> tf(1024);
  auto read_tf_file = [&]() {  // .tf, read or computed and written (vfRay.cu:794-807)
    const std::string f = base + ".tf";
    std::printf("Reading %s file\n", f.c_str());
    if (vfr_read_tf(f.c_str(), tf.data()) != VFR_OK) {
      std::printf("%s file not found!\n Computing TF\n", f.c_str());
      vfr_default_tf(tf.data());
      std::printf("Writing %s file\n", f.c_str());
      vfr_write_tf(f.c_str(), tf.data());
    }
  };
  if (use_cache && vfr_read_mesh_cache(cache.c_str(), nullptr, &nV, nullptr, nullptr, &nT,
                                       nullptr, &numExt, nullptr) == VFR_OK) {
    std::printf("Reading %s (binary cache)\n", cache.c_str());
    vert.resize(4 * (size_t)nV);
    tet.resize(4 * (size_t)nT);
    con.resize(4 * (size_t)nT);
    extf.resize(2 * (size_t)numExt);
    from_cache = vfr_read_mesh_cache(cache.c_str(), vert.data(), &nV, tet.data(), con.data(), &nT,
                                     extf.data(), &numExt, lmt) == VFR_OK;
    if (!from_cache) std::printf("%s unreadable, reading the text files\n", cache.c_str());
  }
  if (!from_cache) {
    fn = base + ".off";
    std::printf("Reading %s file\n", fn.c_str());
    if (vfr_read_off(fn.c_str(), nullptr, &nV, nullptr, &nT) != VFR_OK) {
      std::printf("Cannot read %s aborting!\n", fn.c_str());
      return 1;
    }
    vert.resize(4 * (size_t)nV);
    tet.resize(4 * (size_t)nT);
    if ((rc = vfr_read_off(fn.c_str(), vert.data(), &nV, tet.data(), &nT)) != VFR_OK) {
      std::printf("Cannot read %s aborting!\n", fn.c_str());
      return 1;
    }
    std::printf("Normalizing vertices\n");
    vfr_normalize(vert.data(), nV);

    con.resize(4 * (size_t)nT);
    uint32_t conT = nT;
    fn = base + ".con";
    std::printf("Reading %s file\n", fn.c_str());
    uint32_t hdrT = 0, hdrE = 0;
    bool have = vfr_read_con(fn.c_str(), nullptr, &hdrT, &hdrE) == VFR_OK && hdrT == nT &&
                vfr_read_con(fn.c_str(), con.data(), &conT, &numExt) == VFR_OK;
    if (!have) {
      std::printf("%s file not found!\n Computing conTet\n", fn.c_str());
      if ((rc = vfr_build_con(tet.data(), nT, nV, con.data(), &numExt, 0)) != VFR_OK)
        return die("buildCon", rc);
      std::printf("Writing %s file\n", fn.c_str());
      vfr_write_con(fn.c_str(), con.data(), nT, numExt);
    }

    read_tf_file();

    fn = base + ".extf";
    std::printf("Reading %s file\n", fn.c_str());
    uint32_t ne = 0;
    have = vfr_read_extf(fn.c_str(), nullptr, &ne) == VFR_OK && ne == numExt;
    if (have) {
      extf.resize(2 * (size_t)ne);
      have = vfr_read_extf(fn.c_str(), extf.data(), &ne) == VFR_OK;
    }
    if (!have) {
      std::printf("%s file not found!\n Computing extFaces\n", fn.c_str());
      extf.resize(2 * (size_t)numExt);
      if ((rc = vfr_build_extf(con.data(), nT, extf.data(), numExt, &ne)) != VFR_OK)
        return die("buildExtF", rc);
      std::printf("Writing %s file\n", fn.c_str());
      vfr_write_extf(fn.c_str(), extf.data(), numExt);
    }

    fn = base + ".lmt";
    std::printf("Reading %s file\n", fn.c_str());
    if (vfr_read_lmt(fn.c_str(), lmt) != VFR_OK) {
      std::printf("%s file not found!\n Computing limits\n", fn.c_str());
      vfr_build_lmt(vert.data(), nV, tet.data(), nT, lmt);
      std::printf("Writing %s file\n", fn.c_str());
      vfr_write_lmt(fn.c_str(), lmt);
    }
    if (use_cache) {
      std::printf("Writing %s (binary cache)\n", cache.c_str());
      vfr_write_mesh_cache(cache.c_str(), vert.data(), nV, tet.data(), con.data(), nT, extf.data(),
                           numExt, lmt);
    }
  }

  if (from_cache) read_tf_file();

  std::printf("Volume dataset information: %s.off\n", base.c_str());
  std::printf("  # Tets: %u ; # Verts: %u\n", nT, nV);
  std::printf("  # ExtFaces: %u\n", numExt);
  std::printf("  Max Edge Length: %f\n", lmt[0]);
  std::printf("  Max Z: %f ; Min Z: %f\n", lmt[1], lmt[2]);

  std::vector<float> psi(512 * 512);
  if (psi_path == "generated") {
    vfr_psi_table(psi.data());
    std::printf("psi table: generated\n");
  } else if (!psi_path.empty()) {
    if ((rc = vfr_read_psi_source(psi_path.c_str(), psi.data())) != VFR_OK)
      return die(("reading psi table " + psi_path).c_str(), rc);
    std::printf("psi table: %s\n", psi_path.c_str());
  } else {
    if ((rc = vfr_psi_table_reference(psi.data())) != VFR_OK)
      return die("the reference psi table (data/psiGammaTable512.bin beside the library) is "
                 "missing; use --psi FILE or --psi generated",
                 rc);
    std::printf("psi table: the reference's (psiGammaTable512.h)\n");
  }

  // --- device (vfRay.cu:885-911) ---
  std::printf("***********************************\n");
  std::printf("Initializing CUDA\n");
  Timer tinit;
  vfr_ctx* ctx = nullptr;
  if ((rc = vfr_create(&ctx, device)) != VFR_OK) return die("vfr_create", rc);
  if ((rc = vfr_tables_upload(ctx, tf.data(), psi.data())) != VFR_OK)
    return die("vfr_tables_upload", rc, ctx);
  int mesh = -1;
  rc = vfr_mesh_upload(ctx, vert.data(), nV, tet.data(), con.data(), nT, extf.data(), numExt,
                       lmt[0], lmt[1], lmt[2], &mesh);
  if (rc != VFR_OK) return die("vfr_mesh_upload", rc, ctx);
  std::printf("** Prepare ** Processing time: %d (ms)\n", (int)tinit.ms());
  std::printf("***********************************\n");

  const size_t np = (size_t)W * H;
  std::vector<uint8_t> img(np * 3);
  std::vector<float> rgba(rgba_path.empty() ? 0 : np * 4);
  std::vector<uint32_t> steps(steps_path.empty() ? 0 : np);
  vfr_render_stats st;
  if (mode == VFR_MODE_REF) {
    std::printf("Execute kernel 1 on device\n");
    uint32_t nvis = 0;
    Timer t1;
    if ((rc = vfr_find_visible(ctx, mesh, &nvis, nullptr, nullptr)) != VFR_OK)
      return die("vfr_find_visible", rc, ctx);
    std::printf("Processing time: %.3f (ms)\n", t1.ms());
    std::printf(" # VisFaces: %u\n", nvis);
    std::printf("Execute kernel 2 on device\n");
    Timer t2;
    if ((rc = vfr_project(ctx, mesh, W, H, nullptr, nullptr)) != VFR_OK)
      return die("vfr_project", rc, ctx);
    std::printf("Processing time: %.3f (ms)\n", t2.ms());
    std::printf("Execute kernel 3 on device\n");
    Timer t3;
    rc = vfr_traverse(ctx, mesh, img.data(), rgba.empty() ? nullptr : rgba.data(),
                      steps.empty() ? nullptr : steps.data(), &st);
    if (rc != VFR_OK) return die("vfr_traverse", rc, ctx);
    std::printf("Processing time: %.3f (ms) [kernel %.3f ms, %u rays, %llu steps]\n", t3.ms(),
                st.ms_traverse, st.num_rays, (unsigned long long)st.num_steps);
  } else {
    Timer t;
    rc = vfr_render(ctx, mesh, nullptr, W, H, mode, img.data(),
                    rgba.empty() ? nullptr : rgba.data(), steps.empty() ? nullptr : steps.data(),
                    &st);
    if (rc != VFR_OK) return die("vfr_render", rc, ctx);
    std::printf("Render (composited): %.3f ms [device %.3f ms] # VisFaces: %u, %u rays, %u entries\n",
                t.ms(), st.ms_total, st.num_vis, st.num_rays, st.num_entries);
  }

  std::string img_path = out_path.empty() ? std::string(volume) + "_gpu_img.ppm" : out_path;
  std::printf("Saving ppm image: %s\n", img_path.c_str());
  if ((rc = vfr_write_ppm(img_path.c_str(), img.data(), W, H)) != VFR_OK) return die("ppmWrite", rc);
  if (!rgba_path.empty() && !write_raw(rgba_path, rgba.data(), rgba.size() * 4))
    return die("writing rgba", VFR_ERR_IO);
  if (!steps_path.empty() && !write_raw(steps_path, steps.data(), steps.size() * 4))
    return die("writing steps", VFR_ERR_IO);
  std::printf("Clean up device\n");
  vfr_destroy(ctx);
  return 0;
}
