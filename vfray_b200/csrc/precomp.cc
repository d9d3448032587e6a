// Host-side precomputation and file formats of the VF-Ray render path.
//
// Restates vfRayPreComp.cc with the same float arithmetic where the numbers
// matter for the render (normalizeVertices :84-145, rotateVolume :886-906,
// buildLmt :808-853) and with a scalable algorithm where the reference is
// O(nV * nT) (buildIncid + buildCon :219-501): sorted face triples bucketed by
// their smallest vertex id give the same neighbour ids in O(nT log k).
// Readers and writers keep the reference's text layouts byte for byte.
#include <dlfcn.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vfray.h"

namespace {

int hw_threads(int threads) {
  if (threads > 0) return threads;
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// ---- psi(gamma) table --------------------------------------------------

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_n.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n); w.resize(n);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1; p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1);
      double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1 - z * z) * dp * dp);
  }
}

// psi(tf, tb) = int_0^1 exp(-(tf u + (tb - tf) u^2 / 2)) du: the
// transmittance-weighted mean over a segment whose extinction varies
// linearly from tf (front) to tb (back); with zeta = exp(-(tf+tb)/2) the
// segment colour is Cf (1 - psi) + Cb (psi - zeta), the partial
// pre-integration of Moreland & Angel (2004) that vfRayKernelCPU.cc:458-476
// evaluates.  Composite 20-point Gauss-Legendre, one panel per ~2 units of
// exponent slope, so every panel sees a smooth integrand.
double psi_exact(double tf, double tb, const std::vector<double>& x, const std::vector<double>& w) {
  double slope = std::max(tf, tb);
  int panels = std::min(1024, (int)std::ceil(slope / 2.0) + 1);
  double h = 1.0 / panels, sum = 0;
  double b = 0.5 * (tb - tf);
  for (int p = 0; p < panels; ++p) {
    double a0 = p * h;
    for (size_t k = 0; k < x.size(); ++k) {
      double u = a0 + 0.5 * h * (x[k] + 1.0);
      sum += 0.5 * h * w[k] * std::exp(-(tf * u + b * u * u));
    }
  }
  return sum;
}

std::once_flag g_psi_once;
std::vector<float> g_psi;

void build_psi() {
  g_psi.assign(512 * 512, 0.f);
  std::vector<double> x, w;
  gauss_legendre(20, x, w);
  auto rows = [&](size_t lo, size_t hi) {
    char buf[64];
    for (size_t i = lo; i < hi; ++i) {
      double gf = i / 512.0, tf = gf / (1.0 - gf);
      for (int j = 0; j < 512; ++j) {
        double gb = j / 512.0, tb = gb / (1.0 - gb);
        double v = psi_exact(tf, tb, x, w);
        // 7 decimals, truncated, then parsed as a float literal would be;
        // a value within 1e-15 below a 7-decimal step is taken as that step
        // (psi(0,0) = 1 exactly; the quadrature's own error is ~1e-16)
        long long k = (long long)std::floor(v * 1e7 + 1e-8);
        std::snprintf(buf, sizeof buf, "%lld.%07lld", k / 10000000, k % 10000000);
        g_psi[i * 512 + j] = std::strtof(buf, nullptr);
      }
    }
  };
  std::vector<std::thread> pool;
  int T = hw_threads(0);
  for (int t = 0; t < T; ++t) {
    size_t lo = 512 * t / T, hi = 512 * (t + 1) / T;
    pool.emplace_back(rows, lo, hi);
  }
  for (auto& th : pool) th.join();
}

// ---- text parsing -------------------------------------------------------

struct TextFile {
  std::string data;
  size_t pos = 0;
  bool ok = false;
  explicit TextFile(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return;
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) { std::fclose(f); return; }
    data.resize((size_t)n);
    ok = std::fread(&data[0], 1, (size_t)n, f) == (size_t)n;
    std::fclose(f);
    data.push_back('\0');
  }
  void skip_ws() {
    while (pos < data.size() && (data[pos] == ' ' || data[pos] == '\n' || data[pos] == '\t' ||
                                 data[pos] == '\r'))
      ++pos;
  }
  bool next_u32(uint32_t& v) {
    skip_ws();
    const char* s = data.c_str() + pos;
    char* e;
    errno = 0;
    unsigned long long x = std::strtoull(s, &e, 10);
    if (e == s || errno) return false;
    pos += (size_t)(e - s);
    v = (uint32_t)x;
    return true;
  }
  bool next_f32(float& v) {
    skip_ws();
    const char* s = data.c_str() + pos;
    char* e;
    v = std::strtof(s, &e);
    if (e == s) return false;
    pos += (size_t)(e - s);
    return true;
  }
};

// Whitespace-separated tokens after the .off header: the first nf are
// floats (strtof, as the reference's operator>> reads them), the next nu
// unsigned integers; anything after them is ignored, as a sequential read
// would.  Large files are cut into chunks at whitespace; a first pass counts
// each chunk's tokens, a second parses them into place, one thread per chunk.
bool parse_u32_token(const char* s, const char* e, uint32_t& out) {
  if (s == e) return false;
  unsigned long long x = 0;
  for (const char* c = s; c < e; ++c) {
    if (*c < '0' || *c > '9') return false;
    x = x * 10 + (unsigned)(*c - '0');
    if (x > 0xffffffffull) return false;
  }
  out = (uint32_t)x;
  return true;
}

inline bool is_ws(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r'; }

bool parse_tokens(const char* buf, size_t len, float* fo, size_t nf, uint32_t* uo, size_t nu) {
  const size_t want = nf + nu;
  const int T = (len < (64u << 20)) ? 1 : std::min(hw_threads(0), 32);
  std::vector<size_t> cut(T + 1, len);
  cut[0] = 0;
  for (int t = 1; t < T; ++t) {
    size_t c = std::max(cut[t - 1], len * (size_t)t / (size_t)T);
    while (c < len && !is_ws(buf[c])) ++c;
    cut[t] = c;
  }
  std::vector<size_t> count(T, 0);
  auto count_chunk = [&](int t) {
    size_t n = 0;
    bool in = false;
    for (size_t i = cut[t]; i < cut[t + 1]; ++i) {
      const bool w = is_ws(buf[i]);
      if (!w && !in) ++n;
      in = !w;
    }
    count[t] = n;
  };
  std::vector<char> bad(T, 0);
  std::vector<size_t> first(T + 1, 0);
  auto parse_chunk = [&](int t) {
    size_t k = first[t];
    size_t i = cut[t];
    char tmp[64];
    while (i < cut[t + 1] && k < want) {
      while (i < cut[t + 1] && is_ws(buf[i])) ++i;
      if (i >= cut[t + 1]) break;
      size_t j = i;
      while (j < cut[t + 1] && !is_ws(buf[j])) ++j;
      if (k < nf) {
        const size_t n = std::min<size_t>(j - i, sizeof tmp - 1);
        std::memcpy(tmp, buf + i, n);
        tmp[n] = '\0';
        char* e;
        fo[k] = std::strtof(tmp, &e);
        if (e == tmp) { bad[t] = 1; return; }
      } else if (!parse_u32_token(buf + i, buf + j, uo[k - nf])) {
        bad[t] = 1;
        return;
      }
      ++k;
      i = j;
    }
  };
  auto run = [&](auto&& fn) {
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(fn, t);
    fn(0);
    for (auto& x : th) x.join();
  };
  run(count_chunk);
  for (int t = 0; t < T; ++t) first[t + 1] = first[t] + count[t];
  if (first[T] < want) return false;
  run(parse_chunk);
  for (int t = 0; t < T; ++t)
    if (bad[t]) return false;
  return true;
}

// Binary mesh cache: this header, then vert4 (16 B each), tet4, con4 (16 B
// each) and extf2 (8 B each), native byte order.
constexpr char kCacheMagic[8] = {'V', 'F', 'R', 'M', 'E', 'S', 'H', '1'};
struct CacheHeader {
  char magic[8];
  uint32_t nV = 0, nT = 0, nExt = 0;
  float lmt[3] = {0, 0, 0};
  uint32_t reserved[2] = {0, 0};
};
static_assert(sizeof(CacheHeader) == 40, "cache header layout");

int write_text(const char* path, const std::string& s) {
  FILE* f = std::fopen(path, "w");
  if (!f) return VFR_ERR_IO;
  bool ok = std::fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? VFR_OK : VFR_ERR_IO;
}

// ostream's default formatting of a float (precision 6, %g), which the
// reference writers use (vfRayPreComp.cc:521,638,863).
void put_g(std::string& s, float v) {
  char buf[48];
  std::snprintf(buf, sizeof buf, "%g", (double)v);
  s += buf;
}

void put_u(std::string& s, uint32_t v) {
  char buf[16];
  std::snprintf(buf, sizeof buf, "%u", v);
  s += buf;
}

}  // namespace

extern "C" {

int vfr_psi_table(float* out) {
  if (!out) return VFR_ERR_INVALID;
  std::call_once(g_psi_once, build_psi);
  std::memcpy(out, g_psi.data(), sizeof(float) * 512 * 512);
  return VFR_OK;
}

int vfr_normalize(float* v, uint32_t nV) {
  if (!v || nV == 0) return VFR_ERR_INVALID;
  float mn[4], mx[4], center[3];
  for (int i = 0; i < 4; ++i) mn[i] = mx[i] = v[i];
  for (uint32_t i = 1; i < nV; ++i)
    for (int j = 0; j < 4; ++j) {
      float value = v[4 * (size_t)i + j];
      if (value < mn[j]) mn[j] = value;
      if (value > mx[j]) mx[j] = value;
    }
  for (int i = 0; i < 3; ++i) {
    center[i] = (float)((double)(mn[i] + mx[i]) / 2.0);
    mx[i] -= center[i];
    mn[i] -= center[i];
  }
  float maxCoord = (mx[1] > mx[2]) ? mx[1] : mx[2];
  maxCoord = (mx[0] > maxCoord) ? mx[0] : maxCoord;
  float scaleCoord = (float)(1.0 / (double)maxCoord);
  float scaleScalar = (float)(1.0 / (double)(mx[3] - mn[3]));
  for (uint32_t i = 0; i < nV; ++i) {
    float* p = v + 4 * (size_t)i;
    for (int j = 0; j < 3; ++j) p[j] = (p[j] - center[j]) * scaleCoord;
    p[3] = (p[3] - mn[3]) * scaleScalar;
  }
  return VFR_OK;
}

int vfr_rotate(float* v, uint32_t nV, const float* m) {
  if (!v || !m) return VFR_ERR_INVALID;
  for (uint32_t i = 0; i < nV; ++i) {
    float* p = v + 4 * (size_t)i;
    const float o[4] = {p[0], p[1], p[2], 1.0f};
    float r[4] = {0.f, 0.f, 0.f, 0.f};
    for (int a = 0; a < 4; ++a)
      for (int c = 0; c < 4; ++c) r[a] += m[a * 4 + c] * o[c];
    for (int j = 0; j < 3; ++j) p[j] = r[j];
  }
  return VFR_OK;
}

int vfr_build_con(const uint32_t* tet, uint32_t nT, uint32_t nV, uint32_t* con,
                  uint32_t* num_ext, int threads) {
  if (!tet || !con || nV == 0) return VFR_ERR_INVALID;
  threads = hw_threads(threads);
  for (size_t i = 0; i < (size_t)nT; ++i) {
    const uint32_t* t = tet + 4 * i;
    for (int k = 0; k < 4; ++k) {
      if (t[k] >= nV) return VFR_ERR_MESH;
      for (int l = k + 1; l < 4; ++l)
        if (t[k] == t[l]) return VFR_ERR_MESH;  // a degenerate tet has no well-defined faces
    }
  }
  const size_t nf = 4 * (size_t)nT;
  // Bucket every face (i, f) by the smallest id of its vertex triple
  // (the vertices (f+k)&3, k=0..2 as MOD4(k, f) at vfRayPreComp.cc:444).
  std::vector<uint32_t> start((size_t)nV + 1, 0);
  auto sorted3 = [&](size_t face, uint32_t& a, uint32_t& b, uint32_t& c) {
    const uint32_t* t = tet + 4 * (face >> 2);
    uint32_t f = (uint32_t)(face & 3);
    a = t[(f + 0) & 3]; b = t[(f + 1) & 3]; c = t[(f + 2) & 3];
    if (a > b) std::swap(a, b);
    if (b > c) std::swap(b, c);
    if (a > b) std::swap(a, b);
  };
  for (size_t face = 0; face < nf; ++face) {
    uint32_t a, b, c;
    sorted3(face, a, b, c);
    start[a + 1]++;
  }
  for (size_t v = 0; v < nV; ++v) start[v + 1] += start[v];
  struct Item { uint64_t bc; uint32_t face; };
  std::vector<Item> items(nf);
  {
    std::vector<uint32_t> cur(start.begin(), start.end() - 1);
    for (size_t face = 0; face < nf; ++face) {
      uint32_t a, b, c;
      sorted3(face, a, b, c);
      items[cur[a]++] = Item{((uint64_t)b << 32) | c, (uint32_t)face};
    }
  }
  std::vector<uint64_t> ext_count((size_t)threads, 0);
  // Buckets are independent: the neighbour across face (i, f) is the
  // smallest tet id other than i among the faces with the same triple,
  // which is the tet the reference's incidence search meets first
  // (vfRayPreComp.cc:450-490 scans ascending tet ids).
  auto work = [&](size_t lo, size_t hi, int slot) {
    uint64_t ext = 0;
    for (size_t a = lo; a < hi; ++a) {
      Item* b0 = items.data() + start[a];
      Item* b1 = items.data() + start[a + 1];
      std::sort(b0, b1, [](const Item& x, const Item& y) {
        return x.bc != y.bc ? x.bc < y.bc : x.face < y.face;
      });
      for (Item* g = b0; g < b1;) {
        Item* e = g;
        while (e < b1 && e->bc == g->bc) ++e;
        for (Item* it = g; it < e; ++it) {
          uint32_t self = it->face >> 2, nb = self;
          for (Item* o = g; o < e; ++o) {
            uint32_t ot = o->face >> 2;
            if (ot != self) { nb = ot; break; }  // group is sorted by face, so by tet
          }
          con[it->face] = nb;
          if (nb == self) ++ext;
        }
        g = e;
      }
    }
    ext_count[slot] = ext;
  };
  {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
      size_t lo = (size_t)nV * t / threads, hi = (size_t)nV * (t + 1) / threads;
      pool.emplace_back(work, lo, hi, t);
    }
    for (auto& th : pool) th.join();
  }
  uint64_t ext = 0;
  for (auto c : ext_count) ext += c;
  if (num_ext) *num_ext = (uint32_t)ext;
  return VFR_OK;
}

int vfr_build_extf(const uint32_t* con, uint32_t nT, uint32_t* extf, uint32_t cap,
                   uint32_t* num_ext) {
  if (!con) return VFR_ERR_INVALID;
  uint32_t n = 0;
  for (uint32_t i = 0; i < nT; ++i)
    for (uint32_t f = 0; f < 4; ++f) {
      if (con[4 * (size_t)i + f] != i) continue;
      if (extf) {
        if (n >= cap) return VFR_ERR_INVALID;
        extf[2 * (size_t)n] = i;
        extf[2 * (size_t)n + 1] = f;
      }
      ++n;
    }
  if (num_ext) *num_ext = n;
  return VFR_OK;
}

int vfr_build_lmt(const float* v, uint32_t nV, const uint32_t* tet, uint32_t nT, float* out) {
  if (!v || !tet || !out) return VFR_ERR_INVALID;
  float maxEdge = 0.0f;
  static const int E[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  for (size_t i = 0; i < (size_t)nT; ++i) {
    const uint32_t* t = tet + 4 * i;
    for (int k = 0; k < 4; ++k)
      if (t[k] >= nV) return VFR_ERR_MESH;
    for (int j = 0; j < 6; ++j) {
      const float* a = v + 4 * (size_t)t[E[j][0]];
      const float* b = v + 4 * (size_t)t[E[j][1]];
      float e0 = a[0] - b[0], e1 = a[1] - b[1], e2 = a[2] - b[2];
      float len = std::sqrt(e0 * e0 + e1 * e1 + e2 * e2);
      if (len > maxEdge) maxEdge = len;
    }
  }
  float maxZ = -1.0f, minZ = 1.0f;
  for (size_t i = 0; i < (size_t)nV; ++i) {
    float z = v[4 * i + 2];
    if (z > maxZ) maxZ = z;
    if (z < minZ) minZ = z;
  }
  out[0] = maxEdge; out[1] = maxZ; out[2] = minZ;
  return VFR_OK;
}

int vfr_default_tf(float* tf) {
  if (!tf) return VFR_ERR_INVALID;
  for (int i = 0; i < 256; ++i) {
    float c[4];
    if (i < 64) { c[0] = 1; c[1] = 0; c[2] = 0; }
    else if (i < 128) { c[0] = 1; c[1] = 1; c[2] = 0; }
    else if (i < 192) { c[0] = 0; c[1] = 1; c[2] = 1; }
    else { c[0] = 0; c[1] = 0; c[2] = 1; }
    c[3] = 0.2f;
    std::memcpy(tf + 4 * i, c, sizeof c);
  }
  return VFR_OK;
}

// ---- readers ----

int vfr_read_off(const char* path, float* v, uint32_t* nV, uint32_t* tet, uint32_t* nT) {
  if (!path || !nV || !nT) return VFR_ERR_INVALID;
  if (!v || !tet) {  // sizes only: the header line is enough
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return VFR_ERR_IO;
    unsigned long long a = 0, b = 0;
    const int got = std::fscanf(fp, "%llu %llu", &a, &b);
    std::fclose(fp);
    if (got != 2 || a > 0xffffffffull || b > 0xffffffffull) return VFR_ERR_IO;
    *nV = (uint32_t)a;
    *nT = (uint32_t)b;
    return VFR_OK;
  }
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  uint32_t a, b;
  if (!f.next_u32(a) || !f.next_u32(b)) return VFR_ERR_IO;
  if (*nV < a || *nT < b) return VFR_ERR_INVALID;
  if (!parse_tokens(f.data.c_str() + f.pos, f.data.size() - 1 - f.pos, v, 4 * (size_t)a, tet,
                    4 * (size_t)b))
    return VFR_ERR_IO;
  *nV = a; *nT = b;
  return VFR_OK;
}

int vfr_write_mesh_cache(const char* path, const float* vert4, uint32_t nV, const uint32_t* tet4,
                         const uint32_t* con4, uint32_t nT, const uint32_t* extf2, uint32_t nExt,
                         const float* lmt3) {
  if (!path || !vert4 || !tet4 || !con4 || (!extf2 && nExt) || !lmt3) return VFR_ERR_INVALID;
  CacheHeader h;
  std::memcpy(h.magic, kCacheMagic, 8);
  h.nV = nV; h.nT = nT; h.nExt = nExt;
  std::memcpy(h.lmt, lmt3, sizeof h.lmt);
  FILE* f = std::fopen(path, "wb");
  if (!f) return VFR_ERR_IO;
  bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
            std::fwrite(vert4, 16, nV, f) == nV && std::fwrite(tet4, 16, nT, f) == nT &&
            std::fwrite(con4, 16, nT, f) == nT && std::fwrite(extf2, 8, nExt, f) == nExt;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? VFR_OK : VFR_ERR_IO;
}

int vfr_read_mesh_cache(const char* path, float* vert4, uint32_t* nV, uint32_t* tet4,
                        uint32_t* con4, uint32_t* nT, uint32_t* extf2, uint32_t* nExt,
                        float* lmt3) {
  if (!path || !nV || !nT || !nExt) return VFR_ERR_INVALID;
  FILE* f = std::fopen(path, "rb");
  if (!f) return VFR_ERR_IO;
  CacheHeader h;
  bool ok = std::fread(&h, sizeof h, 1, f) == 1 && std::memcmp(h.magic, kCacheMagic, 8) == 0;
  if (ok) {  // the file must hold exactly the arrays its header names
    std::fseek(f, 0, SEEK_END);
    const long long len = std::ftell(f);
    ok = len == (long long)(sizeof h + 16ull * h.nV + 32ull * h.nT + 8ull * h.nExt);
    std::fseek(f, (long)sizeof h, SEEK_SET);
  }
  if (!ok) { std::fclose(f); return VFR_ERR_IO; }
  if (!vert4 || !tet4 || !con4 || !lmt3 || (!extf2 && h.nExt)) {
    std::fclose(f);
    *nV = h.nV; *nT = h.nT; *nExt = h.nExt;
    return VFR_OK;
  }
  if (*nV < h.nV || *nT < h.nT || *nExt < h.nExt) { std::fclose(f); return VFR_ERR_INVALID; }
  ok = std::fread(vert4, 16, h.nV, f) == h.nV && std::fread(tet4, 16, h.nT, f) == h.nT &&
       std::fread(con4, 16, h.nT, f) == h.nT && std::fread(extf2, 8, h.nExt, f) == h.nExt;
  std::fclose(f);
  if (!ok) return VFR_ERR_IO;
  std::memcpy(lmt3, h.lmt, sizeof h.lmt);
  *nV = h.nV; *nT = h.nT; *nExt = h.nExt;
  return VFR_OK;
}

int vfr_read_con(const char* path, uint32_t* con, uint32_t* nT, uint32_t* num_ext) {
  if (!path || !nT || !num_ext) return VFR_ERR_INVALID;
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  uint32_t ne, nt;
  if (!f.next_u32(ne) || !f.next_u32(nt)) return VFR_ERR_IO;
  if (!con) { *nT = nt; *num_ext = ne; return VFR_OK; }
  if (*nT < nt) return VFR_ERR_INVALID;
  for (size_t i = 0; i < 4 * (size_t)nt; ++i)
    if (!f.next_u32(con[i])) return VFR_ERR_IO;
  *nT = nt; *num_ext = ne;
  return VFR_OK;
}

int vfr_read_extf(const char* path, uint32_t* extf, uint32_t* num_ext) {
  if (!path || !num_ext) return VFR_ERR_INVALID;
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  uint32_t n;
  if (!f.next_u32(n)) return VFR_ERR_IO;
  if (!extf) { *num_ext = n; return VFR_OK; }
  if (*num_ext < n) return VFR_ERR_INVALID;
  for (size_t i = 0; i < 2 * (size_t)n; ++i)
    if (!f.next_u32(extf[i])) return VFR_ERR_IO;
  *num_ext = n;
  return VFR_OK;
}

int vfr_read_lmt(const char* path, float* out) {
  if (!path || !out) return VFR_ERR_INVALID;
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  for (int i = 0; i < 3; ++i)
    if (!f.next_f32(out[i])) return VFR_ERR_IO;
  return VFR_OK;
}

int vfr_read_tf(const char* path, float* tf) {
  if (!path || !tf) return VFR_ERR_INVALID;
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  uint32_t n;
  if (!f.next_u32(n) || n != 256) return VFR_ERR_IO;
  for (int i = 0; i < 1024; ++i)
    if (!f.next_f32(tf[i])) return VFR_ERR_IO;
  return VFR_OK;
}

int vfr_read_psi_source(const char* path, float* out) {
  if (!path || !out) return VFR_ERR_INVALID;
  TextFile f(path);
  if (!f.ok) return VFR_ERR_IO;
  // the initializer: the first '=' followed (after blanks) by '{'
  size_t p = 0;
  for (;;) {
    p = f.data.find('=', p);
    if (p == std::string::npos) return VFR_ERR_IO;
    size_t q = p + 1;
    while (q < f.data.size() && std::strchr(" \t\r\n", f.data[q])) ++q;
    if (q < f.data.size() && f.data[q] == '{') { p = q; break; }
    p = q;
  }
  size_t n = 0;
  const char* s = f.data.c_str();
  while (n < 512 * 512 && s[p]) {
    char c = s[p];
    if (c == '{' || c == '}' || c == ',' || c == ' ' || c == '\n' || c == '\t' || c == '\r') {
      ++p;
      continue;
    }
    if (c == ';') break;
    char* e;
    float v = std::strtof(s + p, &e);
    if (e == s + p) return VFR_ERR_IO;
    if (*e == 'f' || *e == 'F') ++e;
    out[n++] = v;
    p = (size_t)(e - s);
  }
  return n == 512 * 512 ? VFR_OK : VFR_ERR_IO;
}

// The reference's own psi table as this library ships it: 512 x 512 raw
// little-endian float32, [front][back], converted from psiGammaTable512.h by
// bin/psiTable at build time and kept beside the library with the table's
// copyright notice.  $VFRAY_PSI_TABLE names another such file.
int vfr_psi_table_reference(float* out) {
  if (!out) return VFR_ERR_INVALID;
  std::string path;
  if (const char* env = std::getenv("VFRAY_PSI_TABLE")) {
    path = env;
  } else {
    Dl_info info;
    if (!dladdr((void*)&vfr_psi_table_reference, &info) || !info.dli_fname) return VFR_ERR_IO;
    path = info.dli_fname;
    const size_t slash = path.rfind('/');
    path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) +
           "/data/psiGammaTable512.bin";
  }
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return VFR_ERR_IO;
  const size_t n = std::fread(out, sizeof(float), 512 * 512, f);
  const bool more = std::fgetc(f) != EOF;
  std::fclose(f);
  return (n == 512 * 512 && !more) ? VFR_OK : VFR_ERR_IO;
}

// ---- writers ----

int vfr_write_off(const char* path, const float* v, uint32_t nV, const uint32_t* tet, uint32_t nT) {
  if (!path || (!v && nV) || (!tet && nT)) return VFR_ERR_INVALID;
  std::string s;
  s.reserve((size_t)nV * 56 + (size_t)nT * 32 + 32);
  put_u(s, nV); s += ' '; put_u(s, nT); s += '\n';
  char buf[128];
  for (size_t i = 0; i < nV; ++i) {
    const float* p = v + 4 * i;
    std::snprintf(buf, sizeof buf, "%.9g %.9g %.9g %.9g\n", p[0], p[1], p[2], p[3]);
    s += buf;
  }
  for (size_t i = 0; i < nT; ++i) {
    const uint32_t* t = tet + 4 * i;
    std::snprintf(buf, sizeof buf, "%u %u %u %u\n", t[0], t[1], t[2], t[3]);
    s += buf;
  }
  return write_text(path, s);
}

int vfr_write_con(const char* path, const uint32_t* con, uint32_t nT, uint32_t num_ext) {
  if (!path || (!con && nT)) return VFR_ERR_INVALID;
  std::string s;
  s.reserve((size_t)nT * 40 + 32);
  put_u(s, num_ext); s += '\n'; put_u(s, nT); s += '\n';
  for (size_t i = 0; i < nT; ++i) {
    for (int k = 0; k < 4; ++k) {
      put_u(s, con[4 * i + k]);
      s += (k < 3) ? ' ' : '\n';
    }
  }
  return write_text(path, s);
}

int vfr_write_extf(const char* path, const uint32_t* extf, uint32_t n) {
  if (!path || (!extf && n)) return VFR_ERR_INVALID;
  std::string s;
  s.reserve((size_t)n * 16 + 16);
  put_u(s, n); s += '\n';
  for (size_t i = 0; i < n; ++i) {
    put_u(s, extf[2 * i]); s += ' '; put_u(s, extf[2 * i + 1]); s += '\n';
  }
  return write_text(path, s);
}

int vfr_write_lmt(const char* path, const float* in) {
  if (!path || !in) return VFR_ERR_INVALID;
  std::string s;
  put_g(s, in[0]); s += ' '; put_g(s, in[1]); s += ' '; put_g(s, in[2]); s += '\n';
  return write_text(path, s);
}

int vfr_write_tf(const char* path, const float* tf) {
  if (!path || !tf) return VFR_ERR_INVALID;
  std::string s = "256\n";
  for (int i = 0; i < 256; ++i)
    for (int k = 0; k < 4; ++k) {
      put_g(s, tf[4 * i + k]);
      s += (k < 3) ? ' ' : '\n';
    }
  return write_text(path, s);
}

int vfr_clean_tf(const char* in_path, const char* out_path) {
  if (!in_path || !out_path) return VFR_ERR_INVALID;
  // the old layout (cleanTF.cc:31-56): 7 header lines, then 256 lines of
  // "index r g b a", read as doubles
  FILE* f = std::fopen(in_path, "r");
  if (!f) return VFR_ERR_IO;
  int lines = 0, c;
  while (lines < 7 && (c = std::fgetc(f)) != EOF)
    if (c == '\n') ++lines;
  double tf[256][4];
  bool ok = lines == 7;
  for (int i = 0; ok && i < 256; ++i) {
    long idx;
    ok = std::fscanf(f, "%ld %lf %lf %lf %lf", &idx, &tf[i][0], &tf[i][1], &tf[i][2], &tf[i][3]) == 5;
  }
  std::fclose(f);
  if (!ok) return VFR_ERR_IO;
  // the .tf layout with ostream's default double formatting (cleanTF.cc:70-80)
  std::string s = "256\n";
  char buf[48];
  for (int i = 0; i < 256; ++i)
    for (int k = 0; k < 4; ++k) {
      std::snprintf(buf, sizeof buf, "%g", tf[i][k]);
      s += buf;
      s += (k < 3) ? ' ' : '\n';
    }
  return write_text(out_path, s);
}

int vfr_write_ppm(const char* path, const uint8_t* rgb, uint32_t W, uint32_t H) {
  if (!path || !rgb) return VFR_ERR_INVALID;
  FILE* f = std::fopen(path, "w");
  if (!f) return VFR_ERR_IO;
  std::fprintf(f, "P6\n%u %u\n255\n", W, H);
  size_t n = (size_t)W * H * 3;
  bool ok = std::fwrite(rgb, 1, n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? VFR_OK : VFR_ERR_IO;
}

}  // extern "C"
