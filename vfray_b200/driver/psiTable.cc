// psiTable: converts a psiGammaTable512.h-style C source (the reference's
// partial pre-integration table, "float psiGammaTable[512][512] = {...}")
// into the raw table file the library loads by default
// (vfr_psi_table_reference: 512 x 512 little-endian float32, [front][back]),
// and writes the source's leading comment -- the table's copyright notice,
// which its licence asks to be reproduced with every copy -- beside it.
//
//   psiTable <psiGammaTable512.h> <table.bin> <table.NOTICE>
#include <cstdio>
#include <string>
#include <vector>

#include "vfray.h"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "use: %s psiGammaTable512.h table.bin table.NOTICE\n", argv[0]);
    return 2;
  }
  std::vector<float> t(512 * 512);
  int rc = vfr_read_psi_source(argv[1], t.data());
  if (rc != VFR_OK) {
    std::fprintf(stderr, "psiTable: cannot read a 512x512 table from %s (%s)\n", argv[1],
                 vfr_status_string(rc));
    return 1;
  }
  // the notice: the source's first comment block
  std::string text;
  if (FILE* f = std::fopen(argv[1], "rb")) {
    char buf[4096];
    size_t n;
    while (text.size() < (1u << 16) && (n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    std::fclose(f);
  }
  const size_t a = text.find("/*"), b = text.find("*/");
  if (a == std::string::npos || b == std::string::npos || b < a) {
    std::fprintf(stderr, "psiTable: %s has no leading notice comment\n", argv[1]);
    return 1;
  }
  FILE* o = std::fopen(argv[2], "wb");
  FILE* n = std::fopen(argv[3], "wb");
  bool ok = o && n && std::fwrite(t.data(), sizeof(float), t.size(), o) == t.size();
  std::string src = argv[1];
  if (src.rfind('/') != std::string::npos) src = src.substr(src.rfind('/') + 1);
  const std::string notice = "The psi table in psiGammaTable512.bin is converted from " + src +
                             " of the VF-Ray sources, which carries this notice:\n\n" +
                             text.substr(a, b + 2 - a) + "\n";
  ok = ok && std::fwrite(notice.data(), 1, notice.size(), n) == notice.size();
  if (o) ok = (std::fclose(o) == 0) && ok;
  if (n) ok = (std::fclose(n) == 0) && ok;
  if (!ok) {
    std::fprintf(stderr, "psiTable: cannot write %s / %s\n", argv[2], argv[3]);
    return 1;
  }
  return 0;
}
