// cleanTF: converts a transfer function from the old layout (7 header
// lines, then 256 lines "index r g b a") to the .tf layout the renderer
// reads, as the reference's cleanTF.cc:13-88 does; same command line and
// messages, the conversion itself is vfr_clean_tf.
#include <cstdio>

#include "vfray.h"

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "use: %s old.off.tf new.tf\nWhere *.tf is the transfer function file.\n",
                 argv[0]);
    return 1;
  }
  std::printf("Reading %s . . . done!\nWriting %s", argv[1], argv[2]);
  const int rc = vfr_clean_tf(argv[1], argv[2]);
  if (rc != VFR_OK) {
    std::printf("\n%s: %s\n", argv[1], vfr_status_string(rc));
    return 1;
  }
  std::printf(" . . . done!\n");
  return 0;
}
