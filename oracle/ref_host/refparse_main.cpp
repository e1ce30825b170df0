/*
 * Oracle A, project-input side, as a separate process: the reference's own
 * parser (V_02_2015/src/Input/KSimulationData.cpp, compiled unmodified) run
 * on one project, its results written as raw struct images.  TEST
 * INFRASTRUCTURE ONLY.
 *
 *   refparse <run_dir> <project> <world> <out.bin>
 *
 * out.bin = RefProject, WOBJ[8], POBJ[8], DOBJ[32] (the layouts of
 * refhost_parse.cpp and KSimulationObjects.h).
 *
 * Why a separate, sanitizer-built process: ReadPObject_Poly reads each
 * face's comma separator into `char delim[1]` (KSimulationData.cpp:1344,
 * 1369), which stores the comma and a terminating NUL, one byte past the
 * array.  Built with -O2 that byte breaks the parser (it crashes); built with
 * AddressSanitizer the frame has redzones around the array, so the stray
 * byte lands in padding and the parser computes what its source states.
 */
#include <cstdio>
#include <vector_types.h>

#include "DataStructures/KSimulationObjects.h"

extern "C" int refh_project_sizeof(void);
extern "C" int refh_parse(const char* run_dir, const char* project, const char* world, void* out,
                          WOBJ* w_out, int w_cap, POBJ* p_out, int p_cap, DOBJ* d_out, int d_cap);

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: refparse <run_dir> <project> <world> <out.bin>\n");
    return 2;
  }
  static unsigned char rp[1 << 16];
  static WOBJ w[8];
  static POBJ p[8];
  static DOBJ d[32];
  if (refh_project_sizeof() > (int)sizeof(rp)) return 3;
  const int rc = refh_parse(argv[1], argv[2], argv[3], rp, w, 8, p, 8, d, 32);
  if (rc) {
    std::fprintf(stderr, "refh_parse failed: %d\n", rc);
    return 4;
  }
  std::FILE* f = std::fopen(argv[4], "wb");
  if (!f) return 5;
  std::fwrite(rp, 1, (size_t)refh_project_sizeof(), f);
  std::fwrite(w, sizeof(WOBJ), 8, f);
  std::fwrite(p, sizeof(POBJ), 8, f);
  std::fwrite(d, sizeof(DOBJ), 32, f);
  std::fclose(f);
  return 0;
}
