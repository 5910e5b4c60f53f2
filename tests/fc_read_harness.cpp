// Test support: runs the library's input reader (read_system) on a
// directory and prints the FC2 and FC3 term values as hex floats, one per
// line ("f2 <value>" / "f3 <value>"), and each term's index tuple.
#include <cstdio>

#include "../anharmonic-lattice-dynamics_b200/csrc/ald_internal.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  ald::System S;
  const std::string e = ald::read_system(argv[1], S);
  if (!e.empty()) {
    std::printf("ERR %s\n", e.c_str());
    return 1;
  }
  for (size_t j = 0; j < S.f2.size(); ++j)
    std::printf("f2 %a %d %d %d %d\n", S.f2[j], S.t2[4 * j], S.t2[4 * j + 1], S.t2[4 * j + 2], S.t2[4 * j + 3]);
  for (size_t j = 0; j < S.f3.size(); ++j)
    std::printf("f3 %a %d %d %d %d %d %d\n", S.f3[j], S.t3[6 * j], S.t3[6 * j + 1], S.t3[6 * j + 2],
                S.t3[6 * j + 3], S.t3[6 * j + 4], S.t3[6 * j + 5]);
  return 0;
}
