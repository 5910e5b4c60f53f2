// Test support: evaluates the device tetrahedron weights (ald_tet.h) on the
// host.  Reads lines "w1 w2 w3 w4 e" and prints the four corner weights.
#include <cstdio>

#include "../anharmonic-lattice-dynamics_b200/csrc/ald_tet.h"

int main() {
  double w[4], e;
  while (std::scanf("%lf %lf %lf %lf %lf", &w[0], &w[1], &w[2], &w[3], &e) == 5) {
    float en[4] = {(float)w[0], (float)w[1], (float)w[2], (float)w[3]};
    ald::TetSorted ts = ald::tet_sort(en[0], en[1], en[2], en[3]);
    for (int k = 0; k < 4; ++k) std::printf("%.17g ", ald::tet_weight(ts, ald::tet_pos(en, k), e));
    // the four-at-once form used by the delta kernel
    double cp[4] = {0, 0, 0, 0};
    if (!ald::tet_weights4(ts, e, cp)) cp[0] = cp[1] = cp[2] = cp[3] = 0.0;
    for (int k = 0; k < 4; ++k) std::printf("%.17g ", cp[ald::tet_pos(en, k)]);
    std::printf("\n");
  }
  return 0;
}
