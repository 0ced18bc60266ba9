// Instantiates the plain-form launchers for one array height, BRIDCT_H (set by the build;
// the file is compiled once per height so that the eight objects build in parallel).
#include "plain_launch.cuh"

#ifndef BRIDCT_H
#error "compile with -DBRIDCT_H=<8..1024>"
#endif

namespace bridct {

#define BRIDCT_ROW(W)                                                                       \
  {&launch_plain<BRIDCT_H, W, LM_FWD>, &launch_plain<BRIDCT_H, W, LM_INV>,                 \
   &launch_plain<BRIDCT_H, W, LM_RT>}

#define BRIDCT_CAT2(a, b) a##b
#define BRIDCT_CAT(a, b) BRIDCT_CAT2(a, b)

// Fills row[lg(w)][mode] for this height.
void BRIDCT_CAT(plain_table_h, BRIDCT_H)(PlainLauncher (*row)[3]) {
  static const PlainLauncher t[8][3] = {BRIDCT_ROW(8),   BRIDCT_ROW(16),  BRIDCT_ROW(32),
                                        BRIDCT_ROW(64),  BRIDCT_ROW(128), BRIDCT_ROW(256),
                                        BRIDCT_ROW(512), BRIDCT_ROW(1024)};
  for (int i = 0; i < 8; ++i)
    for (int m = 0; m < 3; ++m) row[i][m] = t[i][m];
}

}  // namespace bridct
