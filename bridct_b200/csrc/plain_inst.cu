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

// Fills row[lg(w)][mode] for this height, and the merged-pass launchers of column length
// BRIDCT_H (col[mode]) and row length BRIDCT_H (rowu[mode]).  Two-pass shapes have both axes of at
// least 32 points, so shorter lengths have none.
void BRIDCT_CAT(plain_table_h, BRIDCT_H)(PlainLauncher (*row)[3], UnitLauncher* col, UnitLauncher* rowu) {
  static const PlainLauncher t[8][3] = {BRIDCT_ROW(8),   BRIDCT_ROW(16),  BRIDCT_ROW(32),
                                        BRIDCT_ROW(64),  BRIDCT_ROW(128), BRIDCT_ROW(256),
                                        BRIDCT_ROW(512), BRIDCT_ROW(1024)};
  for (int i = 0; i < 8; ++i)
    for (int m = 0; m < 3; ++m) row[i][m] = t[i][m];
#if BRIDCT_H >= 32
  col[0] = &launch_col_units<BRIDCT_H, LM_FWD>;
  col[1] = &launch_col_units<BRIDCT_H, LM_INV>;
  col[2] = &launch_col_units<BRIDCT_H, LM_RT>;
  rowu[0] = &launch_row_units<BRIDCT_H, LM_FWD>;
  rowu[1] = &launch_row_units<BRIDCT_H, LM_INV>;
  rowu[2] = &launch_row_units<BRIDCT_H, LM_RT>;
#else
  for (int m = 0; m < 3; ++m) col[m] = rowu[m] = nullptr;
#endif
}

#if BRIDCT_H >= 32
int BRIDCT_CAT(merged_strip_cols_h, BRIDCT_H)() { return Geometry<BRIDCT_H, 1024>::kTC; }
int BRIDCT_CAT(merged_block_rows_w, BRIDCT_H)() {
  return Geometry<1024, BRIDCT_H>::kNarrowRows ? Geometry<1024, BRIDCT_H>::kRBn : Geometry<1024, BRIDCT_H>::kRB;
}
#else
int BRIDCT_CAT(merged_strip_cols_h, BRIDCT_H)() { return 0; }
int BRIDCT_CAT(merged_block_rows_w, BRIDCT_H)() { return 0; }
#endif

}  // namespace bridct
