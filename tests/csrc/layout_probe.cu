// Host-side dump of the tile-skewed layout helpers of cgli_launch.h (no GPU
// is used): the position of every 16-byte vector of a record slot for each
// slot index, and the update kernel's block count, for
// tests/test_layout.py.
#include <cstdio>

#include "cgli_launch.h"

int main() {
  for (int t = 0; t < 256; t++)
    for (int u = 0; u < 8; u++) printf("d %d %d %d\n", t, u, cgli::rec_vec_pos<double>(u, t));
  for (int t = 0; t < 256; t++)
    for (int u = 0; u < 4; u++) printf("f %d %d %d\n", t, u, cgli::rec_vec_pos<float>(u, t));
  printf("tile %d %d %d %d\n", cgli::SweepTile<double>::TI, cgli::SweepTile<double>::TJ, cgli::SweepTile<float>::TI,
         cgli::SweepTile<float>::TJ);
  printf("slot %d %d\n", cgli::CR_N, cgli::REC_N);
  return 0;
}
