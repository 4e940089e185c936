// Host harness for tests/test_datum_halo.py: the rows kernel's list of halo
// cells in another datum block (csrc/hb_datum_halo.cuh), compiled for the
// CPU, against the definition on every tile position of a raster of blocks.
#include "hb_datum_halo.cuh"

// Number of disagreements over tiles of TY x TW in nby x nbx blocks of
// block x block cells (SW staged columns per row): a listed cell twice, a
// listed cell outside the staged halo or inside the tile's block, or a halo
// cell outside the block that is not listed.
extern "C" int datum_halo_mismatches(int TY, int TW, int SW, int block, int nby, int nbx,
                                     int *listed_max) {
  int bad = 0;
  *listed_max = 0;
  static unsigned char seen[512 * 64];
  const int H = TY + 4, W = TW + 8;
  if (H * W > (int)sizeof(seen)) return -1;
  for (int y0 = 0; y0 < nby * block; y0 += TY) {
    for (int x0 = 0; x0 < nbx * block; x0 += TW) {
      const int by0 = y0 / block * block, bx0 = x0 / block * block;
      for (int q = 0; q < H * W; q++) seen[q] = 0;
      const hb::DatumHalo d = hb::datum_halo(y0, x0, by0, bx0, TY, TW, SW, block);
      if (d.count() > *listed_max) *listed_max = d.count();
      for (int k = 0; k < d.count(); k++) {
        int i, j;
        hb::datum_halo_cell(d, k, TY, TW, SW, i, j);
        if (i < -2 || i >= TY + 2 || j < -4 || j >= TW + 4) {
          bad++;
          continue;
        }
        const int ry = y0 + i, rx = x0 + j;
        const bool out = ry < by0 || ry >= by0 + block || rx < bx0 || rx >= bx0 + block;
        if (!out || seen[(i + 2) * W + (j + 4)]++) bad++;
      }
      for (int i = -2; i < TY + 2; i++)
        for (int j = -4; j < TW + 4; j++) {
          const int ry = y0 + i, rx = x0 + j;
          const bool out = ry < by0 || ry >= by0 + block || rx < bx0 || rx >= bx0 + block;
          if (out && !seen[(i + 2) * W + (j + 4)]) bad++;
        }
    }
  }
  return bad;
}
