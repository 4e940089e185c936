// hb_datum_halo.cuh -- the staged halo cells of a rows-kernel tile that lie in
// another datum block, whose bed the tile moves into its own datum after the
// tile loads.  __host__ __device__ so that a CPU test can check every tile
// position against the definition (a halo cell outside the tile's block).
#pragma once

#ifndef HB_HD
#ifdef __CUDACC__
#define HB_HD __host__ __device__ __forceinline__
#else
#define HB_HD inline
#endif
#endif

namespace hb {

// A TY x TW tile (inside one block of `block` x `block` cells) stages rows
// -2 .. TY+1 and columns -4 .. TW+3 (SW columns per row).  The halo sides in
// another block: the two rows above (tile at its block's top) and the two
// below (tile at its block's bottom), full width, then the four columns left
// (tile at its block's left edge) and right (right edge) over the rows that
// the row sides leave out.
struct DatumHalo {
  int nT, nB, rlo, nL, nR;
  HB_HD int count() const { return nT + nB + nL + nR; }
};

HB_HD DatumHalo datum_halo(int y0, int x0, int by0, int bx0, int TY, int TW, int SW,
                           int block) {
  DatumHalo d;
  d.nT = y0 == by0 ? 2 * SW : 0;
  d.nB = y0 + TY == by0 + block ? 2 * SW : 0;
  d.rlo = d.nT ? 0 : -2;
  const int rn = (d.nB ? TY : TY + 2) - d.rlo;
  d.nL = x0 == bx0 ? 4 * rn : 0;
  d.nR = x0 + TW == bx0 + block ? 4 * rn : 0;
  return d;
}

// Tile-relative row i and column j of the k-th of those cells, 0 <= k < count().
HB_HD void datum_halo_cell(const DatumHalo &d, int k, int TY, int TW, int SW, int &i, int &j) {
  int q = k;
  if (q < d.nT) {
    i = q / SW - 2;
    j = q % SW - 4;
  } else if ((q -= d.nT) < d.nB) {
    i = TY + q / SW;
    j = q % SW - 4;
  } else if ((q -= d.nB) < d.nL) {
    i = d.rlo + (q >> 2);
    j = (q & 3) - 4;
  } else {
    q -= d.nL;
    i = d.rlo + (q >> 2);
    j = TW + (q & 3);
  }
}

}  // namespace hb
