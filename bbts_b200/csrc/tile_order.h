// Tile order of the grouped tcgen05 launches, as plain index arithmetic shared
// by the kernels (gemm_tc.cuh) and the host tests (tests/cpp/test_host.cc),
// which check on the CPU that every launch visits each tile exactly once.
#pragma once

#if defined(__CUDACC__)
#define BBX_HD __host__ __device__ __forceinline__
#else
#define BBX_HD inline
#endif

namespace bbx {

// Tile-rows per band: tiles inside a problem are visited in bands of this
// many tile-rows, column by column, so concurrently running CTAs share
// operand tiles in L2.
constexpr int kTileBand = 16;

// Tile (tm, tn) of local tile index lt in a problem of tiles_m x tiles_n tiles.
BBX_HD void band_tile(int lt, int tiles_m, int tiles_n, int& tm, int& tn) {
  const int per_band = kTileBand * tiles_n;
  const int band = lt / per_band;
  const int first_m = band * kTileBand;
  const int rows = tiles_m - first_m < kTileBand ? tiles_m - first_m : kTileBand;
  const int r = lt - band * per_band;
  tm = first_m + r % rows;
  tn = r / rows;
}

// Tile of CTA `b` (of `grid`) in round `round`, t0 = round * grid + b: snake
// order, so in odd rounds CTA b takes the round's tile grid - 1 - b and a CTA
// that drew a costly tile early in the list draws a cheap one next (plans sort
// problems by descending tile cost). A partial last round keeps the plain order.
BBX_HD int snake_tile_of(int t0, int round, int total, int b, int grid) {
  const int base = t0 - b;
  if ((round & 1) && base + grid <= total) return base + grid - 1 - b;
  return t0;
}

}  // namespace bbx
