// Tile shapes of the five matvec passes.
#include "dda_host.h"

namespace dda {

// Elements per CTA tile (EPT * NT of the pass kernels): 48 KiB of shared
// memory in either precision.
static int tile_cap(bool dbl) { return dbl ? 12 * 256 : 24 * 256; }

PassCfg make_pass_cfg(const Geo& g, bool dbl) {
  PassCfg c{};
  const int cap = tile_cap(dbl);
  const size_t esz = dbl ? 16 : 8;
  // z passes: NL lines of 3 interleaved transforms each
  c.NL = cap / (3 * g.Lz);
  if (c.NL < 1) c.NL = 1;
  c.WS1 = 3 * g.Lz;
  c.smem1 = (size_t)c.NL * 3 * g.Lz * esz;
  c.grid1 = ((long long)g.nx * g.ny + c.NL - 1) / c.NL;
  // y passes: Tz consecutive kz per (ix) slab
  c.Tz2 = cap / (3 * g.Ly);
  if (c.Tz2 > g.Lz) c.Tz2 = g.Lz;
  if (c.Tz2 < 1) c.Tz2 = 1;
  c.WS2 = 3 * c.Tz2;
  c.smem2 = (size_t)g.Ly * c.WS2 * esz;
  c.ntz2 = (g.Lz + c.Tz2 - 1) / c.Tz2;
  c.grid2 = (long long)g.nx * c.ntz2;
  // x pass: Tz consecutive kz per ky pencil row
  c.Tz3 = cap / (3 * g.Lx);
  if (c.Tz3 > g.Lz) c.Tz3 = g.Lz;
  if (c.Tz3 < 1) c.Tz3 = 1;
  c.WS3 = 3 * c.Tz3;
  c.smem3 = (size_t)g.Lx * c.WS3 * esz;
  c.ntz3 = (g.Lz + c.Tz3 - 1) / c.Tz3;
  c.grid3 = (long long)g.Ly * c.ntz3;
  return c;
}

}  // namespace dda
