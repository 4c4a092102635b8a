// Plain device-side views shared by the library and by kernels compiled at
// run time (no host headers: the run-time compiler sees only what the
// library hands it).
#pragma once

#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

namespace psb {

// A strided view of one grid: element (x, y, z) lives at
// origin[x + y*sy + z*sz]. Dense grids have sy = nx, sz = nx*ny; pitched
// grids have 128-byte rows and a resident halo around the origin.
struct GridView {
  void *origin;
  int64_t sy, sz;
  int n[3];
  int type;      // PSPrimitiveType or -1 when unknown
  int halo;      // cells of resident halo in every direction (0 for dense)
};

struct Dom3 {
  int lo[3];
  int hi[3];
};

}  // namespace psb
