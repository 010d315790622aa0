// tile2d_cfg.cuh -- the compiled register layouts of the 2D tile routine and
// the mapping from a wf_tune region shape (and thread count) to one of them.
#pragma once

#include "tile2d.cuh"

namespace wf {

// TileCfg<rows per thread, columns per thread, warps>: one warp spans the
// region width (32 x columns per thread), the warps stack along i.
using Cfg64x128w = TileCfg<2, 4, 32>;  // 1024 threads, 2 x 4 cells each (64 registers)
using Cfg64x128 = TileCfg<4, 4, 16>;   // 512 threads, 4 x 4 cells each
using Cfg48x128 = TileCfg<3, 4, 16>;   // 512 threads, 3 x 4 cells each
using Cfg48x128w = TileCfg<2, 4, 24>;  // 768 threads, 2 x 4 cells each
using Cfg32x128 = TileCfg<4, 4, 8>;    // 256 threads, 4 x 4 cells each
using Cfg32x64 = TileCfg<4, 2, 8>;     // 256 threads, 4 x 2 cells each
using Cfg8x32 = TileCfg<4, 1, 2>;      // 64 threads (small grids and tests)

inline int check_tune2d(const wf_tune& t) {
  const int rh = t.tile_i, rw = t.tile_j, k = t.steps_per_pass;
  const bool known = (rh == 48 && rw == 128) || (rh == 64 && rw == 128) || (rh == 32 && rw == 128) ||
                     (rh == 32 && rw == 64) || (rh == 8 && rw == 32);
  if (!known)
    return set_error(WF_E_ARG,
                     "2D tune: region %dx%d is not compiled (48x128, 64x128, 32x128, 32x64, 8x32)", rh,
                     rw);
  if (k < 1 || 2 * k >= rh || 2 * k >= rw)
    return set_error(WF_E_ARG, "2D tune: k=%d leaves no core in a %dx%d region", k, rh, rw);
  return WF_OK;
}

// Calls f.template operator()<Cfg>() for the configuration of t: 48 x 128 on
// 768 threads when t.threads >= 768 (else 512); 64 x 128 on 512 threads when
// t.threads == 512 (else 1024).
template <class F>
int dispatch_cfg2d(const wf_tune& t, const F& f) {
  if (t.tile_i == 48)
    return t.threads >= 768 ? f.template operator()<Cfg48x128w>() : f.template operator()<Cfg48x128>();
  if (t.tile_i == 64)
    return t.threads == 512 ? f.template operator()<Cfg64x128>() : f.template operator()<Cfg64x128w>();
  if (t.tile_i == 32 && t.tile_j == 128) return f.template operator()<Cfg32x128>();
  if (t.tile_i == 32) return f.template operator()<Cfg32x64>();
  return f.template operator()<Cfg8x32>();
}

}  // namespace wf
