// pf5d_tiles.cuh -- shared-memory tile geometry of the rate kernels.
//
// A plane tile is TY rows (axis "y") by TX columns (the contiguous axis
// "x").  The composition is staged with a 2-cell halo (HY x HX) so the
// Laplacian can be evaluated on a 1-cell halo; chemical potential and
// mobility live on that 1-cell halo (MY x MX, corners unused).  x-faces:
// TY x (TX+1), face (y, f) between columns f-1 and f; y-faces: (TY+1) x TX,
// face (f, x) between rows f-1 and f.
#pragma once

namespace pf5d {

// NTH: threads of the block (default one per tile point); a block may have
// more threads than tile points so that the halo positions need no second
// pass.
template <int TX, int TY, int NTH = TX * TY>
struct PlaneGeom {
  static constexpr int HX = TX + 4, HY = TY + 4, PX = HX * HY;
  static constexpr int MX = TX + 2, MY = TY + 2, PM = MX * MY;
  static constexpr int NT = NTH;
  static constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
};

}  // namespace pf5d
