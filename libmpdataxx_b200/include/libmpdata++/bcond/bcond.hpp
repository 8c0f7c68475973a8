// Boundary-condition kinds (libmpdata++/bcond/detail/bcond_common.hpp bcond_e).
#pragma once

#include <mpdx.h>

namespace libmpdataxx {
namespace bcond {
// gndsky: the 3D ground / sky condition (bcond/gndsky_3d.hpp), rigid for every field
// this backend fills
enum bcond_e { null, cyclic, open, rigid, gndsky };
inline int to_c(bcond_e b) {
  switch (b) {
    case cyclic: return MPDX_BC_CYCLIC;
    case open: return MPDX_BC_OPEN;
    case rigid: return MPDX_BC_RIGID;
    case gndsky: return MPDX_BC_GNDSKY;
    default: return -1;
  }
}
}  // namespace bcond
}  // namespace libmpdataxx
