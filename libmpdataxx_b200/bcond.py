"""Boundary-condition kinds (libmpdata++/bcond/detail/bcond_common.hpp bcond_e)."""


class _bc:
    def __init__(self, name):
        self.name = name

    def __repr__(self):
        return f"bcond.{self.name}"


cyclic = _bc("cyclic")
open = _bc("open")
rigid = _bc("rigid")
gndsky = _bc("gndsky")  # bcond/gndsky_3d.hpp: ground (left) and sky (right) of the vertical axis, rigid for iles
