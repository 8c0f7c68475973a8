"""MPDATA option bits, bit-for-bit the values of libmpdata++/opts.hpp:34-49."""

fct = 1 << 0         # flux-corrected transport
abs = 1 << 1         # variable-sign signal via the abs() trick
tot = 1 << 2         # third-order terms
pfc = 1 << 3         # where(den != 0, nom / den, 0) in psi fractions
npa = 1 << 4         # (x - |x|) / 2 style negative/positive parts
iga = 1 << 5         # infinite-gauge option
nug = 1 << 6         # non-unit G
dfl = 1 << 7         # divergent-flow correction
khn = 1 << 8         # Kahan summation in donor-cell
div_2nd = 1 << 9
div_3rd = 1 << 10
div_3rd_dt = 1 << 11
fot = 1 << 12

_names = [(nug, "nug"), (iga, "iga"), (abs, "abs"), (dfl, "dfl"), (div_2nd, "div_2nd"), (tot, "tot"),
          (div_3rd, "div_3rd"), (fot, "fot"), (fct, "fct"), (pfc, "pfc"), (npa, "npa"), (khn, "khn")]


def isset(x, y):
    return (x & y) != 0


def opts_string(o):
    """Same spelling and order as libmpdata++/opts.hpp:66-78."""
    s = "|".join(n for b, n in _names if o & b)
    return s if s else "0"
