// MPDATA options and compile-time parameter defaults of the libmpdata++ API
// (same names and bit values as libmpdata++/opts.hpp:34-100), for programs
// that drive the B200 backend through concurr::cuda.
#pragma once

#include <string>

namespace libmpdataxx {
namespace opts {
using opts_t = unsigned long;
constexpr opts_t bit(const opts_t &x) { return opts_t(1) << x; }
constexpr bool isset(const opts_t &x, const opts_t &y) { return 0 != (x & y); }
enum : opts_t {
  fct = bit(0), abs = bit(1), tot = bit(2), pfc = bit(3), npa = bit(4), iga = bit(5), nug = bit(6),
  dfl = bit(7), khn = bit(8), div_2nd = bit(9), div_3rd = bit(10), div_3rd_dt = bit(11), fot = bit(12)
};
inline std::string opts_string(opts_t o) {
  const std::pair<opts_t, const char *> order[] = {{nug, "nug"}, {iga, "iga"}, {abs, "abs"}, {dfl, "dfl"},
                                                   {div_2nd, "div_2nd"}, {tot, "tot"}, {div_3rd, "div_3rd"},
                                                   {fot, "fot"}, {fct, "fct"}, {pfc, "pfc"}, {npa, "npa"}, {khn, "khn"}};
  std::string r;
  for (const auto &p : order)
    if (isset(o, p.first)) r += '|' + std::string(p.second);
  return r.empty() ? "0" : r.substr(1);
}
}  // namespace opts

struct ct_params_default_t {
  enum { opts = opts::iga | opts::fct };
  enum { hint_norhs = 0 };
  enum { delayed_step = 0 };
  struct ix {};
  static constexpr int hint_scale(const int &) { return 0; }
  enum { var_dt = false };
  enum { vip_vab = 0 };
  enum { prs_k_iters = 4 };
  enum { prs_khn = false };
  enum { sgs_scheme = 0 };
  enum { stress_diff = 0 };
  enum { impl_tht = false };
  enum { sptl_intrp = 0 };
  enum { tmprl_extrp = 0 };
  enum { out_intrp_ord = 1 };
};
}  // namespace libmpdataxx
