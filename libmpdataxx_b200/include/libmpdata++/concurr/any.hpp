// concurr::any<real_t, n_dims> (libmpdata++/concurr/any.hpp:15-74): the
// abstract run interface, so that user code can hold any backend through a
// std::unique_ptr<concurr::any<...>>.
#pragma once

#include <stdexcept>
#include <string>

#include "../host_array.hpp"

namespace libmpdataxx {
namespace concurr {

template <typename real_t, int n_dims, class advance_arg_t = int>
class any {
 public:
  using arr_t = host_view<real_t, n_dims>;
  virtual ~any() = default;
  virtual arr_t advectee(int e = 0) = 0;
  virtual arr_t advectee_global(int e = 0) { return advectee(e); }
  virtual void advectee_global_set(const arr_t &a, int e = 0) = 0;
  virtual arr_t advector(int d = 0) = 0;
  virtual arr_t g_factor() = 0;
  // velocity absorber fields (vip_vab); solvers without the option throw (sharedmem.hpp:471-494)
  virtual arr_t vab_coefficient() { throw std::runtime_error("libmpdata++: vab_coeff() called with option vip_vab unset?"); }
  virtual arr_t vab_relaxed_state(int = 0) { throw std::runtime_error("libmpdata++: vab_relaxed_state() called with option vip_vab unset?"); }
  virtual arr_t sclr_array(const std::string &name, int n = 0) = 0;
  virtual void advance(advance_arg_t nt) = 0;
  virtual real_t min(int e = 0) = 0;
  virtual real_t max(int e = 0) = 0;
  virtual real_t time() const = 0;
  virtual bool *panic_ptr() = 0;
};

}  // namespace concurr
}  // namespace libmpdataxx
