// ORACLE -- test infrastructure only.  Boussinesq + GCR pressure solve (filled in below).
#pragma once
#include "mpdata_oracle.hpp"
namespace mpdx_oracle {
template <class T>
struct boussinesq : mpdata<T> {
  long long iters = 0;
  void setup_bq(int, const int *, unsigned, int, const int *, const double *, int) {
    throw std::runtime_error("oracle: boussinesq not available");
  }
  arr<T> &sclr_array(const char *) { throw std::runtime_error("no such scalar array"); }
};
}  // namespace mpdx_oracle
