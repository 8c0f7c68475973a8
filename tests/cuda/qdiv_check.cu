// Checks mpdx::qdiv (reciprocal times Markstein correction) against the CUDA
// '/' operator on random operands over many binades, FP64 and FP32, and
// mpdx::rdivf (FP32 quotient from an approximate reciprocal refined twice) on
// random numerators and denominators over 60 binades each, both signs, plus the
// FCT beta and frac operand ranges, and mpdx::rdivd (the FP64 quotient of the 2D
// march, within one ulp).  Prints the number of mismatches and exits non-zero if
// any qdiv or rdivf quotient differs, or any rdivd quotient is more than one ulp away.
#include <cstdio>

#include "../../libmpdataxx_b200/csrc/mpdx_common.cuh"

__device__ unsigned long long xs(unsigned long long &s) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return s; }

template <class T>
__global__ void k_check(const T *bs, int nb, long long per_thread, unsigned long long *bad) {
  unsigned long long s = 0x9E3779B97F4A7C15ull ^ (blockIdx.x * 1315423911ull + threadIdx.x * 2654435761ull + 1);
  unsigned long long nbad = 0;
  for (int t = 0; t < nb; ++t) {
    const T b = bs[t], y = T(1) / b;
    for (long long i = 0; i < per_thread; ++i) {
      const unsigned long long r = xs(s);
      const double u = double(r >> 11) * (1.0 / 9007199254740992.0) - 0.5;
      const T a = T(ldexp(u, int(r & 63) - 40));
      if (mpdx::qdiv<T>(a, b, y) != a / b) ++nbad;
    }
  }
  atomicAdd(bad, nbad);
}

// random float with a uniformly random 24-bit significand, exponent in [elo, ehi], random sign
__device__ float rnd_float(unsigned long long &s, int elo, int ehi, bool sign) {
  const unsigned long long r = xs(s);
  const int e = elo + int((r >> 40) % unsigned(ehi - elo + 1));
  const float m = 1.0f + float(r & 0x7fffff) * (1.0f / 8388608.0f);
  const float v = ldexpf(m, e);
  return (sign && (r >> 63)) ? -v : v;
}

__global__ void k_check_rdiv(long long per_thread, unsigned long long *bad) {
  unsigned long long s = 0xD1B54A32D192ED03ull ^ (blockIdx.x * 2246822519ull + threadIdx.x * 3266489917ull + 7);
  unsigned long long nbad = 0;
  for (long long i = 0; i < per_thread; ++i) {
    // general operands
    float a = rnd_float(s, -30, 30, true), b = rnd_float(s, -30, 30, true);
    if (mpdx::rdivf(a, b) != a / b) ++nbad;
    // FCT betas: (max - psi) / (sum of fluxes + FLT_EPSILON)
    a = rnd_float(s, -24, 12, false);
    b = rnd_float(s, -30, 12, false) + 1.1920929e-7f;
    if (mpdx::rdivf(a, b) != a / b) ++nbad;
    // frac: (p1 - p0) / ((p1 + p0) + FLT_MIN)
    const float p1 = rnd_float(s, -20, 10, false), p0 = rnd_float(s, -20, 10, false);
    a = p1 - p0;
    b = (p1 + p0) + 1.17549435e-38f;
    if (mpdx::rdivf(a, b) != a / b) ++nbad;
  }
  if (mpdx::rdivf(0.0f, 1.17549435e-38f) != 0.0f) ++nbad;
  atomicAdd(bad, nbad);
}

// mpdx::rdivd against '/': the general operands and the beta and frac ranges of the
// FP64 2D march; counts the quotients that differ and those more than one ulp away
__global__ void k_check_rdivd(long long per_thread, unsigned long long *diff, unsigned long long *far) {
  unsigned long long s = 0x94D049BB133111EBull ^ (blockIdx.x * 2654435761ull + threadIdx.x * 40503ull + 11);
  unsigned long long nd = 0, nf = 0;
  auto rnd = [&](int elo, int ehi, bool sign) {
    const unsigned long long r = xs(s), m = xs(s);
    const int e = elo + int((r >> 40) % unsigned(ehi - elo + 1));
    const double v = ldexp(1.0 + double(m >> 12) * (1.0 / 4503599627370496.0), e);
    return (sign && (r >> 63)) ? -v : v;
  };
  auto check = [&](double a, double b) {
    const double q = mpdx::rdivd(a, b), r = a / b;
    if (q != r) {
      ++nd;
      const long long d = __double_as_longlong(q) - __double_as_longlong(r);
      if (d > 1 || d < -1) ++nf;
    }
  };
  for (long long i = 0; i < per_thread; ++i) {
    check(rnd(-60, 60, true), rnd(-60, 60, true));
    check(rnd(-50, 12, false), rnd(-60, 12, false) + 2.220446049250313e-16);
    const double p1 = rnd(-40, 10, false), p0 = rnd(-40, 10, false);
    check(p1 - p0, (p1 + p0) + 2.2250738585072014e-308);
  }
  atomicAdd(diff, nd);
  atomicAdd(far, nf);
}

int main() {
  const double bd[] = {10.0, 0.1, 3.0, 7.3, 1e-3, 123.456, 0.75, 1.0 / 3.0, 12.5, 0.01};
  const int nb = 10;
  double *dbd; float *dbf; unsigned long long *dbad;
  float bf[nb];
  for (int i = 0; i < nb; ++i) bf[i] = float(bd[i]);
  cudaMalloc(&dbd, sizeof(bd)); cudaMalloc(&dbf, sizeof(bf)); cudaMalloc(&dbad, 2 * sizeof(unsigned long long));
  cudaMemcpy(dbd, bd, sizeof(bd), cudaMemcpyHostToDevice);
  cudaMemcpy(dbf, bf, sizeof(bf), cudaMemcpyHostToDevice);
  cudaMemset(dbad, 0, 2 * sizeof(unsigned long long));
  k_check<double><<<148 * 4, 256>>>(dbd, nb, 1000, dbad);
  k_check<float><<<148 * 4, 256>>>(dbf, nb, 1000, dbad + 1);
  unsigned long long *dbad2;
  cudaMalloc(&dbad2, sizeof(unsigned long long));
  cudaMemset(dbad2, 0, sizeof(unsigned long long));
  k_check_rdiv<<<148 * 4, 256>>>(4000, dbad2);
  unsigned long long *dd3;
  cudaMalloc(&dd3, 2 * sizeof(unsigned long long));
  cudaMemset(dd3, 0, 2 * sizeof(unsigned long long));
  k_check_rdivd<<<148 * 4, 256>>>(2000, dd3, dd3 + 1);
  unsigned long long bad[2] = {1, 1}, bad2 = 1, d3[2] = {1, 1};
  cudaError_t e = cudaMemcpy(bad, dbad, sizeof(bad), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&bad2, dbad2, sizeof(bad2), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(d3, dd3, sizeof(d3), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { std::printf("CUDA error: %s\n", cudaGetErrorString(e)); return 2; }
  const long long n = 148LL * 4 * 256 * 1000 * nb;
  std::printf("qdiv vs '/': %lld operand pairs per type, mismatches fp64 %llu fp32 %llu\n", n, bad[0], bad[1]);
  std::printf("rdivf vs '/': %lld operand pairs, mismatches %llu\n", 148LL * 4 * 256 * 4000 * 3, bad2);
  std::printf("rdivd vs '/': %lld operand pairs, differing %llu, more than one ulp away %llu\n", 148LL * 4 * 256 * 2000 * 3,
              d3[0], d3[1]);
  return (bad[0] || bad[1] || bad2 || d3[1]) ? 1 : 0;
}
