// Stand-in for the part of NTL's RR interface the reference uses: its only
// use on the harness's path is floor(4^b / p) for the Barrett constants
// (aoa-ntt src/cuda/htrans/common.cu:487-497), which an exact rational gives
// (NTL computes it at 2048 bits of precision, far above what that quotient
// needs).  Division is by values below 2^64 only.  Test infrastructure only.
#pragma once
#include <NTL/ZZ.h>

namespace NTL {

class RR {
 public:
  ZZ num, den = ZZ::of(1);
  static void SetPrecision(long) {}
  static void SetOutputPrecision(long) {}
};

inline RR to_RR(const ZZ& z) {
  RR r;
  r.num = z;
  return r;
}
inline RR to_RR(uint64_t v) { return to_RR(ZZ::of(v)); }
inline RR to_RR(long v) { return to_RR(ZZ(v)); }

inline RR operator/(const RR& a, const RR& b) {
  RR r;
  r.num = a.num * b.den;
  r.den = a.den * b.num;
  return r;
}
inline RR floor(const RR& a) { return to_RR(a.num / a.den); }

template <class T>
inline T conv(const RR& r) {
  if (!(r.den == ZZ::of(1))) stand_in_abort("conv: RR is not an integer");
  return conv<T>(r.num);
}

}  // namespace NTL
