// Specialised TMA-pipelined FFT passes, double precision (plain form).
#include "fft2.cuh"

namespace inqb {
template <> bool launch_fft2<double>(Ctx &ctx, const Basis &b, const PassArgs<double> &a, int pro, int epi) {
  return v2::launch<double>(ctx, b, a, pro, epi);
}
template <>
bool launch_fft2_pair<double>(Ctx &ctx, const Basis &b, const PassArgs<double> &a, int axisA, int axisB, bool inverse,
                         const void *inA, void *outA, const void *inB, void *outB) {
  return v2::launch_pair<double>(ctx, b, a, axisA, axisB, inverse, inA, outA, inB, outB);
}
}  // namespace inqb
