// Specialised TMA-pipelined FFT passes, single precision (mixed form).
#include "fft2.cuh"

namespace inqb {
template <> bool launch_fft2<float>(Ctx &ctx, const Basis &b, const PassArgs<float> &a, int pro, int epi) {
  return v2::launch<float>(ctx, b, a, pro, epi);
}
template <>
bool launch_fft2_pair<float>(Ctx &ctx, const Basis &b, const PassArgs<float> &a, int axisA, int axisB, bool inverse,
                         const void *inA, void *outA, const void *inB, void *outB) {
  return v2::launch_pair<float>(ctx, b, a, axisA, axisB, inverse, inA, outA, inB, outB);
}
}  // namespace inqb
