// Specialised TMA-pipelined FFT passes, single precision (mixed form).
#include "fft2.cuh"

namespace inqb {
template <> bool launch_fft2<float>(Ctx &ctx, const Basis &b, const PassArgs<float> &a, int pro, int epi) {
  return v2::launch<float>(ctx, b, a, pro, epi);
}
}  // namespace inqb
