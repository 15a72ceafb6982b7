// Specialised TMA-pipelined FFT passes, double precision (plain form).
#include "fft2.cuh"

namespace inqb {
template <> bool launch_fft2<double>(Ctx &ctx, const Basis &b, const PassArgs<double> &a, int pro, int epi) {
  return v2::launch<double>(ctx, b, a, pro, epi);
}
}  // namespace inqb
