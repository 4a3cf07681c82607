// Corrector coefficient sets of the reference (FSLBM.cu:177-232): the active order 4<->2 blend
// and the orders 6..14 and 8<->6, 6<->4 blends it keeps as alternatives. The decimals are the
// reference's, formed in FP32 or FP64 as the reference forms its active set (FSLBM.cu:231).
#include "internal.h"

namespace fslbm {

template <class T>
static int fd_table(int order, T b, T* c) {
  for (int k = 0; k < 9; ++k) c[k] = T(0);
  switch (order) {
    case 0: case 4:   // 4 <-> 2 (blend 1: order 4, 0: order 2)
      c[0] = T(-6.0) - T(1.5) * b; c[1] = T(1.0) + T(0.3333333333) * b; c[2] = T(-0.0833333333) * b;
      return 2;
    case 6:           // 6 <-> 4
      c[0] = T(-7.5) - T(0.66666666666) * b; c[1] = T(1.3333333) + T(0.16666666666) * b;
      c[2] = T(-0.08333333) - T(0.0666666666666) * b; c[3] = T(0.01111111) * b;
      return 3;
    case 8:           // 8 <-> 6
      c[0] = T(-8.166666666666666) - T(0.375) * b; c[1] = T(1.5) + T(0.1) * b;
      c[2] = T(-0.15) - T(0.05) * b; c[3] = T(0.01111111) + T(0.014285714285714) * b;
      c[4] = T(-0.001785714285714) * b;
      return 4;
    case 10:
      c[0] = T(-8.78166666666); c[1] = T(1.66666666); c[2] = T(-0.23809523809);
      c[3] = T(0.03968253968); c[4] = T(-0.00496031746); c[5] = T(0.00031746031);
      return 5;
    case 12:
      c[0] = T(-8.94833333333); c[1] = T(1.71428571429); c[2] = T(-0.26785714285);
      c[3] = T(0.05291005291); c[4] = T(-0.00892857142); c[5] = T(0.00103896103);
      c[6] = T(-0.00006012506);
      return 6;
    case 14:
      c[0] = T(-9.16453231293); c[1] = T(1.77777777778); c[2] = T(-0.31111111111);
      c[3] = T(0.07542087542); c[4] = T(-0.01767676767); c[5] = T(3.48096348e-3);
      c[6] = T(-5.1800052e-4); c[7] = T(5.0742908e-5); c[8] = T(-2.4281274e-6);
      return 8;
    default:
      return 0;
  }
}

int fd_coefficients(int order, double blend, int fp32, double* c) {
  if (fp32) {
    float f[9];
    const int K = fd_table<float>(order, float(blend), f);
    for (int k = 0; k < 9; ++k) c[k] = double(f[k]);
    return K;
  }
  return fd_table<double>(order, blend, c);
}

}  // namespace fslbm

extern "C" int fslbm_fd_coefficients(int order, double blend, fslbm_dtype dtype, double* c, int* taps) {
  if (!c) return FSLBM_ERR_ARG;
  const int K = fslbm::fd_coefficients(order, blend, dtype != FSLBM_F64, c);
  if (taps) *taps = K;
  return K ? FSLBM_OK : FSLBM_ERR_ARG;
}
