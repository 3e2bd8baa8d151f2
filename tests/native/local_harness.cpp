// Host build of the walk's local-expansion arithmetic (tree_b200/csrc/local.cuh)
// for the CPU tests: the same source the device compiles, run in FP32 on the
// host through ctypes.
#include <cstring>
#include "local.cuh"

extern "C" {

// m: 33 floats in CellMoments order (q, d[3], s[6], t[10], h[12], q_ion)
void loc_coefs(int order, const float* d, const float* m, float* c) {
  tg::CellMoments cm;
  static_assert(sizeof(tg::CellMoments) == 33 * sizeof(float), "CellMoments layout");
  std::memcpy(&cm, m, sizeof(cm));
  if (order >= 4) tg::local_coefs<4>(d[0], d[1], d[2], cm, c);
  else if (order == 3) tg::local_coefs<3>(d[0], d[1], d[2], cm, c);
  else tg::local_coefs<2>(d[0], d[1], d[2], cm, c);
}

// out: fx, fy, fz, phi, phi_ion
void loc_eval(const float* c, const float* t, float* out) {
  tg::local_eval(c, t[0], t[1], t[2], out[0], out[1], out[2], out[3], out[4]);
}

}
