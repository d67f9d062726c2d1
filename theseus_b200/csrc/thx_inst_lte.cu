// thx_inst_lte.cu -- instantiates the FP64 LTE Helmholtz kernels.  Compiled
// with -DTHX_DIM=<2|3> and either -DTHX_N=<nodes per direction> (LTEEC volume
// and gradient kernels of one order) or without THX_N (the face kernels).
#include "thx_launch.cuh"

#define THX_CAT3(a, b, c) a##_##b##_##c
#define THX_CAT2(a, b) a##_##b
#define THX_XCAT3(a, b, c) THX_CAT3(a, b, c)
#define THX_XCAT2(a, b) THX_CAT2(a, b)

namespace thx {

#ifdef THX_N
LteKernels THX_XCAT3(lte_kernels, THX_DIM, THX_N)() {
  LteKernels k;
  k.vol[0] = &launch_volume<double, THX_DIM, THX_N, VOL_LTEEC, false, false>;
  k.vol[1] = &launch_volume<double, THX_DIM, THX_N, VOL_LTEEC, true, false>;
  k.grad = &launch_grad<double, THX_DIM, THX_N, true>;
  return k;
}
#else
LteFaceKernels THX_XCAT2(lte_face_kernels, THX_DIM)() {
  LteFaceKernels k;
  k.face[0] = &launch_face<double, THX_DIM, SURF_LTEEC, false>;
  k.face[1] = &launch_face<double, THX_DIM, SURF_LTEEC, true>;
  return k;
}
#endif

}  // namespace thx
