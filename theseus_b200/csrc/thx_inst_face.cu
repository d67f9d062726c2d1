// thx_inst_face.cu -- instantiates the face-flux kernels of one
// (precision, dimension) pair.  Compiled with -DTHX_PREC and -DTHX_DIM.
#include "thx_launch.cuh"

#define THX_CAT3(a, b, c) a##_##b##_##c
#define THX_NAME(P, D) THX_CAT3(face_kernels, P, D)
#define THX_TYPE2(P) FaceKernels##P
#define THX_TYPE(P) THX_TYPE2(P)
#define THX_RT2(P) PREC_T_##P
#define THX_RT(P) THX_RT2(P)

namespace thx {

THX_TYPE(THX_PREC) THX_NAME(THX_PREC, THX_DIM)() {
  using R = THX_RT(THX_PREC);
  THX_TYPE(THX_PREC) k;
#define THX_SET(S)                                             \
  k.face[S][0] = &launch_face<R, THX_DIM, S, false>;           \
  k.face[S][1] = &launch_face<R, THX_DIM, S, true>;            \
  k.faceb[S][0] = &launch_face_batched<R, THX_DIM, S, false>;  \
  k.faceb[S][1] = &launch_face_batched<R, THX_DIM, S, true>;
  THX_SET(SURF_CHANDRASHEKAR)
  THX_SET(SURF_RANOCHA)
  THX_SET(SURF_PIROZZOLI)
  THX_SET(SURF_HLL)
  THX_SET(SURF_LLF)
  THX_SET(SURF_ROE)
#undef THX_SET
  k.entropy = &launch_entropy<R, THX_DIM>;
#if THX_PREC == 0
  k.facel[SURF_CHANDRASHEKAR] = &launch_face_list<R, THX_DIM, SURF_CHANDRASHEKAR>;
  k.facel[SURF_RANOCHA] = &launch_face_list<R, THX_DIM, SURF_RANOCHA>;
  k.facel[SURF_PIROZZOLI] = &launch_face_list<R, THX_DIM, SURF_PIROZZOLI>;
  k.facel[SURF_HLL] = &launch_face_list<R, THX_DIM, SURF_HLL>;
  k.facel[SURF_LLF] = &launch_face_list<R, THX_DIM, SURF_LLF>;
  k.facel[SURF_ROE] = &launch_face_list<R, THX_DIM, SURF_ROE>;
#else
  for (auto &f : k.facel) f = nullptr;
#endif
#if THX_PREC == 0
#define THX_SETBND(S)                                   \
  k.bnd[S][0] = &launch_bnd<THX_DIM, S, false>;          \
  k.bnd[S][1] = &launch_bnd<THX_DIM, S, true>;
  THX_SETBND(SURF_CHANDRASHEKAR)
  THX_SETBND(SURF_RANOCHA)
  THX_SETBND(SURF_PIROZZOLI)
  THX_SETBND(SURF_HLL)
  THX_SETBND(SURF_LLF)
  THX_SETBND(SURF_ROE)
#undef THX_SETBND
#else
  for (auto &b : k.bnd) b[0] = b[1] = nullptr;
#endif
  return k;
}

}  // namespace thx
