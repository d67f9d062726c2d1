// thx_inst_order.cu -- instantiates the volume, gradient and indicator kernels
// of one (precision, dimension, order) triple.  Compiled once per triple with
// -DTHX_PREC=<0 double|1 float> -DTHX_DIM=<2|3> -DTHX_N=<nodes per direction>.
#include "thx_launch.cuh"

#ifndef THX_PREC
#error "THX_PREC must be defined"
#endif

#define THX_CAT4(a, b, c, d) a##_##b##_##c##_##d
#define THX_NAME(P, D, N) THX_CAT4(order_kernels, P, D, N)
#define THX_TYPE2(P) OrderKernels##P
#define THX_TYPE(P) THX_TYPE2(P)
#define THX_RT2(P) PREC_T_##P
#define THX_RT(P) THX_RT2(P)

namespace thx {

THX_TYPE(THX_PREC) THX_NAME(THX_PREC, THX_DIM, THX_N)() {
  using R = THX_RT(THX_PREC);
  THX_TYPE(THX_PREC) k;
  k.vol[VOL_CHANDRASHEKAR][0][0] = &launch_volume<R, THX_DIM, THX_N, VOL_CHANDRASHEKAR, false, false>;
  k.vol[VOL_CHANDRASHEKAR][0][1] = &launch_volume<R, THX_DIM, THX_N, VOL_CHANDRASHEKAR, false, true>;
  k.vol[VOL_CHANDRASHEKAR][1][0] = &launch_volume<R, THX_DIM, THX_N, VOL_CHANDRASHEKAR, true, false>;
  k.vol[VOL_CHANDRASHEKAR][1][1] = &launch_volume<R, THX_DIM, THX_N, VOL_CHANDRASHEKAR, true, true>;
  k.vol[VOL_RANOCHA][0][0] = &launch_volume<R, THX_DIM, THX_N, VOL_RANOCHA, false, false>;
  k.vol[VOL_RANOCHA][0][1] = &launch_volume<R, THX_DIM, THX_N, VOL_RANOCHA, false, true>;
  k.vol[VOL_RANOCHA][1][0] = &launch_volume<R, THX_DIM, THX_N, VOL_RANOCHA, true, false>;
  k.vol[VOL_RANOCHA][1][1] = &launch_volume<R, THX_DIM, THX_N, VOL_RANOCHA, true, true>;
  k.vol[VOL_PIROZZOLI][0][0] = &launch_volume<R, THX_DIM, THX_N, VOL_PIROZZOLI, false, false>;
  k.vol[VOL_PIROZZOLI][0][1] = &launch_volume<R, THX_DIM, THX_N, VOL_PIROZZOLI, false, true>;
  k.vol[VOL_PIROZZOLI][1][0] = &launch_volume<R, THX_DIM, THX_N, VOL_PIROZZOLI, true, false>;
  k.vol[VOL_PIROZZOLI][1][1] = &launch_volume<R, THX_DIM, THX_N, VOL_PIROZZOLI, true, true>;
  k.vol[VOL_CENTRAL][0][0] = &launch_volume<R, THX_DIM, THX_N, VOL_CENTRAL, false, false>;
  k.vol[VOL_CENTRAL][0][1] = &launch_volume<R, THX_DIM, THX_N, VOL_CENTRAL, false, true>;
  k.vol[VOL_CENTRAL][1][0] = &launch_volume<R, THX_DIM, THX_N, VOL_CENTRAL, true, false>;
  k.vol[VOL_CENTRAL][1][1] = &launch_volume<R, THX_DIM, THX_N, VOL_CENTRAL, true, true>;
#define THX_SETT(V)                                                              \
  k.vol_tma[V][0] = &launch_volume_tma<R, THX_DIM, THX_N, V, false>;             \
  k.vol_tma[V][1] = &launch_volume_tma<R, THX_DIM, THX_N, V, true>;
  THX_SETT(VOL_CHANDRASHEKAR)
  THX_SETT(VOL_RANOCHA)
  THX_SETT(VOL_PIROZZOLI)
  THX_SETT(VOL_CENTRAL)
#undef THX_SETT
#if THX_PREC == 0
  k.grad = &launch_grad_sv<R, THX_DIM, THX_N>;  // FP64: entropy variables precomputed
#else
  k.grad = &launch_grad<R, THX_DIM, THX_N>;     // FP32: evaluated in the kernel (cheaper)
#endif
  k.blend = &launch_blend<R, THX_DIM, THX_N>;
  k.fv = &launch_fv<R, THX_DIM, THX_N>;
#define THX_SETB(V)                                                              \
  k.volb[V][0] = &launch_volume_batched<R, THX_DIM, THX_N, V, false>;             \
  k.volb[V][1] = &launch_volume_batched<R, THX_DIM, THX_N, V, true>;
  THX_SETB(VOL_CHANDRASHEKAR)
  THX_SETB(VOL_RANOCHA)
  THX_SETB(VOL_PIROZZOLI)
  THX_SETB(VOL_CENTRAL)
#undef THX_SETB
  k.gradb = &launch_grad_batched<R, THX_DIM, THX_N>;
  k.epb = Shape<THX_DIM, THX_N>::EPB;
  k.epb_half = half_epb<THX_DIM, THX_N>();
  for (auto &row : k.volb_half)
    for (auto &v : row) v = nullptr;
  k.gradb_half = nullptr;
  if constexpr (half_epb<THX_DIM, THX_N>() > 0) {
    constexpr int H = half_epb<THX_DIM, THX_N>();
#define THX_SETH(V)                                                                \
  k.volb_half[V][0] = &launch_volume_batched<R, THX_DIM, THX_N, V, false, H>;      \
  k.volb_half[V][1] = &launch_volume_batched<R, THX_DIM, THX_N, V, true, H>;
    THX_SETH(VOL_CHANDRASHEKAR)
    THX_SETH(VOL_RANOCHA)
    THX_SETH(VOL_PIROZZOLI)
    THX_SETH(VOL_CENTRAL)
#undef THX_SETH
    k.gradb_half = &launch_grad_batched<R, THX_DIM, THX_N, H>;
  }
#if THX_PREC == 0
  k.voll[VOL_CHANDRASHEKAR] = &launch_volume_list<R, THX_DIM, THX_N, VOL_CHANDRASHEKAR>;
  k.voll[VOL_RANOCHA] = &launch_volume_list<R, THX_DIM, THX_N, VOL_RANOCHA>;
  k.voll[VOL_PIROZZOLI] = &launch_volume_list<R, THX_DIM, THX_N, VOL_PIROZZOLI>;
  k.voll[VOL_CENTRAL] = &launch_volume_list<R, THX_DIM, THX_N, VOL_CENTRAL>;
  k.fvl = &launch_fv_list<R, THX_DIM, THX_N>;
  k.blendl = &launch_blend_list<R, THX_DIM, THX_N>;
#else
  for (auto &v : k.voll) v = nullptr;
  k.fvl = nullptr;
  k.blendl = nullptr;
#endif
  return k;
}

}  // namespace thx
