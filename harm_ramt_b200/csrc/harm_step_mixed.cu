// Mixed-precision instantiations of the step kernels: FP32 interface states,
// wavespeeds and face fluxes (FP32 face geometry, FP32 flux storage), with
// the con-to-prim solve, conserved update, geometric source, EMF and dt in
// FP64.  This translation unit is built with multiply-add contraction and
// fast FP32 division and square root; it is not bit-identical to the
// reference (harm_step.cu is).
#include "harm_step_impl.cuh"

namespace harm {

void launch_flux_mixed(int para, int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a,
                       const CUtensorMap& prim_map)
{
  if (ffde) {
    if (para) flux_rows_launch<float, true, true>(g, b, s, a, prim_map);
    else flux_rows_launch<float, false, true>(g, b, s, a, prim_map);
  } else if (para) flux_rows_launch<float, true, false>(g, b, s, a, prim_map);
  else flux_rows_launch<float, false, false>(g, b, s, a, prim_map);
}

void launch_emf_mixed(dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const double* pv)
{
  k_emf<float><<<g, b, 0, s>>>(a, pv);
}

void launch_update_mixed(int ffde, dim3 g, dim3 b, cudaStream_t s, const StepArgs& a, const CUtensorMap& map,
                         const double* pi, const double* pb, double* pf, double c2)
{
  if (ffde) update_launch<float, true>(g, b, s, a, map, pi, pb, pf, c2);
  else update_launch<float, false>(g, b, s, a, map, pi, pb, pf, c2);
}

}  // namespace harm
