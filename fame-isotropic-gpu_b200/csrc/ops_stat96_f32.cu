// Operator stage kernels with the compile-time 96 x 96 x 96 geometry (cubic Simple
// lattice at Nx = 96), FP32: the CG and refinement hot path and the operator benchmark.
#include "op_kernels.cuh"

namespace fame {
template __global__ void k_plane_inv<float, false, IN_CG, false, 0, Stat96>(PlaneInArgs<float>);
template __global__ void k_plane_inv<float, false, IN_VEC, false, 0, Stat96>(PlaneInArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ, 0, Stat96>(PencilArgs<float>);
template __global__ void k_pencil<float, false, PEN_QBQ_CG, 0, Stat96>(PencilArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_CGR, false, 0, Stat96>(PlaneOutArgs<float>);
template __global__ void k_plane_fwd<float, false, EPI_OUT, false, 0, Stat96>(PlaneOutArgs<float>);
FAME_DEFINE_LAUNCH_GETTER(launches_ops_stat96_f32)
}  // namespace fame
