// Launchers of the kernels that are templated on the species count (the
// stencil stage, the fused RK2 stages and the adjoint VJP).  Each species
// count is instantiated in its own translation unit (launch_ns.cu compiled
// with ARCOS_NS = 1..6), so the library builds in parallel; the host code
// dispatches on the run-time count to launch_*_ns<NS>.
#pragma once
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "stage_kernel.cuh"
#include "fused_kernel.cuh"
#include "adjoint_kernel.cuh"
#include "march_kernel.cuh"

namespace arcos {

// Reaction tables up to this many nodes are staged in shared memory by k_stage.
constexpr int NODES_SMEM_MAX = 4 * 1024 / (int) sizeof (TableNode);

// Tile shapes the autotuner chooses from: (warps per block, rows per thread);
// tiles are 32 columns wide and WY * RPW rows high.
constexpr int N_TILE_CFG = 3;
constexpr int TILE_WY[N_TILE_CFG] = {4, 8, 8};
constexpr int TILE_RPW[N_TILE_CFG] = {4, 4, 2};

// Segment heights of the marching kernel (tile shapes N_TILE_CFG ..).
constexpr int N_MARCH_H = 3;
constexpr int MARCH_H[N_MARCH_H] = {16, 32, 64};

// Each launches (occ == nullptr) or returns the resident blocks per SM in
// *occ (after setting the kernel's dynamic shared-memory limit).
template <int NS>
cudaError_t launch_stage_ns (int mode, int cfg, const Model &M, const StageArgs &A, int blocks,
                             cudaStream_t s, int *occ);
template <int NS>
cudaError_t launch_fused_ns (bool s2, bool tree, int cfg, const Model &M, const FusedArgs &A, int blocks,
                             cudaStream_t s, int *occ);
template <int NS>
cudaError_t launch_march_ns (bool s2, bool tree, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s);
template <int NS>
cudaError_t launch_vjp_ns (const Model &M, const VjpArgs &A, int blocks, size_t smem, cudaStream_t st,
                           int *occ);
template <int NS>
cudaError_t launch_vjp_split_ns (const Model &M, const VjpArgs &A, int blocks_f, int blocks_r, size_t smem_r,
                                 cudaStream_t st, int *occ);

#define ARCOS_DECLARE_NS(N)                                                                          \
  extern template cudaError_t launch_stage_ns<N> (int, int, const Model &, const StageArgs &, int,   \
                                                  cudaStream_t, int *);                              \
  extern template cudaError_t launch_fused_ns<N> (bool, bool, int, const Model &, const FusedArgs &,  \
                                                  int, cudaStream_t, int *);                         \
  extern template cudaError_t launch_vjp_ns<N> (const Model &, const VjpArgs &, int, size_t,         \
                                                cudaStream_t, int *);                                \
  extern template cudaError_t launch_vjp_split_ns<N> (const Model &, const VjpArgs &, int, int,      \
                                                      size_t, cudaStream_t, int *);                  \
  extern template cudaError_t launch_march_ns<N> (bool, bool, const Model &, const FusedArgs &, int, \
                                                  cudaStream_t);
ARCOS_DECLARE_NS (1)
ARCOS_DECLARE_NS (2)
ARCOS_DECLARE_NS (3)
ARCOS_DECLARE_NS (4)
ARCOS_DECLARE_NS (5)
ARCOS_DECLARE_NS (6)
#undef ARCOS_DECLARE_NS

}  // namespace arcos
