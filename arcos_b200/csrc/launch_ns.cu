// The kernels templated on the species count, for one count: ARCOS_NS
// (compiled once per count, 1..6, and linked into the library).
#include "launch.cuh"

#ifndef ARCOS_NS
#error "compile with -DARCOS_NS=<species count>"
#endif

namespace arcos {

template <int NS, int MODE, int WY, int RPW>
size_t
stage_smem_t (int n_nodes, int stage_eabs)
{
  using LY = TileLayout<NS, MODE, WY, RPW>;
  size_t b = sizeof (double) * (size_t) ((stage_eabs ? LY::NA : LY::NA - 1) * LY::PLANE + LY::OPP);
  if (n_nodes > 0 && n_nodes <= NODES_SMEM_MAX) b += sizeof (TableNode) * (size_t) n_nodes;
  return b;
}

template <int NS, int MODE, int WY, int RPW, bool FAST>
cudaError_t
launch_stage_t (const Model &M, const StageArgs &A, int blocks, cudaStream_t s, int *occ)
{
  const size_t sm = stage_smem_t<NS, MODE, WY, RPW> (A.n_nodes, A.stage_eabs);
  cudaFuncSetAttribute (k_stage<NS, MODE, WY, RPW, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
  if (occ) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor (occ, k_stage<NS, MODE, WY, RPW, FAST>, 32 * WY, sm);
    return cudaGetLastError ();
  }
  k_stage<NS, MODE, WY, RPW, FAST><<<blocks, 32 * WY, sm, s>>> (M, A);
  return cudaGetLastError ();
}

template <int NS, int MODE>
cudaError_t
launch_stage_c (int cfg, const Model &M, const StageArgs &A, int blocks, cudaStream_t s, int *occ)
{
  const bool fast = !A.exact;
  switch (cfg) {
  case 0: return fast ? launch_stage_t<NS, MODE, 4, 4, true> (M, A, blocks, s, occ)
                      : launch_stage_t<NS, MODE, 4, 4, false> (M, A, blocks, s, occ);
  case 1: return fast ? launch_stage_t<NS, MODE, 8, 4, true> (M, A, blocks, s, occ)
                      : launch_stage_t<NS, MODE, 8, 4, false> (M, A, blocks, s, occ);
  default: return fast ? launch_stage_t<NS, MODE, 8, 2, true> (M, A, blocks, s, occ)
                       : launch_stage_t<NS, MODE, 8, 2, false> (M, A, blocks, s, occ);
  }
}

template <int NS>
cudaError_t
launch_stage_ns (int mode, int cfg, const Model &M, const StageArgs &A, int blocks, cudaStream_t s, int *occ)
{
  switch (mode) {
  case M_DERIV: return launch_stage_c<NS, M_DERIV> (cfg, M, A, blocks, s, occ);
  case M_S1: return launch_stage_c<NS, M_S1> (cfg, M, A, blocks, s, occ);
  case M_S2: return launch_stage_c<NS, M_S2> (cfg, M, A, blocks, s, occ);
  case M_AMR2: return launch_stage_c<NS, M_AMR2> (cfg, M, A, blocks, s, occ);
  default: return cudaErrorInvalidValue;
  }
}

template <int NS, bool S2, int WY, int RPW, bool TREE>
cudaError_t
launch_fused_t (const Model &M, const FusedArgs &A, int blocks, cudaStream_t s, int *occ)
{
  const size_t sm = sizeof (double) * 2 * fused_buffer_doubles<NS, WY, RPW> (A.stage_eabs);
  cudaFuncSetAttribute (k_fused<NS, S2, WY, RPW, TREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
  if (occ) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor (occ, k_fused<NS, S2, WY, RPW, TREE>, 32 * WY, sm);
    return cudaGetLastError ();
  }
  k_fused<NS, S2, WY, RPW, TREE><<<blocks, 32 * WY, sm, s>>> (M, A);
  return cudaGetLastError ();
}

template <int NS, bool S2, bool TREE>
cudaError_t
launch_fused_c (int cfg, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s, int *occ)
{
  switch (cfg) {
  case 0: return launch_fused_t<NS, S2, 4, 4, TREE> (M, A, blocks, s, occ);
  case 1: return launch_fused_t<NS, S2, 8, 4, TREE> (M, A, blocks, s, occ);
  default: return launch_fused_t<NS, S2, 8, 2, TREE> (M, A, blocks, s, occ);
  }
}

template <int NS>
cudaError_t
launch_fused_ns (bool s2, bool tree, int cfg, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s,
                 int *occ)
{
  if (tree)
    return s2 ? launch_fused_c<NS, true, true> (cfg, M, A, blocks, s, occ)
              : launch_fused_c<NS, false, true> (cfg, M, A, blocks, s, occ);
  return s2 ? launch_fused_c<NS, true, false> (cfg, M, A, blocks, s, occ)
            : launch_fused_c<NS, false, false> (cfg, M, A, blocks, s, occ);
}

template <int NS>
cudaError_t
launch_vjp_ns (const Model &M, const VjpArgs &A, int blocks, size_t smem, cudaStream_t st, int *occ)
{
  if (occ) {
    cudaError_t e = cudaFuncSetAttribute (k_vjp<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor (occ, k_vjp<NS>, VjpTile<NS>::NT, smem);
  }
  k_vjp<NS><<<blocks, VjpTile<NS>::NT, smem, st>>> (M, A);
  return cudaGetLastError ();
}

// The split form of the VJP (faces, then reactions); with occ the two
// kernels' resident blocks per SM (occ[0] faces, occ[1] reactions).
template <int NS>
cudaError_t
launch_vjp_split_ns (const Model &M, const VjpArgs &A, int blocks_f, int blocks_r, size_t smem_r,
                     cudaStream_t st, int *occ)
{
  const size_t smem_f = sizeof (double) * VjpTileF::END;
  if (occ) {
    cudaError_t e = cudaFuncSetAttribute (k_vjp_faces<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_f);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor (&occ[0], k_vjp_faces<NS>, VjpTileF::NT, smem_f);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute (k_vjp_react<NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_r);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute (k_vjp_react<NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem_r);
    if (e != cudaSuccess) return e;
    int o1 = 0, o2 = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor (&o1, k_vjp_react<NS, false>, 256, smem_r);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor (&o2, k_vjp_react<NS, true>, 256, smem_r);
    occ[1] = o1 < o2 ? o1 : o2;
    return e;
  }
  bool generic = false;
  for (int r = 0; r < M.nreact; r++) generic = generic || M.r_nin[r] > 2;
  k_vjp_faces<NS><<<blocks_f, VjpTileF::NT, smem_f, st>>> (M, A);
  cudaError_t e = cudaGetLastError ();
  if (e != cudaSuccess) return e;
  if (generic) k_vjp_react<NS, true><<<blocks_r, 256, smem_r, st>>> (M, A);
  else k_vjp_react<NS, false><<<blocks_r, 256, smem_r, st>>> (M, A);
  return cudaGetLastError ();
}

template <int NS, bool S2, bool TREE>
cudaError_t
launch_march_t (const Model &M, const FusedArgs &A, int blocks, cudaStream_t s)
{
  const size_t sm = march_smem_bytes<NS> ();
  cudaFuncSetAttribute (k_march<NS, S2, TREE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) sm);
  k_march<NS, S2, TREE><<<blocks, 32 * MARCH_WPB, sm, s>>> (M, A);
  return cudaGetLastError ();
}

template <int NS>
cudaError_t
launch_march_ns (bool s2, bool tree, const Model &M, const FusedArgs &A, int blocks, cudaStream_t s)
{
  if (tree) return s2 ? launch_march_t<NS, true, true> (M, A, blocks, s) : launch_march_t<NS, false, true> (M, A, blocks, s);
  return s2 ? launch_march_t<NS, true, false> (M, A, blocks, s) : launch_march_t<NS, false, false> (M, A, blocks, s);
}

template cudaError_t launch_march_ns<ARCOS_NS> (bool, bool, const Model &, const FusedArgs &, int, cudaStream_t);
template cudaError_t launch_stage_ns<ARCOS_NS> (int, int, const Model &, const StageArgs &, int, cudaStream_t, int *);
template cudaError_t launch_fused_ns<ARCOS_NS> (bool, bool, int, const Model &, const FusedArgs &, int, cudaStream_t, int *);
template cudaError_t launch_vjp_ns<ARCOS_NS> (const Model &, const VjpArgs &, int, size_t, cudaStream_t, int *);
template cudaError_t launch_vjp_split_ns<ARCOS_NS> (const Model &, const VjpArgs &, int, int, size_t, cudaStream_t, int *);

}  // namespace arcos
