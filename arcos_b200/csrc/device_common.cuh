// Device-side data structures shared by all kernels of the arcos CDR library.
//
// Storage: every grid ("patch") owns one block of device memory holding all its
// arrays.  Each array keeps the reference rz_array shape (src/rz_array.c:23-96:
// two ghost cells per side, r fastest, theta planes -2..ntheta+1 in 3-D) but
// its rows are padded to `pitch` doubles (a multiple of 4, so every row starts
// on a 32-byte sector and double2 accesses of even columns are aligned).
// Element (ir, iz, it) of an array, with ir/iz relative to the patch origin
// (interior 0..nr-1 / 0..nz-1) and it the theta plane, lives at
//     base + (ir + 2) + (iz + 2) * pitch + (it - theta0) * plane_stride.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define ARCOS_MAXS 16
#define ARCOS_MAXR 32
#define ARCOS_MAXIN 4
#define ARCOS_MAXOUT 6
#define ARCOS_MAXPLANES 68   // ntheta <= 64
#define ARCOS_MAX_PHOTO 8    // photoionization terms
#define ARCOS_MAXLEVELS 16   // refinement levels

namespace arcos {

// Array kinds inside a patch block (per storage set).
enum Kind { K_DENS = 0, K_DDENS = 1, K_ER = 2, K_EZ = 3, K_ETHETA = 4, K_EABS = 5, K_CHARGE = 6 };

struct PatchDesc {
  int nr, nz, ntheta, planes;   // planes = 1 (2-D) or ntheta + 4
  int r0, z0, level, ext_bound; // absolute origin at `level`, boundary mask (grid.h:22-31)
  int pitch, ns, theta0, parent;
  long long plane_stride;       // pitch * (nz + 4)
  long long asz;                // doubles per array (padded)
  double dr, dz;                // spacing at this level
  double *base;                 // start of this patch's arrays
  int fam;                      // family (independent grid tree) this patch belongs to
  int pad_;
  double *adj;                  // adjoint work arrays of this patch (same layout), or null

  // index of an array within the block: [set][dens s | d_dens s | er ez etheta eabs charge]
  __host__ __device__ inline int array_index (int set, int kind, int s) const {
    const int per_set = 2 * ns + 5;
    int k;
    if (kind == K_DENS) k = s;
    else if (kind == K_DDENS) k = ns + s;
    else k = 2 * ns + (kind - K_ER);
    return set * per_set + k;
  }
  __host__ __device__ inline double *arr (int set, int kind, int s = 0) const {
    return base + (long long) array_index (set, kind, s) * asz;
  }
  // offset of interior-relative (ir, iz) on plane `it` (theta index, -2..ntheta+1)
  __host__ __device__ inline long long off (int ir, int iz, int it) const {
    return (long long) (ir + 2) + (long long) (iz + 2) * pitch
           + (long long) (it - theta0) * plane_stride;
  }
};

// A tile of the stencil work list: columns [c0, c0 + width) and rows
// [zb, zb + zlen) of one theta plane of one patch.
struct WorkItem {
  int patch, plane, c0, width, zb, zlen;
};

// One node of a reaction table as the device uses it.  thr is the smallest
// |E| whose reference lookup (reaction.c:127-136) lands at or above this node;
// val/e1/slope reproduce reaction.c:137-142 with pow() evaluated on the host.
struct __align__ (16) TableNode {
  double val, e1, slope, thr;
};

struct Model {
  int ns, nreact;
  int mobile[ARCOS_MAXS];
  double charge[ARCOS_MAXS];
  double mass[ARCOS_MAXS];
  int r_nin[ARCOS_MAXR], r_nout[ARCOS_MAXR];
  int r_in[ARCOS_MAXR][ARCOS_MAXIN];
  int r_out[ARCOS_MAXR][ARCOS_MAXOUT];
  int r_steps[ARCOS_MAXR];
  // accumulation program of each reaction: the d_dens updates of react_apply
  // (reaction.c:147-155) in order, species with zero charge dropped
  int r_nops[ARCOS_MAXR];
  // the same folded per species (fast form): net count of +rate updates and
  // the number of times each species is an input
  signed char r_coef[ARCOS_MAXR][8];
  signed char r_in_count[ARCOS_MAXR][8];
  signed char r_op_sp[ARCOS_MAXR][ARCOS_MAXIN + ARCOS_MAXOUT];
  signed char r_op_neg[ARCOS_MAXR][ARCOS_MAXIN + ARCOS_MAXOUT];
  int r_node_off[ARCOS_MAXR];     // first node of the reaction in the node array
  double r_e_min[ARCOS_MAXR], r_e_step[ARCOS_MAXR];
  double r_under[ARCOS_MAXR], r_over[ARCOS_MAXR];
  float r_inv_step_f[ARCOS_MAXR];   // 1/e_step for the single-precision position estimate
  double diffusion_coeff, nu_a, nu_d, nu_rt, warn_min_timestep, z_cutoff, dtheta;
  int bnd_sign[4];                // cdr_ext_bnd_cond[] (cdr.c:79-84), index BND_*
  int per_plane;
  int pad_;
};

// Device scalar state of a run (time step, CFL maxima, error flags).
struct DevState {
  double h_attempt;               // the attempted step (cdr_rk2's h argument)
  double h;                       // the step of the current RK2 step
  unsigned long long dmax_key[2]; // max of mobile densities (ordered keys), ping-pong
  unsigned long long emax_key[2][3]; // per storage set: max |er|, |ez|, |etheta| (root)
  int step;                       // number of completed steps
  int small_dt_count;             // steps below warn_min_timestep
  int error;                      // sticky ARCOS_ERR_* bits (1 << code)
  unsigned int done_blocks;       // last-block detection in the stage-2 kernel
  unsigned int neg[2];            // per step (ping-pong): the state may hold negative densities
  double courant_const[4];        // dr_min, dz_min, rdtheta_min, is_3d
  int dt_cap;                     // capacity of the dt log
  int counted_step;               // step whose small h was last counted (-1: none)
  int small_dt_step;              // step whose h was the sixth small one
  int pad_;
  double *dt_log;                 // steps taken
};

// Order-preserving map of doubles to unsigned keys (for atomicMax).
__host__ __device__ inline unsigned long long dkey (double x) {
  unsigned long long b;
#ifdef __CUDA_ARCH__
  b = (unsigned long long) __double_as_longlong (x);
#else
  union { double d; unsigned long long u; } cv; cv.d = x; b = cv.u;
#endif
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ inline double dkey_inv (unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ULL) ? (k & 0x7fffffffffffffffULL) : ~k;
#ifdef __CUDA_ARCH__
  return __longlong_as_double ((long long) b);
#else
  union { double d; unsigned long long u; } cv; cv.u = b; return cv.d;
#endif
}

}  // namespace arcos
