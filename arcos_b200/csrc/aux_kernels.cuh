// Streaming and ghost-fill kernels of the arcos CDR library: everything on the
// path except the stencil stage kernel.  Every kernel takes a list of patches
// (blockIdx.y selects the patch) so one launch covers a whole grid family, or a
// single patch for the per-patch launch mode.
#pragma once
#include "device_common.cuh"
#include "stage_kernel.cuh"

namespace arcos {

// ---- host transfers: rows of w doubles, packed (the host rz_array layout)
// <-> rows of `pitch` doubles (the device layout).  A host<->device copy moves
// the packed image linearly and one of these kernels repitches it on the
// device: a pitched DMA of ~4 KB rows runs well below the link's rate. ----
__global__ void
k_unpack_rows (const double *__restrict__ src, double *__restrict__ dst, int w, long long rows, int pitch)
{
  for (long long r = blockIdx.x; r < rows; r += gridDim.x)
    for (int x = threadIdx.x; x < w; x += blockDim.x) dst[r * pitch + x] = src[r * w + x];
}

__global__ void
k_pack_rows (const double *__restrict__ src, double *__restrict__ dst, int w, long long rows, int pitch)
{
  for (long long r = blockIdx.x; r < rows; r += gridDim.x)
    for (int x = threadIdx.x; x < w; x += blockDim.x) dst[r * w + x] = src[r * pitch + x];
}

// ---- A13: cdr_nonegative (cdr.c:703-721): dens = MYMAX(0, dens) over the
// whole arrays (ghosts included) of every species. ----
__global__ void
k_nonneg (const PatchDesc *pd, const int *plist, int set)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  double *a = P.arr (set, K_DENS, 0);
  const long long n = P.asz * P.ns;       // the species arrays are contiguous
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long) gridDim.x * blockDim.x)
    a[i] = clamp0 (a[i]);
}

// The same over a flat list of chunks: chunk b is
// elements [start, start + chunk) of the species arrays of patch `patch`, so a
// tree of patches of any sizes is one launch with every block busy.
struct Chunk {
  int patch, start;
};

__global__ void
k_nonneg_chunks (const PatchDesc *pd, const Chunk *chunks, int set, int chunk)
{
  const Chunk ch = chunks[blockIdx.x];
  const PatchDesc P = pd[ch.patch];
  double *a = P.arr (set, K_DENS, 0);
  const long long n = P.asz * P.ns;
  const long long end = (long long) ch.start + chunk < n ? (long long) ch.start + chunk : n;
  // four independent loads per thread in flight; a value changes only when it
  // is below zero (clamp0 keeps NaN and -0), so only those are written back
  for (long long i0 = ch.start + threadIdx.x; i0 < end; i0 += 4 * blockDim.x) {
    double v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const long long i = i0 + (long long) k * blockDim.x;
      v[k] = i < end ? a[i] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const long long i = i0 + (long long) k * blockDim.x;
      if (i < end && 0 > v[k]) a[i] = 0.0;
    }
  }
}

// ---- A10: cdr_update (cdr.c:1091-1097): dens[dst] = dens[src] + h d_dens[src] ----
__global__ void
k_update (const PatchDesc *pd, const int *plist, int src, int dst, const DevState *st,
          double h_host, int use_dev_h)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  const double h = use_dev_h ? st[P.fam].h : h_host;
  const double *n = P.arr (src, K_DENS, 0), *d = P.arr (src, K_DDENS, 0);
  double *o = P.arr (dst, K_DENS, 0);
  const long long len = P.asz * P.ns;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (long long) gridDim.x * blockDim.x)
    o[i] = n[i] + h * d[i];
}

// ---- A11: cdr_rk2_update (cdr.c:1125-1132):
// dens[0] = dens[0] + 0.5 h d_dens[0] + 0.5 h d_dens[1] ----
__global__ void
k_rk2_update (const PatchDesc *pd, const int *plist, const DevState *st, double h_host,
              int use_dev_h)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  const double h = use_dev_h ? st[P.fam].h : h_host;
  double *n = P.arr (0, K_DENS, 0);
  const double *d1 = P.arr (0, K_DDENS, 0), *d2 = P.arr (1, K_DDENS, 0);
  const long long len = P.asz * P.ns;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (long long) gridDim.x * blockDim.x)
    n[i] = n[i] + 0.5 * h * d1[i] + 0.5 * h * d2[i];
}

// ---- A14: cdr_calc_charge (cdr.c:361-389): charge = sum_s (n_s q_s)/ntheta over
// the 2-ghost extent of the real planes (ghost planes set to 0). ----
__global__ void
k_charge (const Model M, const PatchDesc *pd, const int *plist, int set)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  double *ch = P.arr (set, K_CHARGE);
  const long long len = P.asz;
  const int nr4 = P.nr + 4;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (long long) gridDim.x * blockDim.x) {
    const long long pl = i / P.plane_stride;
    const int it = (int) pl + P.theta0;
    const int col = (int) ((i % P.plane_stride) % P.pitch);
    double q = 0.0;
    if (it >= 0 && it < P.ntheta && col < nr4) {
      for (int s = 0; s < P.ns; s++)
        q += (P.arr (set, K_DENS, s)[i] * M.charge[s]) / P.ntheta;
    }
    ch[i] = q;
  }
}

// charge of the RK2 intermediate state max(0, n0) + h d0 on the interior (the
// charge cdr_update computes for the field solve of stage 2; the fused stage
// kernels never store n*).
__global__ void
k_charge_star (const Model M, const PatchDesc *pd, const int *plist, int src,
               const DevState *st)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  const double h = st[P.fam].h;
  double *ch = P.arr (1, K_CHARGE);
  const long long len = P.asz;
  const int nr4 = P.nr + 4;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (long long) gridDim.x * blockDim.x) {
    const long long pl = i / P.plane_stride;
    const int it = (int) pl + P.theta0;
    const long long rem = i % P.plane_stride;
    const int col = (int) (rem % P.pitch) - 2, row = (int) (rem / P.pitch) - 2;
    double q = 0.0;
    if (it >= 0 && it < P.ntheta && col >= 0 && col < P.nr && row >= 0 && row < P.nz) {
      for (int s = 0; s < P.ns; s++) {
        const double v = clamp0 (P.arr (src, K_DENS, s)[i]) + h * P.arr (0, K_DDENS, s)[i];
        q += (v * M.charge[s]) / P.ntheta;
      }
    }
    if (col + 2 < nr4) ch[i] = q;
  }
}

// ---- A16: cdr_set_ext_bnd (cdr.c:726-768) with set_axis_bnd (:798-824) and
// rz_copy_bnd / rz_set_bnd (rz_array.c:196-235).  The reference copies side by
// side over the whole array: axis, right, bottom, top.  The z sides copy the r
// sides' ghost columns (the corners), so a z-side thread takes the value its
// source cell has once the r sides are done (p1, reading only interior cells);
// an r-side thread leaves a corner to the z side when that side is external
// (its value would be overwritten), and otherwise reads a ghost row that no
// side of this call writes.  So every write is independent and one launch of
// (patch, species, slice) blocks does the lot.  The two r sides (and the two
// z sides) touch disjoint cells, since a patch has at least 2 x 2 cells. ----
__global__ void
k_ext_bnd (const Model M, const PatchDesc *pd, const int *plist, int set)
{
  const PatchDesc P = pd[plist[blockIdx.x]];
  const int nr = P.nr, nz = P.nz, nt = P.ntheta, eb = P.ext_bound;
  const int s = blockIdx.y;
  if (s >= P.ns || eb == 0) return;
  double *a = P.arr (set, K_DENS, s);
  const double sg1 = (double) M.bnd_sign[1], sg2 = (double) M.bnd_sign[2], sg3 = (double) M.bnd_sign[3];
  const int rows = nz + 4, cols = nr + 4;
  const int nrs = (eb & 3) ? nt * rows : 0;           // r-side items (plane, row)
  const int nzs = (eb & 12) ? nt * cols : 0;          // z-side items (plane, column)
  // cell (c, r) of plane it, r an interior row, after the r sides
  auto p1 = [&] (int c, int r, int it) -> double {
    if (c < 0 && (eb & 1)) return a[P.off (-1 - c, r, (it + nt / 2) % nt)];
    if (c >= nr && (eb & 2)) return sg1 * a[P.off (2 * nr - 1 - c, r, it)];
    return a[P.off (c, r, it)];
  };
  for (int i = blockIdx.z * blockDim.x + threadIdx.x; i < nrs + nzs; i += gridDim.z * blockDim.x) {
    if (i < nrs) {
      const int it = i / rows, iz = i - it * rows - 2;
      if ((iz < 0 && (eb & 4)) || (iz >= nz && (eb & 8))) continue;
      if (eb & 1) {                                   // axis: the opposite plane
        const int it2 = (it + nt / 2) % nt;
        const double v0 = a[P.off (0, iz, it2)], v1 = a[P.off (1, iz, it2)];
        a[P.off (-1, iz, it)] = v0;
        a[P.off (-2, iz, it)] = v1;
      }
      if (eb & 2) {                                   // r = r1
        const double v0 = a[P.off (nr - 1, iz, it)], v1 = a[P.off (nr - 2, iz, it)];
        a[P.off (nr, iz, it)] = sg1 * v0;
        a[P.off (nr + 1, iz, it)] = sg1 * v1;
      }
    } else {
      const int j = i - nrs, it = j / cols, ir = j - it * cols - 2;
      if (eb & 4) {                                   // z = z0
        const double v0 = p1 (ir, 0, it), v1 = p1 (ir, 1, it);
        a[P.off (ir, -1, it)] = sg2 * v0;
        a[P.off (ir, -2, it)] = sg2 * v1;
      }
      if (eb & 8) {                                   // z = z1
        const double v0 = p1 (ir, nz - 1, it), v1 = p1 (ir, nz - 2, it);
        a[P.off (ir, nz, it)] = sg3 * v0;
        a[P.off (ir, nz + 1, it)] = sg3 * v1;
      }
    }
  }
}

// ---- A16: rz_set_periodic (rz_array.c:153-174) for the arrays cdr_set_periodic
// names (cdr.c:288-310): planes nt-1, nt-2, 0, 1 -> -1, -2, nt, nt+1.
// `what` bit 0: dens and d_dens, bit 1: etheta, er, ez. ----
__global__ void
k_periodic (const PatchDesc *pd, const int *plist, int set, int what)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  const int nt = P.ntheta;
  if (nt == 1) return;
  const long long ps = P.plane_stride;
  const int narr = ((what & 1) ? 2 * P.ns : 0) + ((what & 2) ? 3 : 0);
  const long long total = (long long) narr * 4 * ps;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long) gridDim.x * blockDim.x) {
    const long long e = i % ps;
    const int cp = (int) ((i / ps) % 4);
    int ai = (int) (i / ps / 4);
    double *a;
    if (what & 1) {
      if (ai < P.ns) a = P.arr (set, K_DENS, ai);
      else if (ai < 2 * P.ns) a = P.arr (set, K_DDENS, ai - P.ns);
      else { ai -= 2 * P.ns; a = P.arr (set, ai == 0 ? K_ETHETA : (ai == 1 ? K_ER : K_EZ)); }
    } else {
      a = P.arr (set, ai == 0 ? K_ETHETA : (ai == 1 ? K_ER : K_EZ));
    }
    const int from[4] = {nt - 1, nt - 2, 0, 1}, to[4] = {-1, -2, nt, nt + 1};
    a[(long long) (to[cp] - P.theta0) * ps + e] = a[(long long) (from[cp] - P.theta0) * ps + e];
  }
}

// ---- A17: restrict_from (cdr.c:2050-2078) for every child of one level:
// parent(ir, iz) = 0.25 * sum_{2x2} r_c n_c / r_p.  Item i of a child runs over
// its covered parent cells, ir fastest, then iz, plane, species. ----
struct RestrictGeom {
  int ir0, iz0, wr, wz, total;
};

__device__ __forceinline__ RestrictGeom
restrict_geom (const PatchDesc &C, int ntheta_parent)
{
  const int cr0 = C.r0, cz0 = C.z0, cr1 = C.r0 + C.nr, cz1 = C.z0 + C.nz;
  RestrictGeom G;
  G.ir0 = (cr0 >> 1) + (cr0 % 2);
  G.iz0 = (cz0 >> 1) + (cz0 % 2);
  G.wr = (cr1 >> 1) - G.ir0;
  G.wz = (cz1 >> 1) - G.iz0;
  // 32-bit indices (a child's covered cells x planes x species stay far below 2^31)
  G.total = (G.wr <= 0 || G.wz <= 0) ? 0 : G.wr * G.wz * ntheta_parent * C.ns;
  return G;
}

// the four child values of item i, in the order the sum takes them
struct RestrictLoad {
  double v[4];
  long long dst;
  int ir, s;
};

__device__ __forceinline__ RestrictLoad
restrict_load (const PatchDesc &C, const PatchDesc &Pp, const RestrictGeom &G, int i, int set)
{
  RestrictLoad L;
  const int q = i / G.wr, ir = G.ir0 + (i - q * G.wr);
  const int q2 = q / G.wz, iz = G.iz0 + (q - q2 * G.wz);
  const int s = q2 / Pp.ntheta, it = q2 - s * Pp.ntheta;
  const double *cn = C.arr (set, K_DENS, s);
  const long long o = C.off ((ir << 1) - C.r0, (iz << 1) - C.z0, it);
  L.v[0] = cn[o];
  L.v[1] = cn[o + C.pitch];
  L.v[2] = cn[o + 1];
  L.v[3] = cn[o + 1 + C.pitch];
  L.dst = Pp.off (ir - Pp.r0, iz - Pp.z0, it);
  L.ir = ir;
  L.s = s;
  return L;
}

__device__ __forceinline__ void
restrict_store (const PatchDesc &C, const PatchDesc &Pp, const RestrictLoad &L, int set)
{
  const double ra = ((double) (L.ir << 1) + 0.5) * C.dr, rb = ((double) ((L.ir << 1) + 1) + 0.5) * C.dr;
  double sum = 0;
  sum += ra * L.v[0];
  sum += ra * L.v[1];
  sum += rb * L.v[2];
  sum += rb * L.v[3];
  Pp.arr (set, K_DENS, L.s)[L.dst] = 0.25 * sum / (((double) L.ir + 0.5) * Pp.dr);
}

__global__ void
k_restrict (const PatchDesc *pd, const int *children, int set)
{
  const PatchDesc C = pd[children[blockIdx.y]];
  const PatchDesc Pp = pd[C.parent];
  const RestrictGeom G = restrict_geom (C, Pp.ntheta);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.total; i += gridDim.x * blockDim.x)
    restrict_store (C, Pp, restrict_load (C, Pp, G, i, set), set);
}

// A block of flat work of a ghost phase over one level of a tree: items
// [first, first + per block) of child `child` (parent `parent`, ghost strip
// `strip` for the interpolation).  Built once per tree, so a level of patches
// of any sizes is one launch with every block busy.
struct WorkBlk {
  int child, parent, strip, first;
};

constexpr int RESTRICT_PER_THREAD = 4;
constexpr int RESTRICT_THREADS = 256;
constexpr int RESTRICT_PER_BLOCK = RESTRICT_PER_THREAD * RESTRICT_THREADS;

__global__ void __launch_bounds__ (RESTRICT_THREADS)
k_restrict_blk (const PatchDesc *pd, const WorkBlk *wb, int set)
{
  const WorkBlk W = wb[blockIdx.x];
  const PatchDesc C = pd[W.child];
  const PatchDesc Pp = pd[W.parent];
  const RestrictGeom G = restrict_geom (C, Pp.ntheta);
  const int end = min (G.total, W.first + RESTRICT_PER_BLOCK);
  RestrictLoad L[RESTRICT_PER_THREAD];
#pragma unroll
  for (int k = 0; k < RESTRICT_PER_THREAD; k++) {
    const int i = W.first + k * RESTRICT_THREADS + threadIdx.x;
    if (i < end) L[k] = restrict_load (C, Pp, G, i, set);
  }
#pragma unroll
  for (int k = 0; k < RESTRICT_PER_THREAD; k++) {
    const int i = W.first + k * RESTRICT_THREADS + threadIdx.x;
    if (i < end) restrict_store (C, Pp, L[k], set);
  }
}

// The 9-point quadratic table laid out as interpol2.c:260-280 has it: 57
// numbers, because the line "0.25, 0, -0.25" of the rz row appears twice.
// interpol_set_coeffs (interpol2.c:173-185) reads 9 numbers per coefficient
// (1, z, r, z^2, rz, r^2; column i*3+j, i over r, j over z), so the rz and
// r^2 rows it uses are shifted.  Kept exactly as the reference reads it.
__constant__ double c_quad[57] = {
  -0.1111111111111111,  0.2222222222222222, -0.1111111111111111,
   0.2222222222222222,  0.5555555555555556,  0.2222222222222222,
  -0.1111111111111111,  0.2222222222222222, -0.1111111111111111,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667,  0,                   0.1666666666666667,
  -0.1666666666666667, -0.1666666666666667, -0.1666666666666667,
   0,                   0,                   0,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.1666666666666667, -0.3333333333333333,  0.1666666666666667,
   0.25,                0,                  -0.25,
   0.25,                0,                  -0.25,
   0,                   0,                   0,
  -0.25,                0,                   0.25,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667,
  -0.3333333333333333, -0.3333333333333333, -0.3333333333333333,
   0.1666666666666667,  0.1666666666666667,  0.1666666666666667
};

// ---- A17: child ghost strips from the parent (cdr_set_bnd cdr.c:1888-1948 ->
// map_grid / map_interpol / interpol_inner, mapper.c:41-97,178-312, with the
// quadratic-masses interpolation of interpol2.c:116-241).  A strip is a
// rectangle [sr0,sr1) x [sz0,sz1) of child cells; each fine cell takes the
// stencil centred on the coarse cell (ir>>1, iz>>1) when that coarse cell is
// inside the range map_interpol loops over. ----
struct StripDesc {
  int child, sr0, sz0, sr1, sz1;
};

// The fine cells a strip writes: [fr0, fr0 + wr) x [fz0, fz0 + wz) over planes
// and species, ir fastest (total = 0 when the strip misses the parent).
struct InterpGeom {
  int fr0, fz0, wr, wz, total;
};

__host__ __device__ inline int imax_ (int a, int b) { return a > b ? a : b; }
__host__ __device__ inline int imin_ (int a, int b) { return a < b ? a : b; }

__host__ __device__ inline InterpGeom
interp_geom (const StripDesc &S, const PatchDesc &C, const PatchDesc &Pp)
{
  InterpGeom G;
  G.total = 0;
  G.fr0 = G.fz0 = G.wr = G.wz = 0;
  const int pr0 = Pp.r0, pz0 = Pp.z0, pr1 = Pp.r0 + Pp.nr, pz1 = Pp.z0 + Pp.nz;
  // grid_overlap (parent, strip, s_buff = 1, t_buff = 0), grid.c:145-198
  const int left = imax_ (S.sr0, (pr0 - 1) << 1), right = imin_ (S.sr1, (pr1 + 1) << 1);
  const int bottom = imax_ (S.sz0, (pz0 - 1) << 1), top = imin_ (S.sz1, (pz1 + 1) << 1);
  if (left >= right || bottom >= top) return G;
  // map_interpol coarse range (mapper.c:199-210)
  const int r0c = imax_ (left >> 1, pr0 - 1), r1c = imin_ (((right - 1) >> 1) + 1, pr1 + 1);
  const int z0c = imax_ (bottom >> 1, pz0 - 1), z1c = imin_ (((top - 1) >> 1) + 1, pz1 + 1);
  // fine cells written (interpol_inner, mapper.c:296-299)
  const int fr0 = imax_ (S.sr0 - 2, r0c << 1), fr1 = imin_ (S.sr1 + 2, r1c << 1);
  const int fz0 = imax_ (S.sz0 - 2, z0c << 1), fz1 = imin_ (S.sz1 + 2, z1c << 1);
  if (fr1 <= fr0 || fz1 <= fz0) return G;
  G.fr0 = fr0; G.fz0 = fz0; G.wr = fr1 - fr0; G.wz = fz1 - fz0;
  G.total = G.wr * G.wz * C.ntheta * C.ns;        // a strip's cells: far below 2^31
  return G;
}

// FAST (the division-free step): the coefficients are scaled by reciprocal
// powers of the parent's spacing instead of divided by the powers
// (interpol_set_coeffs divides twice per coefficient, interpol2.c:180); the
// result differs in the last bits only.
template <bool FAST>
__device__ __forceinline__ void
interp_item (const PatchDesc &C, const PatchDesc &Pp, const InterpGeom &G, int i, int set)
{
  const int q = i / G.wr, ir = G.fr0 + (i - q * G.wr);
  const int q2 = q / G.wz, iz = G.fz0 + (q - q2 * G.wz);
  const int s = q2 / C.ntheta, it = q2 - s * C.ntheta;
  const int pr = ir >> 1, pz = iz >> 1;
  const int pr0 = Pp.r0, pz0 = Pp.z0;
  // stay inside the ghost extents of child and parent
  if (ir - C.r0 < -2 || ir - C.r0 >= C.nr + 2 || iz - C.z0 < -2 || iz - C.z0 >= C.nz + 2) return;
  if (pr - 1 - pr0 < -2 || pr + 1 - pr0 >= Pp.nr + 2 || pz - 1 - pz0 < -2 || pz + 1 - pz0 >= Pp.nz + 2) return;
  const double Lr = Pp.dr, Lz = Pp.dz;
  const double *pn = Pp.arr (set, K_DENS, s);
  // interpol_set_stencil_at (interpol2.c:116-155)
  double st[9];
  const long long pb = Pp.off (pr - 1 - pr0, pz - 1 - pz0, it);
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) st[a * 3 + b] = pn[pb + a + (long long) b * Pp.pitch];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double r = ((double) (pr + a - 1) + 0.5) * Lr;
#pragma unroll
    for (int b = 0; b < 3; b++) st[a * 3 + b] = r * st[a * 3 + b];
  }
  // interpol_set_coeffs (interpol2.c:161-186)
  double cf[6], Lrn[4], Lzn[4];
  int pindx = 0, mindx = 0;
  if (FAST) {
    Lrn[0] = 1.0; Lzn[0] = 1.0;
    Lrn[1] = 1.0 / Lr; Lzn[1] = 1.0 / Lz;
    Lrn[2] = Lrn[1] * Lrn[1]; Lzn[2] = Lzn[1] * Lzn[1];
#pragma unroll
    for (int ip = 0; ip < 3; ip++)
#pragma unroll
      for (int n = 0; n <= ip; n++) {
        double sum = 0;
#pragma unroll
        for (int j = 0; j < 9; j++) sum = __fma_rn (c_quad[mindx + j], st[j], sum);
        mindx += 9;
        cf[pindx++] = sum * (Lrn[n] * Lzn[ip - n]);
      }
  } else {
    Lrn[0] = 1.0; Lzn[0] = 1.0;
#pragma unroll
    for (int ip = 0; ip < 3; ip++) {
      Lrn[ip + 1] = Lrn[ip] * Lr;
      Lzn[ip + 1] = Lzn[ip] * Lz;
#pragma unroll
      for (int n = 0; n <= ip; n++) {
        double sum = 0;
#pragma unroll
        for (int j = 0; j < 9; j++) sum += c_quad[mindx++] * st[j];
        cf[pindx++] = sum / Lrn[n] / Lzn[ip - n];
      }
    }
  }
  // interpol_apply + gen_apply (interpol2.c:190-241), masses: divide by r
  const double r = ((double) ir + 0.5) * C.dr, z = ((double) iz + 0.5) * C.dz;
  const double dr_ = r - ((double) pr + 0.5) * Lr, dz_ = z - ((double) pz + 0.5) * Lz;
  double res;
  if (dr_ == dz_)
    res = cf[0] + dr_ * (cf[1] + cf[2] + dr_ * (cf[3] + cf[4] + cf[5]));
  else
    res = cf[0] + dz_ * (cf[1] + dz_ * cf[3]) + dr_ * (cf[2] + dz_ * cf[4] + dr_ * cf[5]);
  C.arr (set, K_DENS, s)[C.off (ir - C.r0, iz - C.z0, it)] = res / r;
}

template <bool FAST>
__global__ void
k_interp (const PatchDesc *pd, const StripDesc *strips, int set)
{
  const StripDesc S = strips[blockIdx.y];
  const PatchDesc C = pd[S.child];
  const PatchDesc Pp = pd[C.parent];
  const InterpGeom G = interp_geom (S, C, Pp);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < G.total; i += gridDim.x * blockDim.x)
    interp_item<FAST> (C, Pp, G, i, set);
}

constexpr int INTERP_THREADS = 256;
constexpr int INTERP_PER_BLOCK = INTERP_THREADS;

// The same over a flat list of work blocks (one item per thread).
template <bool FAST>
__global__ void __launch_bounds__ (INTERP_THREADS)
k_interp_blk (const PatchDesc *pd, const StripDesc *strips, const WorkBlk *wb, int set)
{
  const WorkBlk W = wb[blockIdx.x];
  const StripDesc S = strips[W.strip];
  const PatchDesc C = pd[W.child];
  const PatchDesc Pp = pd[W.parent];
  const InterpGeom G = interp_geom (S, C, Pp);
  const int i = W.first + threadIdx.x;
  if (i < G.total) interp_item<FAST> (C, Pp, G, i, set);
}

// ---- A17: sibling matching (match_grids, cdr.c:1808-1882), as a gather
// resolved on the host into (destination, source) element pairs of the
// density arrays of one storage set (offsets from the pool base).  Two phases so that
// every read sees the values from before the matching, as the reference's
// copies see them once the chains are resolved. ----
__global__ void
k_match_gather (const double *base, const long long *src, int n, double *tmp)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    tmp[i] = base[src[i]];
}
__global__ void
k_match_scatter (double *base, const long long *dst, int n, const double *tmp)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    base[dst[i]] = tmp[i];
}

// ---- A15: cdr_add_ext_field (cdr.c:595-625) over the full extent of every
// plane; the per-plane values of e0_r / e0_theta (cstream.c:435-455) are
// evaluated on the host.  Also counts non-zero etheta values (after the add). ----
__global__ void
k_add_ext (const PatchDesc *pd, const int *plist, int set, const double *ext_r,
           const double *ext_t, const double *ext_z, int *etz)
{
  const int p = plist[blockIdx.y];
  const PatchDesc P = pd[p];
  double *er = P.arr (set, K_ER), *ez = P.arr (set, K_EZ), *et = P.arr (set, K_ETHETA);
  const long long len = P.asz;
  const int nr4 = P.nr + 4;
  int nz_count = 0;
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (long long) gridDim.x * blockDim.x) {
    const int pl = (int) (i / P.plane_stride);
    const int col = (int) ((i % P.plane_stride) % P.pitch);
    if (pl >= P.planes || col >= nr4) continue;
    const int fam = P.fam;
    er[i] += ext_r[fam * ARCOS_MAXPLANES + pl];
    ez[i] += ext_z[fam];
    et[i] += ext_t[fam * ARCOS_MAXPLANES + pl];
    if (et[i] != 0.0) nz_count++;
  }
  if (nz_count) atomicAdd (etz + p * 2 + set, nz_count);
}

// ---- A15: cdr_calc_eabs (cdr.c:668-695) on the interior of the real planes,
// plus the maxima of |er|, |ez|, |etheta| over the root grid that cdr_courant
// takes (cdr.c:998-1005). ----
__global__ void
k_eabs (const PatchDesc *pd, const int *plist, int set, DevState *st)
{
  const int p = plist[blockIdx.y];
  const PatchDesc P = pd[p];
  const double *er = P.arr (set, K_ER), *ez = P.arr (set, K_EZ), *et = P.arr (set, K_ETHETA);
  double *ea = P.arr (set, K_EABS);
  const long long total = (long long) P.nr * P.nz * P.ntheta;
  unsigned long long km[3] = {0, 0, 0};
  for (long long i = (long long) blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long) gridDim.x * blockDim.x) {
    const int ir = (int) (i % P.nr), iz = (int) ((i / P.nr) % P.nz), it = (int) (i / P.nr / P.nz);
    const long long o = P.off (ir, iz, it);
    const double a = 0.5 * (er[o] + er[P.off (ir - 1, iz, it)]);
    const double b = 0.5 * (ez[o] + ez[P.off (ir, iz - 1, it)]);
    double c = 0;
    if (P.ntheta != 1) c = 0.5 * (et[o] + et[P.off (ir, iz, it - 1)]);
    ea[o] = sqrt (a * a + b * b + c * c);
    if (P.level == 0) {
      const double v[3] = {fabs (er[o]), fabs (ez[o]), fabs (et[o])};
      for (int k = 0; k < 3; k++)
        if (v[k] == v[k]) { const unsigned long long kk = dkey (v[k]); km[k] = kk > km[k] ? kk : km[k]; }
    }
  }
  if (P.level == 0) {
    for (int k = 0; k < 3; k++) {
      unsigned long long x = km[k];
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync (0xffffffffu, x, o);
        x = y > x ? y : x;
      }
      if ((threadIdx.x & 31) == 0 && x) atomicMax (&st[P.fam].emax_key[set][k], x);
    }
  }
}

// ---- the maximum of the mobile densities over the root's interior, clamped as
// after cdr_nonegative (cdr.c:1007-1012), into dmax_key[slot] ----
__global__ void
k_dmax (const Model M, const PatchDesc *pd, const int *plist, int set, DevState *st, int slot_rel)
{
  const PatchDesc P = pd[plist[blockIdx.y]];
  if (P.level != 0) return;
  const int nr = P.nr, nz = P.nz, ns = P.ns, rows = nz * P.ntheta;
  const long long asz = P.asz;                 // the species arrays of a set are consecutive
  const double *d0 = P.arr (set, K_DENS, 0);
  // max over the clamped values, -0 taken as +0 (the ordered keys put +0
  // above -0) and NaN never greater; -1 while nothing was seen
  double vm = -1.0;
  // blocks over the rows (z, theta), threads along r: no division per cell
#pragma unroll 2
  for (int j = blockIdx.x; j < rows; j += gridDim.x) {
    const int it = j / nz, iz = j - it * nz;
    const double *row = d0 + P.off (0, iz, it);
    for (int ir = threadIdx.x; ir < nr; ir += blockDim.x)
      for (int s = 0; s < ns; s++) {
        if (!M.mobile[s]) continue;
        const double v = clamp0 (row[(long long) s * asz + ir]) + 0.0;
        vm = v > vm ? v : vm;
      }
  }
  unsigned long long km = vm >= 0.0 ? dkey (vm) : 0ULL;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync (0xffffffffu, km, o);
    km = y > km ? y : km;
  }
  // one atomic per block: the warps' maxima meet in shared memory first
  __shared__ unsigned long long wmax[32];
  const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) wmax[w] = km;
  __syncthreads ();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nw; k++) km = wmax[k] > km ? wmax[k] : km;
    DevState *s = st + P.fam;
    if (km) atomicMax (&s->dmax_key[(s->step + slot_rel) & 1], km);
  }
}

// Starts a step of every family: h from the reduced maxima (cfl_step), and
// resets the slot the coming stage-2 kernel reduces into.
__global__ void
k_cfl (const Model M, DevState *st, int nfam, int eset)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfam) return;
  DevState *s = st + f;
  const int k = s->step;
  s->dmax_key[(k + 1) & 1] = dkey (-1.0);
  cfl_step (s, M, k & 1, eset, k);
}

// Resets the max-density slot (step + slot_rel) of every family.
__global__ void
k_reset_dmax (DevState *st, int nfam, int slot_rel)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < nfam) st[f].dmax_key[(st[f].step + slot_rel) & 1] = dkey (-1.0);
}

// Start of a field-solve step, stream-ordered: the current dmax slot is
// reset and the state counts as unchecked for the stage-1 clamp.
__global__ void
k_run_reset (DevState *st, int nfam)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nfam) return;
  st[f].dmax_key[st[f].step & 1] = dkey (-1.0);
  st[f].neg[st[f].step & 1] = 1u;
  st[f].neg[(st[f].step + 1) & 1] = 0u;
}

// Before a set's field is post-processed: its E_theta counters and field
// maxima start over.
__global__ void
k_field_reset (int *etz, int np, int set, DevState *st, int nfam)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < np) etz[i * 2 + set] = 0;
  if (i < nfam)
    for (int k = 0; k < 3; k++) st[i].emax_key[set][k] = dkey (-1.0);
}

// Ends a step of every family whose stage-2 kernel did not fold the CFL.
__global__ void
k_step_end (DevState *st, int nfam)
{
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < nfam) st[f].step += 1;
}

}  // namespace arcos
