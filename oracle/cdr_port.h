/* ORACLE — test infrastructure only (CPU restatement of the arcos CDR density
 * update).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it; the product library never links it.
 *
 * Arrays use the reference rz_array layout (include/rz_array.h:11-22,
 * src/rz_array.c:23-96): r is the fastest index, two ghost cells on every
 * side in r and z, z stride nr+4, theta stride (nr+4)(nz+4); 2-D grids hold
 * one plane, 3-D grids hold ntheta+4 planes starting at theta = -2.
 */
#ifndef ORACLE_CDR_PORT_H
#define ORACLE_CDR_PORT_H

#define PORT_MAX_SPECIES 16
#define PORT_MAX_REACT 32
#define PORT_MAX_IN 4
#define PORT_MAX_OUT 6

/* Boundary numbering and masks of include/grid.h:14-31. */
#define PORT_BND_LEFT 0
#define PORT_BND_RIGHT 1
#define PORT_BND_BOTTOM 2
#define PORT_BND_TOP 3
#define PORT_MASK(b_) (1 << (b_))

typedef struct {
  int nin, nout;
  int input[PORT_MAX_IN];
  int output[PORT_MAX_OUT];
  double e_min, e_step, underflow, overflow;
  int steps;
  const double *values;       /* steps + 2 entries (the last repeats values[steps]) */
} port_reaction;

typedef struct {
  int no_species;
  double charge[PORT_MAX_SPECIES];
  double mass[PORT_MAX_SPECIES];
  double diffusion_coeff, nu_a, nu_d, nu_rt;
  int bnd_cond[4];            /* cdr_ext_bnd_cond[] signs (index RIGHT/BOTTOM/TOP) */
  double E_x, E_y, E_z;
  double z_cutoff;
  int max_ntheta;
  double dtheta;
  const double *dr, *dz;      /* per level, level 0 first */
  int nreact;
  port_reaction react[PORT_MAX_REACT];
  int per_plane;              /* 1: drift/diffusion on every theta plane */
  int zero_all;               /* 1: every grid's d_dens starts at zero (static trees) */
  int field_mode;             /* 0 zero, 1 fixed arrays, 2 host Poisson (root) */
  /* photoionization (src/photo.c:268-360), the entry ending the reactions
   * list (src/rt.c:38-47); terms in the order photo_calc visits them */
  int n_photo;
  double photo_A[8], photo_es[8];
  int photo_src, photo_e, photo_pi;
} port_model;

typedef struct port_grid port_grid;
struct port_grid {
  int r0, z0, r1, z1, ntheta, level, ext_bound;
  port_grid *parent, *next, *first_child;
  double *dens[PORT_MAX_SPECIES + 1];  /* dens[no_species] aliases eabs */
  double *d_dens[PORT_MAX_SPECIES];
  double *er, *ez, *etheta, *eabs, *charge;
  const double *fixed_er, *fixed_ez, *fixed_et;   /* field_mode 1 */
  int owns;                   /* arrays allocated by the port (RK2 intermediate) */
};

#endif
