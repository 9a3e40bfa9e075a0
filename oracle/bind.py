"""ORACLE — test infrastructure only.  ctypes bindings for the two CPU oracles:

* ``PortTree`` drives oracle/liboracle_port.so, the CPU restatement
  (oracle/cdr_port.c);
* ``RefTree`` drives oracle/_ref/libarcos_ref.so, the reference's own C sources
  plus the restated Fortran kernel (oracle/Makefile, oracle/ref_harness.c).

Both take the product's host-side descriptions (arcos_b200.model / grids) so a
test can build the same problem three times: port, reference, device.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile
from typing import List, Optional, Sequence

import numpy as np

from arcos_b200.grids import GridSpec
from arcos_b200.model import KineticModel, Params
from arcos_b200.react_table import write_react_table

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle_port.so")
REF_SO = os.path.join(HERE, "_ref", "libarcos_ref.so")
REF_OMP_SO = os.path.join(HERE, "_ref", "libarcos_ref_omp.so")

MAXS, MAXR, MAXIN, MAXOUT = 16, 32, 4, 6
DP = C.POINTER(C.c_double)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


class PortReaction(C.Structure):
    _fields_ = [("nin", C.c_int), ("nout", C.c_int), ("input", C.c_int * MAXIN),
                ("output", C.c_int * MAXOUT), ("e_min", C.c_double),
                ("e_step", C.c_double), ("underflow", C.c_double),
                ("overflow", C.c_double), ("steps", C.c_int), ("values", DP)]


class PortModel(C.Structure):
    _fields_ = [("no_species", C.c_int), ("charge", C.c_double * MAXS),
                ("mass", C.c_double * MAXS), ("diffusion_coeff", C.c_double),
                ("nu_a", C.c_double), ("nu_d", C.c_double), ("nu_rt", C.c_double),
                ("bnd_cond", C.c_int * 4), ("E_x", C.c_double), ("E_y", C.c_double),
                ("E_z", C.c_double), ("z_cutoff", C.c_double), ("max_ntheta", C.c_int),
                ("dtheta", C.c_double), ("dr", DP), ("dz", DP), ("nreact", C.c_int),
                ("react", PortReaction * MAXR), ("per_plane", C.c_int),
                ("zero_all", C.c_int), ("field_mode", C.c_int),
                ("n_photo", C.c_int), ("photo_A", C.c_double * 8), ("photo_es", C.c_double * 8),
                ("photo_src", C.c_int), ("photo_e", C.c_int), ("photo_pi", C.c_int)]


class PortGrid(C.Structure):
    pass


PortGrid._fields_ = [("r0", C.c_int), ("z0", C.c_int), ("r1", C.c_int), ("z1", C.c_int),
                     ("ntheta", C.c_int), ("level", C.c_int), ("ext_bound", C.c_int),
                     ("parent", C.POINTER(PortGrid)), ("next", C.POINTER(PortGrid)),
                     ("first_child", C.POINTER(PortGrid)),
                     ("dens", DP * (MAXS + 1)), ("d_dens", DP * MAXS),
                     ("er", DP), ("ez", DP), ("etheta", DP), ("eabs", DP), ("charge", DP),
                     ("fixed_er", DP), ("fixed_ez", DP), ("fixed_et", DP), ("owns", C.c_int)]

_port = None


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError(f"oracle port library missing: {PORT_SO} (run make -C oracle)")
        lib = C.CDLL(PORT_SO)
        assert lib.port_model_size() == C.sizeof(PortModel), "port_model layout mismatch"
        assert lib.port_grid_size() == C.sizeof(PortGrid), "port_grid layout mismatch"
        lib.port_rk2.restype = C.c_double
        lib.port_courant.restype = C.c_double
        lib.port_model_size.restype = C.c_size_t
        lib.port_grid_size.restype = C.c_size_t
        lib.oracle_poisson_cyl.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, DP, DP, DP]
        lib.oracle_poisson_mode.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                            C.c_double, DP, DP, DP, DP]
        lib.oracle_dft_tables.argtypes = [C.c_int, DP, DP]
        lib.oracle_r2hc.argtypes = [C.c_int, DP, C.c_long, DP, C.c_long, DP, DP]
        lib.oracle_hc2r.argtypes = [C.c_int, DP, C.c_long, DP, C.c_long, DP, DP]
        lib.oracle_wk.argtypes = [C.c_int, DP, DP]
        lib.oracle_theta_field.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                           DP, DP, DP, DP, C.c_long]
        lib.port_advect_vec.argtypes = [C.c_double, C.c_double, DP, DP, DP, DP, C.c_double,
                                        C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
        _port = lib
    return _port


# Builds of the reference (oracle/Makefile), by variant:
#   "plain"   the reference C + the restated Fortran kernel (the oracle itself)
#   "omp"     the same with OpenMP (timing on all host cores)
#   "bigtab"  "plain" with react_table's MAX_TABLE_SIZE raised to 1024
#   "dropin"  the reference C without its Fortran wrapper, linked against the
#             device library: cdr.c:945 calls the device's arcos_cdr_advect_vec
#   "adapter" "dropin" plus the cdr_grid_t adapter, whose cdr_rk2 replaces the
#             reference's (renamed cdr_rk2_host) and runs the step on the device
REF_VARIANTS = {"plain": REF_SO, "omp": REF_OMP_SO,
                "bigtab": os.path.join(HERE, "_ref", "libarcos_ref_bigtab.so"),
                "dropin": os.path.join(HERE, "_ref", "libarcos_ref_dropin.so"),
                "adapter": os.path.join(HERE, "_ref", "libarcos_ref_adapter.so")}
_refs = {}


def _variant(omp) -> str:
    if isinstance(omp, str):
        return omp
    return "omp" if omp else "plain"


def ref_available(omp=False) -> bool:
    return os.path.exists(REF_VARIANTS[_variant(omp)])


def ref_lib(omp=False):
    """The reference build ``omp`` (a variant name, or a bool for omp/plain).
    Each build keeps its own process globals (loaded RTLD_LOCAL)."""
    path = REF_VARIANTS[_variant(omp)]
    if path not in _refs:
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle library missing: {path}")
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        lib._path = path
        for fn in ("ref_cdr_rk2", "ref_courant", "ref_rk2_sw"):
            getattr(lib, fn).restype = C.c_double
        lib.ref_cdr_rk2.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.ref_rk2_sw.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
        lib.ref_array.restype = DP
        lib.ref_array.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]
        lib.ref_setup.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double]
        lib.ref_update.argtypes = [C.c_int, C.c_int, C.c_double]
        lib.ref_advect_vec.argtypes = [C.c_double, C.c_double, DP, DP, DP, C.c_int, DP, C.c_int,
                                       C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_int, C.c_int]
        lib.ref_set_field_mode.argtypes = [C.c_int, C.c_int]
        lib.ref_set_photo.argtypes = [C.c_int, DP, DP, C.c_int, C.c_int, C.c_int]
        lib.ref_set_refine_params.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double,
                                              C.c_double, C.c_int, C.c_int, C.c_int]
        lib.ref_cdr_refine.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int]
        _refs[path] = lib
    return _refs[path]


FIELD_ZERO, FIELD_FIXED, FIELD_POISSON = 0, 1, 2


class _TreeBase:
    """Shared shape bookkeeping: ``specs`` lists the grids, parents first."""

    def __init__(self, params: Params, model: KineticModel, specs: Sequence[GridSpec]):
        self.params, self.model, self.specs = params, model, list(specs)
        self.S = model.no_species


class PortTree(_TreeBase):
    def __init__(self, params: Params, model: KineticModel, specs: Sequence[GridSpec],
                 field_mode: int = FIELD_ZERO, zero_all: bool = False):
        super().__init__(params, model, specs)
        lib = port_lib()
        self.lib = lib
        drs, dzs = params.grid_sizes()
        self._dr = np.array(drs, dtype=np.float64)
        self._dz = np.array(dzs, dtype=np.float64)
        m = PortModel()
        m.no_species = self.S
        for s, sp in enumerate(model.species):
            m.charge[s] = sp.charge
            m.mass[s] = sp.mass
        m.diffusion_coeff, m.nu_a, m.nu_d, m.nu_rt = (params.diffusion_coeff, params.nu_a,
                                                      params.nu_d, params.nu_rt)
        m.bnd_cond[1] = params.cdr_bnd_right
        m.bnd_cond[2] = params.cdr_bnd_bottom
        m.bnd_cond[3] = params.cdr_bnd_top
        m.E_x, m.E_y, m.E_z = params.E0_x, params.E0_y, params.E0_z
        m.z_cutoff = params.z_cutoff
        m.max_ntheta = params.max_ntheta
        m.dtheta = params.dtheta
        m.dr = _dp(self._dr)
        m.dz = _dp(self._dz)
        self._tables = []
        m.nreact = len(model.reactions)
        for r, re in enumerate(model.reactions):
            pr = m.react[r]
            pr.nin, pr.nout = len(re.inputs), len(re.outputs)
            for i, x in enumerate(re.inputs):
                pr.input[i] = x
            for i, x in enumerate(re.outputs):
                pr.output[i] = x
            t = re.table
            pr.e_min, pr.e_step, pr.underflow, pr.overflow, pr.steps = (
                t.e_min, t.e_step, t.underflow, t.overflow, t.steps)
            v = np.ascontiguousarray(t.padded_values())
            self._tables.append(v)
            pr.values = _dp(v)
        m.per_plane = 1 if params.per_plane else 0
        m.zero_all = 1 if zero_all else 0
        m.field_mode = field_mode
        # photo terms in the order photo_calc visits them (last-first)
        m.n_photo = len(model.photo)
        for i, t in enumerate(reversed(model.photo)):
            m.photo_A[i], m.photo_es[i] = t.A, t.lam
        m.photo_src, m.photo_e, m.photo_pi = model.photo_source, model.photo_electrons, model.photo_ions
        self.m = m
        self.grids: List[PortGrid] = []
        self.arrays = []
        for gid, sp in enumerate(self.specs):
            g = PortGrid()
            g.r0, g.z0, g.r1, g.z1 = sp.r0, sp.z0, sp.r1, sp.z1
            g.ntheta, g.level, g.ext_bound = sp.ntheta, sp.level, sp.ext_bound
            arr = {"dens": [sp.zeros() for _ in range(self.S)],
                   "d_dens": [sp.zeros() for _ in range(self.S)],
                   "er": sp.zeros(), "ez": sp.zeros(), "etheta": sp.zeros(),
                   "eabs": sp.zeros(), "charge": sp.zeros()}
            for s in range(self.S):
                g.dens[s] = _dp(arr["dens"][s])
                g.d_dens[s] = _dp(arr["d_dens"][s])
            for k in ("er", "ez", "etheta", "eabs", "charge"):
                setattr(g, k, _dp(arr[k]))
            g.dens[self.S] = g.eabs
            self.grids.append(g)
            self.arrays.append(arr)
        for gid, sp in enumerate(self.specs):
            if sp.parent >= 0:
                lib.port_add_child(C.byref(self.grids[sp.parent]), C.byref(self.grids[gid]))
                self.grids[gid].level = sp.level

    # -- field --
    def set_fixed_field(self, gid: int, er, ez, et):
        arr = self.arrays[gid]
        arr["fixed"] = [np.ascontiguousarray(x, dtype=np.float64) for x in (er, ez, et)]
        g = self.grids[gid]
        g.fixed_er, g.fixed_ez, g.fixed_et = (_dp(x) for x in arr["fixed"])

    def calc_field(self):
        self.lib.port_calc_field(C.byref(self.m), C.byref(self.grids[0]), C.byref(self.grids[0]))

    # -- operations (root = grid 0) --
    def rk2(self, h: float):
        st = C.c_int(0)
        hh = self.lib.port_rk2(C.byref(self.m), C.byref(self.grids[0]), C.c_double(h), C.byref(st))
        return hh, st.value

    def courant(self):
        st = C.c_int(0)
        h = self.lib.port_courant(C.byref(self.m), C.byref(self.grids[0]), C.byref(st))
        return h, st.value

    def rk2_frozen(self, h: float):
        """One cdr_rk2 step with exactly the step size h (no CFL limit)."""
        self.lib.port_rk2_frozen(C.byref(self.m), C.byref(self.grids[0]), C.c_double(h))

    def calc_d_dens(self):
        self.lib.port_calc_d_dens(C.byref(self.m), C.byref(self.grids[0]))

    def calc_d_dens_grid(self, gid: int):
        self.lib.port_calc_d_dens_grid(C.byref(self.m), C.byref(self.grids[gid]))

    def prepare(self):
        self.lib.port_prepare(C.byref(self.m), C.byref(self.grids[0]))

    def call(self, name: str, gid: int = 0):
        getattr(self.lib, name)(C.byref(self.m), C.byref(self.grids[gid]))

    def dens(self, gid: int, s: int) -> np.ndarray:
        return self.arrays[gid]["dens"][s]

    def array(self, gid: int, what: str, s: int = 0) -> np.ndarray:
        a = self.arrays[gid][what]
        return a[s] if isinstance(a, list) else a


_WHAT = {"dens": 0, "d_dens": 1, "er": 2, "ez": 3, "etheta": 4, "eabs": 5, "charge": 6}


class RefTree(_TreeBase):
    """The reference's own code on the same problem.  The reference keeps its
    state in process globals, so only one RefTree is live at a time."""

    def __init__(self, params: Params, model: KineticModel, specs: Sequence[GridSpec],
                 field_mode: int = FIELD_ZERO, omp=False):
        super().__init__(params, model, specs)
        lib = ref_lib(omp)
        self.lib = lib
        p = params
        lib.ref_setup(p.L_r, p.L_z, p.gridpoints_r, p.gridpoints_z, p.max_ntheta, p.max_levels,
                      p.diffusion_coeff, p.nu_a, p.nu_d, p.nu_rt, p.E0_x, p.E0_y, p.E0_z,
                      p.cdr_bnd_bottom, p.cdr_bnd_top, p.cdr_bnd_right, p.warn_min_timestep)
        for sp in model.species:
            lib.ref_add_species(C.c_double(sp.charge), C.c_double(sp.mass))
        self._tmp = tempfile.TemporaryDirectory(prefix="arcos_ref_tables_")
        nr = len(model.reactions)
        nin = (C.c_int * max(nr, 1))()
        nout = (C.c_int * max(nr, 1))()
        ins = (C.c_int * (max(nr, 1) * MAXIN))()
        outs = (C.c_int * (max(nr, 1) * MAXOUT))()
        names = b""
        for r, re in enumerate(model.reactions):
            nin[r], nout[r] = len(re.inputs), len(re.outputs)
            for i, x in enumerate(re.inputs):
                ins[r * MAXIN + i] = x
            for i, x in enumerate(re.outputs):
                outs[r * MAXOUT + i] = x
            path = os.path.join(self._tmp.name, f"r{r}.reaction")
            if re.table.points > 500 and _variant(omp) != "bigtab":
                raise ValueError("the reference stores at most 500 table points (react_table.h:5); "
                                 "use the 'bigtab' build")
            write_react_table(path, re.table, "table written for the reference oracle")
            names += path.encode() + b"\0"
        lib.ref_set_reactions(nr, nin, ins, nout, outs, C.c_char_p(names + b"\0"))
        if model.photo:
            A = np.array([t.A for t in model.photo], dtype=np.float64)
            lam = np.array([t.lam for t in model.photo], dtype=np.float64)
            self._photo = (A, lam)
            lib.ref_set_photo(len(model.photo), _dp(A), _dp(lam), model.photo_electrons,
                              model.photo_source, model.photo_ions)
        lib.ref_finish_setup()
        self.gids = []
        for sp in self.specs:
            parent = self.gids[sp.parent] if sp.parent >= 0 else -1
            self.gids.append(lib.ref_grid_new(sp.r0, sp.z0, sp.r1, sp.z1, sp.ntheta, sp.level,
                                              sp.ext_bound, parent))
        lib.ref_set_field_mode(field_mode, self.gids[0])

    def array(self, gid: int, what: str, s: int = 0) -> np.ndarray:
        n = C.c_int(0)
        ptr = self.lib.ref_array(self.gids[gid], _WHAT[what], s, C.byref(n))
        sp = self.specs[gid]
        a = np.ctypeslib.as_array(ptr, shape=(n.value,))
        return a.reshape(sp.shape)

    def dens(self, gid: int, s: int) -> np.ndarray:
        return self.array(gid, "dens", s)

    def set_fixed_field(self, gid: int, er, ez, et):
        e = [np.ascontiguousarray(x, dtype=np.float64) for x in (er, ez, et)]
        self.lib.ref_set_fixed_field(self.gids[gid], _dp(e[0]), _dp(e[1]), _dp(e[2]))

    def rk2(self, h: float, t: float = 0.0):
        return self.lib.ref_cdr_rk2(self.gids[0], C.c_double(h), C.c_double(t))

    def rk2_sw(self, h: float, per_plane: bool, zero_all: bool):
        return self.lib.ref_rk2_sw(self.gids[0], C.c_double(h), C.c_double(0.0),
                                   int(per_plane), int(zero_all))

    def call(self, name: str, gid: int = 0):
        getattr(self.lib, name)(self.gids[gid])

    def courant(self):
        return self.lib.ref_courant(self.gids[0])

    def cdr_refine(self, gid: int, threshold_eabs: float, level_eabs: int, threshold_charge: float,
                   threshold_dens: float, threshold_edge: float, brick_dr: int = 8, brick_dz: int = 8,
                   max_level: int = 4, contains_edge: bool = False):
        """The reference's cdr_refine (src/cdr.c:1630-1682) on grid ``gid``:
        the children it creates, in creation order, as (r0, z0, r1, z1,
        contains_edge); the tree is left unchanged."""
        self.lib.ref_set_refine_params(threshold_eabs, level_eabs, threshold_charge, threshold_dens,
                                       threshold_edge, brick_dr, brick_dz, max_level)
        cap = 4096
        buf = (C.c_int * (5 * cap))()
        n = self.lib.ref_cdr_refine(self.gids[gid], int(contains_edge), buf, cap)
        assert n <= cap
        return [tuple(buf[5 * i: 5 * i + 5]) for i in range(n)]


def poisson_field(nr: int, nz: int, dr: float, dz: float, charge: np.ndarray):
    """Host field stand-in of oracle/poisson_host.c: (er, ez) in rz layout."""
    lib = port_lib()
    er = np.zeros((nz + 4, nr + 4))
    ez = np.zeros((nz + 4, nr + 4))
    ch = np.ascontiguousarray(charge, dtype=np.float64).reshape(nz + 4, nr + 4)
    lib.oracle_poisson_cyl(nr, nz, dr, dz, _dp(ch), _dp(er), _dp(ez))
    return er, ez


def poisson_mode(nr: int, nz: int, dr: float, dz: float, elmbda: float, es: float,
                 charge: np.ndarray):
    """One Helmholtz mode of oracle/poisson_host.c: (er, ez, etheta = phi on
    the interior) in rz layout."""
    lib = port_lib()
    er, ez, et = (np.zeros((nz + 4, nr + 4)) for _ in range(3))
    ch = np.ascontiguousarray(charge, dtype=np.float64).reshape(nz + 4, nr + 4)
    lib.oracle_poisson_mode(nr, nz, dr, dz, elmbda, es, _dp(ch), _dp(er), _dp(ez), _dp(et))
    return er, ez, et


def dft_tables(n: int):
    """The twiddle table of oracle/dft_host.c: cos, sin of 2 pi m / n."""
    lib = port_lib()
    c, s = np.zeros(n), np.zeros(n)
    lib.oracle_dft_tables(n, _dp(c), _dp(s))
    return c, s


def dft(x: np.ndarray, sign: int) -> np.ndarray:
    """r2hc (sign > 0) or hc2r (sign < 0) of oracle/dft_host.c along the last axis."""
    lib = port_lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    c, s = dft_tables(n)
    out = np.empty_like(x)
    fn = lib.oracle_r2hc if sign > 0 else lib.oracle_hc2r
    for i in np.ndindex(x.shape[:-1]):
        xi = np.ascontiguousarray(x[i])
        yi = np.empty(n)
        fn(n, _dp(xi), 1, _dp(yi), 1, _dp(c), _dp(s))
        out[i] = yi
    return out


def wk_tables(n: int):
    """w2k, wk of a theta period of n planes (init_wk_a, src/cstream.c:309-344)."""
    lib = port_lib()
    w2k, wk = np.zeros(n), np.zeros(n)
    lib.oracle_wk(n, _dp(w2k), _dp(wk))
    return w2k, wk


def theta_field(nr: int, nz: int, nt: int, dr: float, dz: float, charge: np.ndarray):
    """The field solve of a 3-D root grid by theta modes (oracle/poisson_host.c
    oracle_theta_field), before the external field: returns (charge in theta
    modes, er, ez, etheta), each (nt + 4, nz + 4, nr + 4) with the ghost planes
    of the field zero."""
    lib = port_lib()
    shape = (nt + 4, nz + 4, nr + 4)
    ch = np.ascontiguousarray(charge, dtype=np.float64).reshape(shape).copy()
    er, ez, et = (np.zeros(shape) for _ in range(3))
    plen = (nz + 4) * (nr + 4)
    o = 2 * plen
    def p(a):                                   # pointer to plane 0
        return C.cast(a.ctypes.data + 8 * o, DP)
    lib.oracle_theta_field(nr, nz, nt, 0, dr, dz, p(ch), p(er), p(ez), p(et), plen)
    return ch, er, ez, et
