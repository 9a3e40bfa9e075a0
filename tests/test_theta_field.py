"""The field solve on a 3-D grid: theta transforms and one Helmholtz problem
per theta mode (cdr_calc_field_r, src/cdr.c:532-580 -> cdr_dft_charge_r,
pois_solve_a per mode with lambda = -w2k[k] (src/poisson.c:836-848),
cdr_dft_field_r with dft_diff, src/dft.c:37-128).

CPU part (this file):
* the transforms of oracle/dft_host.c against the definition of FFTW's r2hc
  / hc2r (FFTW itself is not installed): numpy's FFT gives the same
  halfcomplex numbers to rounding, and hc2r(r2hc(x)) = n x;
* the Helmholtz solve of oracle/poisson_host.c: its phi satisfies the
  discrete operator (hstcyl's 5-point cylindrical stencil plus
  elmbda / r^2) to rounding;
* the oracle's 3-D field-in-the-loop steps against the reference's own
  cdr_calc_field_r, dft_transform and dft_diff (compiled from the reference
  sources against the FFTW shim), bit for bit.

The device side is in test_gpu_theta_field.py.
"""
import numpy as np
import pytest

from arcos_b200 import workloads
from oracle import bind
from parity_util import max_ulp, port_tree

needs_ref = pytest.mark.skipif(not bind.ref_available(), reason="reference build absent")


@pytest.mark.parametrize("n", [2, 4, 5, 8, 16, 32])
def test_dft_matches_the_halfcomplex_definition(n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(7, n))
    y = bind.dft(x, +1)
    f = np.fft.rfft(x, axis=-1)
    ref = np.zeros_like(x)
    ref[:, : n // 2 + 1] = f.real
    for k in range(1, (n + 1) // 2):
        ref[:, n - k] = f[:, k].imag
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    back = bind.dft(y, -1)
    assert np.max(np.abs(back - n * x)) <= 1e-13 * n * np.max(np.abs(x))


def test_wk_tables_are_the_forward_difference_in_theta():
    n = 8
    w2k, wk = bind.wk_tables(n)
    dth = 2 * np.pi / n
    k = np.arange(n)
    assert np.allclose(w2k, 2 / dth ** 2 * (1 - np.cos(k * dth)), rtol=1e-14, atol=1e-14)
    for kk in range(1, n // 2):
        assert wk[kk] == pytest.approx((np.cos(kk * dth) - 1) / dth, rel=1e-14)
        assert wk[n - kk] == pytest.approx(np.sin(kk * dth) / dth, rel=1e-14)
    assert wk[0] == 0.0


@pytest.mark.parametrize("elmbda,es", [(0.0, 0.0), (-3.5, 0.0), (-40.0, -2.0)])
def test_helmholtz_mode_solves_the_discrete_operator(elmbda, es):
    nr, nz, dr, dz = 24, 40, 0.05, 0.1
    rng = np.random.default_rng(3)
    q = np.zeros((nz + 4, nr + 4))
    q[2:-2, 2:-2] = rng.normal(size=(nz, nr))
    er, ez, phi4 = bind.poisson_mode(nr, nz, dr, dz, elmbda, es, q)
    phi = phi4[2:-2, 2:-2]                      # [z, r]
    # ghosts: Dirichlet (antisymmetric) at r = L_r, z = 0, z = L_z; the axis
    # term carries r_{-1/2} = 0
    p = np.zeros((nz + 2, nr + 1))
    p[1:-1, :nr] = phi
    p[1:-1, nr] = -phi[:, nr - 1]
    p[0, :nr] = -phi[0]
    p[-1, :nr] = -phi[-1]
    r = (np.arange(nr) + 0.5) * dr
    rm, rp = np.arange(nr) * dr, (np.arange(nr) + 1) * dr
    c = p[1:-1, :nr]
    left = np.concatenate([c[:, :1], c[:, :-1]], axis=1)
    lap_r = (rp * (p[1:-1, 1:nr + 1] - c) - rm * (c - left)) / (r * dr * dr)
    lap_z = (p[2:, :nr] - 2 * c + p[:-2, :nr]) / (dz * dz)
    res = lap_r + lap_z + (elmbda / r ** 2 + es) * c + q[2:-2, 2:-2]
    assert np.max(np.abs(res)) <= 1e-10 * np.max(np.abs(q[2:-2, 2:-2]))
    # the axis face of er: phi(-1) = phi(0) for the symmetric mode, -phi(0) otherwise
    sgn = 1.0 if elmbda == 0.0 else -1.0
    assert np.array_equal(er[2:-2, 1], -(phi[:, 0] - sgn * phi[:, 0]) / dr)


def ref_tree(pb, field_mode):
    import copy
    t = bind.RefTree(copy.deepcopy(pb.params), pb.model, pb.specs, field_mode=field_mode)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            t.dens(g, s)[...] = a
    return t


@needs_ref
@pytest.mark.parametrize("ntheta,per_plane", [(4, True), (4, False), (8, True), (5, True)])
def test_port_matches_reference_3d_field_in_loop(ntheta, per_plane):
    pb = workloads.plain(nr=20, nz=36, ntheta=ntheta, ion_mass=0.0, noise=0.3, seed=11)
    pb.params.per_plane = per_plane
    port = port_tree(pb, field_mode=bind.FIELD_POISSON, per_plane=per_plane)
    ref = ref_tree(pb, bind.FIELD_POISSON)
    port.call("port_calc_charge")
    ref.call("ref_calc_charge_r")
    for _ in range(3):
        # the literal reference (per_plane False: the Fortran sees the theta = -2
        # plane only), or its switch that runs drift/diffusion on every plane
        h_ref = ref.rk2_sw(50.0, per_plane=True, zero_all=False) if per_plane else ref.rk2(50.0)
        assert port.rk2(50.0)[0] == h_ref
    for w in ("dens", "d_dens"):
        for s in range(pb.model.no_species):
            assert max_ulp(port.array(0, w, s), ref.array(0, w, s)) == 0, (w, s)
    for w in ("er", "ez", "etheta", "eabs", "charge"):
        assert max_ulp(port.array(0, w, 0), ref.array(0, w, 0)) == 0, w
    # the field is genuinely three-dimensional
    et = port.array(0, "etheta", 0)
    assert np.max(np.abs(et[2:-2, 2:-2, 2:-2])) > 0
