"""The allocation-free narrow seam (arcos_cdr_advect_vec_dev_noalloc) against
the allocating one (arcos_cdr_advect_vec_dev), two calls in a row with
different slabs and parameters, and against the CPU oracle's restatement of
the Fortran kernel (port_advect_vec); results must be bit-identical.
Collected last so it also runs after every other test has used the
library."""
import ctypes as C

import numpy as np
import pytest

from arcos_b200._lib import ARCOS_OK, lib
from oracle import bind

pytestmark = pytest.mark.gpu

VP = C.c_void_p


def _bind(L):
    for name in ("arcos_cdr_advect_vec_dev", "arcos_cdr_advect_vec_dev_noalloc"):
        f = getattr(L, name)
        f.argtypes = [C.c_double, C.c_double, VP, VP, VP, VP, C.c_double, C.c_double, C.c_double,
                      C.c_int, C.c_int, C.c_int, C.c_int, VP]
        f.restype = C.c_int


def _slab(rng, r0, r1, z0, z1):
    shape = (z1 - z0 + 4, r1 - r0 + 4)
    dens = rng.random(shape) ** 3
    dens[:, 3] = dens[:, 4]                      # flat stretch: the |dC| mask
    return dens, rng.normal(size=shape), rng.normal(size=shape), rng.normal(size=shape)


def test_noalloc_matches_allocating_seam(cuda_device):
    import torch
    L = lib()
    _bind(L)
    rng = np.random.default_rng(1)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [((6, 70, 0, 90), 1.0, -1.0, 0.1, 1 / 64), ((0, 45, 3, 40), 0.5, 1.0, 0.05, 1 / 128)]
    for (r0, r1, z0, z1), mass, charge, D, h in cases:
        dens, er, ez, d0 = _slab(rng, r0, r1, z0, z1)
        t = [torch.from_numpy(x).cuda() for x in (dens, er, ez)]
        out_a = torch.from_numpy(d0).cuda()
        out_b = torch.from_numpy(d0).cuda()
        ptr = lambda x: VP(x.data_ptr())
        rc = L.arcos_cdr_advect_vec_dev(mass, charge, ptr(t[0]), ptr(out_a), ptr(t[1]), ptr(t[2]),
                                        D, h, h, r0, r1, z0, z1, VP(stream))
        assert rc == ARCOS_OK
        rc = L.arcos_cdr_advect_vec_dev_noalloc(mass, charge, ptr(t[0]), ptr(out_b), ptr(t[1]), ptr(t[2]),
                                                D, h, h, r0, r1, z0, z1, VP(stream))
        assert rc == ARCOS_OK
        torch.cuda.synchronize()
        a, b = out_a.cpu().numpy(), out_b.cpu().numpy()
        assert not np.array_equal(a, d0)
        assert np.array_equal(a, b)
        # the oracle on the same slab (arcos_f90/src/cdr_advect_diffu_vec.f90:45-132)
        d_port = d0.copy()
        P = bind._dp
        bind.port_lib().port_advect_vec(mass, charge, P(dens), P(d_port), P(er), P(ez), D, h, h,
                                        r0, r1, z0, z1)
        assert np.array_equal(b, d_port)


def test_noalloc_rejects_oversize_slab(cuda_device):
    import torch
    L = lib()
    _bind(L)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = VP(x.data_ptr())
    rc = L.arcos_cdr_advect_vec_dev_noalloc(1.0, -1.0, p, p, p, p, 0.1, 0.01, 0.01, 0, 4000, 0, 4000,
                                            VP(torch.cuda.current_stream().cuda_stream))
    assert rc != ARCOS_OK
    assert b"16 MiB" in L.arcos_last_error()
