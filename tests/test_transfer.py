"""arcos_upload / arcos_download round trips: the packed host image of an
array (the reference's rz_array layout, ghosts included) moves by one linear
copy and a repitch kernel; every value must come back bit for bit, for odd
widths (row padding), 3-D planes, every array kind and both storage sets."""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200.cdr import CdrTree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nr,nz,ntheta", [(45, 51, 1), (37, 29, 4), (64, 128, 1)])
def test_upload_download_round_trip(cuda_device, nr, nz, ntheta):
    pb = workloads.plain(nr=nr, nz=nz, ntheta=ntheta, ion_mass=1.0, noise=1e-3, seed=8)
    dev = CdrTree(pb.params, pb.model, pb.specs)
    rng = np.random.default_rng(9)
    shape = pb.specs[0].shape
    for set_ in (0, 1):
        for what, species in (("dens", 0), ("dens", 1), ("er", 0), ("ez", 0), ("eabs", 0), ("charge", 0)):
            a = rng.standard_normal(shape)
            dev.upload(0, what, a, species, set=set_)
            b = dev.download(0, what, species, set=set_)
            assert np.array_equal(a, b), (what, species, set_)
    # one array does not disturb its neighbours in the same block
    x = rng.standard_normal(shape)
    y = rng.standard_normal(shape)
    dev.upload(0, "dens", x, 0)
    dev.upload(0, "dens", y, 1)
    assert np.array_equal(dev.download(0, "dens", 0), x)
    assert np.array_equal(dev.download(0, "dens", 1), y)
    dev.close()
