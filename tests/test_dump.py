"""FP64 dump and load of device arrays (arcos_dump), in place of the
reference's "%15.5e" text dumps (rz_dump_3d, src/rz_array.c:352-407): the
same cell order (theta outermost, then r, z fastest), lossless."""
import numpy as np
import pytest

from arcos_b200 import workloads
from arcos_b200._lib import ArcosError
from arcos_b200.cdr import CdrTree

pytestmark = pytest.mark.gpu


def _tree(pb):
    t = CdrTree(pb.params, pb.model, pb.specs)
    for s in range(2):
        t.upload(0, "dens", pb.dens[0][s], s)
    return t


@pytest.mark.parametrize("ntheta", [1, 4])
def test_dump_order_and_round_trip(cuda_device, tmp_path, ntheta):
    pb = workloads.plain(nr=24, nz=40, ntheta=ntheta, ion_mass=1.0, noise=1e-3, seed=5)
    a = _tree(pb)
    path = tmp_path / "ne.f64"
    a.dump(path, 0, "dens", 0)
    raw = np.fromfile(path, dtype=np.uint8)
    assert bytes(raw[:8]) == b"ARCOSF64"
    hdr = np.frombuffer(raw[8:32].tobytes(), dtype=np.int32)
    assert list(hdr[:3]) == [24, 40, ntheta]
    cells = np.frombuffer(raw[32:].tobytes(), dtype=np.float64)
    arr = pb.dens[0][0]
    t0 = 0 if ntheta == 1 else 2
    expect = np.stack([arr[t0 + it, 2:-2, 2:-2].T for it in range(ntheta)]).ravel()   # (theta, r, z)
    assert np.array_equal(cells, expect)
    # load into another tree: the interior bit for bit, the ghosts untouched
    pb2 = workloads.plain(nr=24, nz=40, ntheta=ntheta, ion_mass=1.0, noise=1e-3, seed=6)
    b = _tree(pb2)
    before = b.download(0, "dens", 0)
    b.load(path, 0, "dens", 0)
    after = b.download(0, "dens", 0)
    sl = (slice(t0, t0 + ntheta), slice(2, -2), slice(2, -2))
    assert np.array_equal(after[sl], arr[sl])
    mask = np.ones(after.shape, bool)
    mask[sl] = False
    assert np.array_equal(after[mask], before[mask])
    a.close()
    b.close()


def test_load_refuses_another_shape(cuda_device, tmp_path):
    a = _tree(workloads.plain(nr=24, nz=40, ion_mass=1.0, seed=1))
    b = _tree(workloads.plain(nr=24, nz=48, ion_mass=1.0, seed=1))
    path = tmp_path / "x.f64"
    a.dump(path)
    with pytest.raises(ArcosError):
        b.load(path)
    with pytest.raises(ArcosError):
        b.load(tmp_path / "absent.f64")
    a.close()
    b.close()
