"""Generates the golden fixtures of tests/golden from the reference build
(oracle/_ref: the reference C sources with the restated Fortran kernel).

Run in a container that has the reference tree:  python tests/golden/make_golden.py
Each case stores its inputs (densities of every grid) and the reference's
state and step sizes after a few cdr_rk2 steps.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from arcos_b200 import workloads  # noqa: E402
from oracle import bind  # noqa: E402

CASES = {
    # name: (builder kwargs, steps, rk2 flavour)
    "plain2d": (("plain", dict(nr=24, nz=40, ion_mass=1.0, noise=1e-3, seed=21)), 4, "exact"),
    "plain2d_immobile_ions": (("plain", dict(nr=20, nz=36, ion_mass=0.0, noise=1e-3, seed=22)), 4, "exact"),
    "theta_per_plane": (("plain", dict(nr=16, nz=24, ntheta=4, ion_mass=1.0, noise=1e-6, seed=23)), 2, "per_plane"),
    "theta_ref_exact": (("plain", dict(nr=16, nz=24, ntheta=4, ion_mass=1.0, noise=1e-6, seed=24)), 2, "exact"),
    "amr": (("amr", dict(n_patches=9, levels=3, root_nr=32, root_nz=64, side_lo=8, side_hi=20, seed=25)), 2, "zero_all"),
    "kinetic": (("kinetic_batch", dict(n_inst=1, points=300, sizes_r=(24,), sizes_z=(32,), seed=26)), 3, "exact"),
}


def run_case(name):
    (kind, kw), steps, flavour = CASES[name]
    pb = getattr(workloads, kind)(**kw)
    if name == "theta_ref_exact":
        pb.params.per_plane = False
    import copy
    params = copy.deepcopy(pb.params)
    if pb.family_E:
        params.E0_x, params.E0_y, params.E0_z = pb.family_E[0]
    ref = bind.RefTree(params, pb.model, pb.specs, field_mode=bind.FIELD_FIXED)
    for g, per in enumerate(pb.dens):
        for s, a in enumerate(per):
            ref.dens(g, s)[...] = a
    for g, (er, ez, et) in enumerate(pb.fields):
        ref.set_fixed_field(g, er, ez, et if et is not None else pb.specs[g].zeros())
    dts = []
    for _ in range(steps):
        if flavour == "exact":
            dts.append(ref.rk2(50.0))
        elif flavour == "per_plane":
            dts.append(ref.rk2_sw(50.0, per_plane=True, zero_all=False))
        else:
            dts.append(ref.rk2_sw(50.0, per_plane=False, zero_all=True))
    out = {"dts": np.array(dts), "steps": steps}
    for g in range(len(pb.specs)):
        for s in range(pb.model.no_species):
            out[f"in_g{g}_s{s}"] = pb.dens[g][s]
            out[f"out_g{g}_s{s}"] = ref.dens(g, s).copy()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return out


if __name__ == "__main__":
    for name in CASES:
        run_case(name)
        print("wrote", name)
