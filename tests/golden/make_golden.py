"""Generates the golden fixtures of tests/golden/ from the reference itself.

    make -C oracle            # builds oracle/_ref/pdref_harness from the reference sources
    python tests/golden/make_golden.py

Each case is a small synthetic deck written by pdmtel_b200.decks into
tests/golden/decks/<case>/pds_input.txt; the reference harness
(oracle/ref_harness.cpp) runs it through the reference's own InitialProblem,
CalcIntgPointDisplRK4, CalcBondBasedMotionRK4 and RK4, and the dumped FP64
state is stored as tests/golden/<case>.npz.  The fixtures are what the oracle
and the CUDA path are pinned against; nothing at test time needs the
reference sources.
"""
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from pdmtel_b200 import decks as D  # noqa: E402
from pdb_io import read_pdb  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "pdref_harness")


def cases():
    h = 1e-3
    out = {}
    # FGI 2x2x2 + MLS, boundary factors on, fixed left face, pulled right face
    d = D.config_bar(dims=(8, 5, 4), spacing=h, traction_as_veloc=0.05, dt=1e-8, steps=100, bdry_eff=1)
    out["fgi_velo"] = (d, dict(force=(2e-8, 1e-8), traj=(6, 3)))
    # CCI (original beta), displacement-gradient faces, damping, stable time step
    dims = (8, 5, 4)
    d = D.Deck(dims=dims, spacing=2.0, horizon=6.0, total_time=2.0, total_step=50, safety=1.1,
               materials=[(1.0e5, 1e14, 6e10, 2e-6)], damping=0.06, bdry_eff=1, cci=(1, 0),
               bcs=[D.BC(D.DISPLGRAD, (1, 1, 1), (-2.5e-5, 0, 0, 0, 1e-4, 0, 0, 0, -2.5e-5), 8e-4, 2.0)],
               bc_spaces=[D.Space(1, D.face_box(dims, 2.0, 1, -1)), D.Space(1, D.face_box(dims, 2.0, 1, +1))])
    out["cci_grad"] = (d, dict(force=(0.5, 0.25), traj=(4, 2)))
    # CCI modified beta, velocity and ramped displacement faces
    d = D.Deck(dims=(7, 6, 4), spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=2e-8,
               damping=0.01, bdry_eff=0, cci=(1, 1),
               bcs=[D.BC(D.VELOC, (1, 1, 0), (0.02, -0.01, 0.0), 3e-8, 2.0), D.BC(D.DISPL, (1, 0, 1), (1e-7, 0, -2e-7), 1e-7, 1.0)],
               bc_spaces=[D.Space(1, D.face_box((7, 6, 4), h, 0, -1)), D.Space(2, D.face_box((7, 6, 4), h, 0, +1))])
    out["cci_mdf"] = (d, dict(force=(5e-8, 2e-8), traj=(5, 5)))
    # slit deletion with +-v velocity layers (the plate case in miniature)
    d = D.config_plate(dims=(12, 10, 3), spacing=h, slit_half_length=2.0e-3, vel=0.05, dt=1e-8, steps=100)
    out["fgi_slit"] = (d, dict(force=(2e-8, 1e-8), traj=(6, 3)))
    # 3x3x3 Gauss points, ramped displacement gradient, boundary factors
    dims = (7, 5, 5)
    d = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               damping=0.02, bdry_eff=1, intg_point=3,
               bcs=[D.BC(D.DISPLGRAD, (1, 0, 1), (1e-4, 0, 0, 0, 0, 0, 0, 2e-5, -5e-5), 5e-8, 1.0),
                    D.BC(D.DISPL, (0, 1, 0), (0, 3e-9, 0), 1.0, 2.0)],
               bc_spaces=[D.Space(1, D.face_box(dims, h, 2, -1)), D.Space(2, D.face_box(dims, h, 0, +1))])
    out["fgi3_ramp"] = (d, dict(force=(3e-8, 1e-8), traj=(4, 2)))
    # one Gauss point (no MLS), a cylindrical deletion space, traction parsed
    dims = (9, 7, 3)
    d = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               bdry_eff=0, intg_point=1,
               deletion_spaces=[D.Space(0, (1.6e-3, 0.0, 0.0, -1.0, 1.0), geo=2)],
               bcs=[D.BC(D.VELOC, (0, 0, 1), (0, 0, 0.03), 1.0, 2.0)],
               bc_spaces=[D.Space(1, D.face_box(dims, h, 0, -1))])
    out["fgi1_hole"] = (d, dict(force=(2e-8, 1e-8), traj=(4, 4)))
    return out


def run(mode, workdir, out, *args):
    r = subprocess.run([HARNESS, mode, workdir, out] + [str(a) for a in args], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"harness {mode} {workdir} failed: {r.stderr[-400:]}")


def main():
    if not os.path.exists(HARNESS):
        raise SystemExit("oracle/_ref/pdref_harness missing: run `make -C oracle` first")
    tmp = os.path.join(ROOT, "_work", "golden_tmp")
    os.makedirs(tmp, exist_ok=True)
    for name, (deck, spec) in cases().items():
        ddir = os.path.join(HERE, "decks", name)
        deck.write(ddir)
        wd = os.path.join(tmp, name)
        os.makedirs(wd, exist_ok=True)
        shutil.copy(os.path.join(ddir, "pds_input.txt"), os.path.join(wd, "pds_input.txt"))
        data = {}
        t, dts = spec["force"]
        run("force", wd, os.path.join(wd, "force.bin"), t, dts)
        for k, v in read_pdb(os.path.join(wd, "force.bin")).items():
            data[k] = v
        nsteps, every = spec["traj"]
        run("traj", wd, os.path.join(wd, "traj.bin"), nsteps, every)
        for k, v in read_pdb(os.path.join(wd, "traj.bin")).items():
            if k.startswith(("U_", "V_", "ug_")) or k in ("ke", "ee", "times"):
                data["traj_" + k] = v
        data["force_args"] = np.array([t, dts])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
        print(name, int(data["n"][0]), "nodes", len(data["fam_col"]), "halves")


if __name__ == "__main__" and "--kat" not in sys.argv:
    main()


def sample_like_deck():
    """The parameters of the reference's sample deck (cubic_in_tension, CCI,
    two displacement-gradient boundary layers), written with this package's
    deck writer."""
    dims = (20, 40, 20)
    bc = D.BC(D.DISPLGRAD, (1, 1, 1), (-2.5e-5, 0, 0, 0, 1e-4, 0, 0, 0, -2.5e-5), 8e-4, 2.0)
    return D.Deck(dims=dims, spacing=2.0, horizon=6.0, total_time=2.0, total_step=50, dump=50, safety=1.1,
                  materials=[(1.0e5, 1e14, 6e10, 2e-6)],
                  material_spaces=[D.Space(1, (-500, 500, -500, 500, -500, 500))],
                  bcs=[bc, bc, bc],
                  bc_spaces=[D.Space(1, (-500, 500, -40, -38, -500, 500)), D.Space(2, (-500, 500, 38, 40, -500, 500))],
                  damping=0.06, bdry_eff=1, cci=(1, 0), title="cubic_in_tension")


def make_kat():
    """Known answers of larger decks: bond counts and energies of the first
    steps, from the reference harness."""
    import json
    tmp = os.path.join(ROOT, "_work", "golden_tmp")
    kat = {}
    wd = os.path.join(tmp, "sample_like")
    sample_like_deck().write(wd)
    sample_like_deck().write(os.path.join(HERE, "decks", "sample_like"))
    run("traj", wd, os.path.join(wd, "traj.bin"), 2, 100)
    g = read_pdb(os.path.join(wd, "traj.bin"))
    kat["sample_like"] = {"bonds": int(g["num_bonds"][0]), "ke": g["ke"].tolist(), "ee": g["ee"].tolist(),
                          "dt": float(g["dt"][0]), "u2_sum_abs": float(np.abs(g["U_2"]).sum()),
                          "v2_sum_abs": float(np.abs(g["V_2"]).sum())}
    wd = os.path.join(tmp, "bar")
    D.config_bar(traction_as_veloc=0.05).write(wd)
    run("setup", wd, os.path.join(wd, "setup.bin"))
    g = read_pdb(os.path.join(wd, "setup.bin"))
    kat["bar_20x10x10"] = {"bonds": int(g["num_bonds"][0]), "max_family": int(np.diff(g["fam_ptr"]).max()),
                           "num_max_family": int(g["num_max_family"][0])}
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    print(kat)


if __name__ == "__main__" and "--kat" in sys.argv:
    make_kat()
