"""Generates the golden fixtures of tests/golden/ from the reference itself.

    make -C oracle REF=<reference dir>   # builds oracle/_ref/pdref_harness
    python tests/golden/make_golden.py           # the small decks, tests/golden/*.npz
    python tests/golden/make_golden.py --kat     # known answers of larger decks, kat.json
    python tests/golden/make_golden.py --long    # the 20x10x10 bar over 100 steps, long/*.npz
    python tests/golden/make_golden.py --static  # the linearised stiffness pass, static/*.npz
    python tests/golden/make_golden.py --outputs # the reference's output files, outputs/<case>/
    python tests/golden/make_golden.py --ai      # adaptive-trapezoid decks, tests/golden/ai/*.npz

Each case is a small synthetic deck written by pdmtel_b200.decks into
tests/golden/decks/<case>/pds_input.txt; the reference harness
(oracle/ref_harness.cpp) runs it through the reference's own InitialProblem,
CalcIntgPointDisplRK4, CalcBondBasedMotionRK4 and RK4, and the dumped FP64
state is stored as tests/golden/<case>.npz.  The fixtures are what the oracle
and the CUDA path are pinned against; nothing at test time needs the
reference sources.
"""
import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

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
    tmp = tempfile.mkdtemp(prefix="pdgolden_")
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
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__" and not {"--kat", "--long", "--static", "--outputs", "--ai"} & set(sys.argv):
    main()


def ai_cases():
    """Adaptive-trapezoid (ai_on) decks.  Boundary conditions prescribe every
    direction (DISPL or DISPLGRAD with flags 1 1 1): a family node with a
    VELOC condition, or an unflagged direction, makes the reference's
    integrand read an unset local (pdIntgManager2.cpp:122-174), which no
    fixture can pin."""
    h = 1e-3
    out = {}
    dims = (7, 5, 5)
    grad = D.BC(D.DISPLGRAD, (1, 1, 1), (1e-4, 0, 0, 0, 0, 0, 0, 2e-5, -5e-5), 5e-8, 1.0)
    pull = D.BC(D.DISPL, (1, 1, 1), (1e-7, 3e-9, -2e-8), 1.0, 2.0)
    spaces = [D.Space(1, D.face_box(dims, h, 2, -1)), D.Space(2, D.face_box(dims, h, 0, +1))]
    # trapezoid index 3 (5 points per direction), MLS, boundary factors
    d = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               damping=0.02, bdry_eff=1, ai_mls=1, intg_point=3, bcs=[grad, pull], bc_spaces=spaces)
    out["ai_mls3"] = (d, dict(force=(1e-8, 1e-8), traj=(2, 1)))
    # trapezoid index 2, a wider horizon (other cuts of the cell by the sphere)
    dims2 = (8, 6, 5)
    d = D.Deck(dims=dims2, spacing=h, horizon=3.5 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               bdry_eff=0, ai_mls=1, intg_point=2, bcs=[pull, D.BC(D.DISPL, (1, 1, 1), (0, 0, 0), 1.0, 2.0)],
               bc_spaces=[D.Space(1, D.face_box(dims2, h, 0, +1)), D.Space(2, D.face_box(dims2, h, 0, -1))])
    out["ai_mls2_d35"] = (d, dict(force=(2e-8, 1e-8), traj=(2, 2)))
    # trapezoid index 1, horizon 2.515 dx, a slit
    dims3 = (9, 6, 4)
    d = D.Deck(dims=dims3, spacing=h, horizon=2.515 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               slits=[(-0.0015, -0.0005, -1.0, 0.0002, -1.0, 1.0)],
               bdry_eff=1, ai_mls=1, intg_point=1, bcs=[pull], bc_spaces=[D.Space(1, D.face_box(dims3, h, 0, +1))])
    out["ai_mls1_slit"] = (d, dict(force=(2e-8, 1e-8), traj=(3, 3)))
    # (ai_on 1 0, without MLS, is left out: the reference's RK4 path deletes
    # element 0 of a zero-length contributor array in ~pdIntgManager
    # (pdIntgManager.cpp:37-46, pdDataManager.cpp:1892-1901) and crashes)
    # a small critical stretch: points past it break their bonds
    d = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=100, fixed_dt=1e-8,
               materials=[(72e9, 1e20, 2.0e-4, 2440.0)], bdry_eff=0, ai_mls=1, intg_point=1,
               bcs=[D.BC(D.DISPL, (1, 1, 1), (4e-6, 0, 0), 3e-8, 1.0), D.BC(D.DISPL, (1, 1, 1), (0, 0, 0), 1.0, 2.0)],
               bc_spaces=[D.Space(1, D.face_box(dims, h, 0, +1)), D.Space(2, D.face_box(dims, h, 0, -1))])
    out["ai_break"] = (d, dict(force=(1e-8, 1e-8), traj=(4, 1)))
    return out


def _ai_one(args):
    name, deck, spec, tmp = args
    ddir = os.path.join(HERE, "decks", name)
    deck.write(ddir)
    wd = os.path.join(tmp, name)
    os.makedirs(wd, exist_ok=True)
    shutil.copy(os.path.join(ddir, "pds_input.txt"), os.path.join(wd, "pds_input.txt"))
    data = {}
    t, dts = spec["force"]
    run("force", wd, os.path.join(wd, "force.bin"), t, dts)
    data.update(read_pdb(os.path.join(wd, "force.bin")))
    if spec["traj"]:
        nsteps, every = spec["traj"]
        run("traj", wd, os.path.join(wd, "traj.bin"), nsteps, every)
        for k, v in read_pdb(os.path.join(wd, "traj.bin")).items():
            if k.startswith(("U_", "V_", "broken_")) or k in ("ke", "ee", "times"):
                data["traj_" + k] = v
    data["force_args"] = np.array([t, dts])
    os.makedirs(os.path.join(HERE, "ai"), exist_ok=True)
    np.savez_compressed(os.path.join(HERE, "ai", name + ".npz"), **data)
    return name, int(data["n"][0]), len(data["fam_col"])


def make_ai():
    from multiprocessing import get_context
    tmp = tempfile.mkdtemp(prefix="pdgolden_ai_")
    jobs = [(name, deck, spec, tmp) for name, (deck, spec) in ai_cases().items()]
    with get_context("spawn").Pool(len(jobs)) as pool:
        for name, n, h in pool.imap_unordered(_ai_one, jobs):
            print(name, n, "nodes", h, "halves", flush=True)
    shutil.rmtree(tmp, ignore_errors=True)


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
    tmp = tempfile.mkdtemp(prefix="pdgolden_")
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
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__" and "--kat" in sys.argv:
    make_kat()


# ---- the 20x10x10 bar over 100 RK4 steps (tests/golden/long/) ----
#
# The plain-FP64 config: 20x10x10 nodes, spacing 1 mm, horizon 3.015 mm, FGI
# 2x2x2 points with MLS, dt 1e-8 s, 100 steps from rest, with the boundary-
# effect factor off and on.  The reference applies no traction load (type 4 is
# parsed and never used, pdDataManager.cpp:2534-2592), so the right face is
# pulled with a velocity condition instead; the left face is fixed.  These
# decks hold full 250-node families and, with bdryEff on, nodes of all three
# branches of InitBdryEffectFactor (full family, one face, several faces,
# pdDataManager.cpp:1412-1461).
#
# Arrays that are compared bit for bit are stored as SHA-256 digests of their
# little-endian bytes (family lists, contributor lists, MLS coefficients,
# Gauss-point displacements); the state every 10 steps is stored as digests,
# and in full at steps 10, 50 and 100 together with the boundary-effect
# factors, the stage-1 k vector at a non-trivial displacement and the
# energies of every step, so that a mismatch can be measured.

LONG_STEPS = 100
LONG_EVERY = 10
LONG_FULL = (10, 50, 100)


def digest(a):
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.astype(a.dtype.newbyteorder("<")).tobytes()).hexdigest()


def long_cases():
    return {f"bar20_bE{b}": D.config_bar(dims=(20, 10, 10), spacing=1e-3, traction_as_veloc=0.05, dt=1e-8,
                                         steps=LONG_STEPS, bdry_eff=b) for b in (0, 1)}


def sample_nodes(n, dims):
    """Nodes whose MLS coefficients are stored in full: a corner, an edge, a
    face and interior nodes, and a seeded handful of others."""
    nx, ny, nz = dims
    pick = lambda x, y, z: x + nx * (y + ny * z)
    fixed = [pick(0, 0, 0), pick(10, 0, 0), pick(10, 5, 0), pick(10, 5, 5), pick(19, 9, 9), pick(3, 4, 5),
             pick(16, 5, 4), pick(1, 1, 1)]
    rng = np.random.default_rng(20)
    return np.unique(np.concatenate([fixed, rng.choice(n, 24, replace=False)])).astype(np.int64)


def make_long():
    out_dir = os.path.join(HERE, "long")
    os.makedirs(out_dir, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="pdgolden_long_")
    for name, deck in long_cases().items():
        ddir = os.path.join(out_dir, "decks", name)
        deck.write(ddir)
        wd = os.path.join(tmp, name)
        os.makedirs(wd, exist_ok=True)
        shutil.copy(os.path.join(ddir, "pds_input.txt"), os.path.join(wd, "pds_input.txt"))
        t, dts = 2e-8, 1e-8
        run("force", wd, os.path.join(wd, "force.bin"), t, dts)
        f = read_pdb(os.path.join(wd, "force.bin"))
        n = int(f["n"][0])
        npt = int(f["num_gauss"][0])
        keep = sample_nodes(n, deck.dims)
        cb_ptr = f["cb_ptr"]
        co = f["coeff"]
        samples = []
        for i in keep:
            b, e = cb_ptr[i], cb_ptr[i + 1]
            samples.append(co[b * npt:e * npt])
        data = {
            "n": f["n"], "dims": np.array(deck.dims, dtype=np.int64), "num_bonds": f["num_bonds"],
            "min_bond": f["min_bond"], "dt": f["dt"], "params": f["params"], "iparams": f["iparams"],
            **{k: f[k] for k in ("mat", "bc", "spring", "mat_ymod", "mat_density", "mat_ecrit", "mat_grav", "bc_type",
                                 "bc_dir", "bc_val", "bc_end", "bc_load", "gw")},
            "fam_ptr": f["fam_ptr"], "bdry_eff": f["bdry_eff"], "cb_ptr": cb_ptr,
            "sha_fam_col": np.array(digest(f["fam_col"])), "sha_broken": np.array(digest(f["broken"])),
            "sha_cb_idx": np.array(digest(f["cb_idx"])), "sha_coeff": np.array(digest(co)),
            "sha_gauss_x": np.array(digest(f["gauss_x"])),
            "coeff_nodes": keep, "coeff_samples": np.concatenate(samples),
            "force_args": np.array([t, dts]), "u_test": f["u_test"], "v_test": f["v_test"],
            "k": f["k"], "vbuf": f["vbuf"], "eed": f["eed"],
            "sha_ug_force": np.array(digest(f["ug"])),
        }
        if "num_max_family" in f:
            data["num_max_family"] = f["num_max_family"]
        run("traj", wd, os.path.join(wd, "traj.bin"), LONG_STEPS, LONG_EVERY)
        tr = read_pdb(os.path.join(wd, "traj.bin"))
        for s in range(LONG_EVERY, LONG_STEPS + 1, LONG_EVERY):
            for q in ("U", "V", "ug"):
                data[f"sha_{q}_{s}"] = np.array(digest(tr[f"{q}_{s}"]))
            if s in LONG_FULL:
                data[f"U_{s}"] = tr[f"U_{s}"]
                data[f"V_{s}"] = tr[f"V_{s}"]
        data["ke"], data["ee"], data["times"] = tr["ke"], tr["ee"], tr["times"]
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), **data)
        print(name, n, "nodes", int(f["num_bonds"][0]), "bonds", "max family", int(np.diff(f["fam_ptr"]).max()))
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__" and "--long" in sys.argv:
    make_long()


# ---- the linearised stiffness operator (tests/golden/static/) ----
#
# pdDataManager::CalcDampingCoeff (pdDataManager2.cpp:1616-1907) forms K u
# matrix-free with the coefficients of pdSolve::AssembleEquation (pdSolve.cpp:
# 195-527) and returns the per-dof sum of |K_ij| (times dt^2/4) and
# 2 sqrt(u.Ku / u.Mu).  The decks carry no boundary condition and no slit, so
# that K is the unconstrained operator of the whole family: two materials (the
# min spring rule), Gauss-point and CCI decks, and a deletion hole.  dt = 2
# makes the dt^2/4 scale exactly 1.

STATIC_DT = 2.0


def static_cases():
    h = 1e-3
    out = {}
    dims = (8, 5, 4)
    out["static_bar"] = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=10,
                               fixed_dt=1e-8, intg_point=1)
    dims = (7, 6, 4)
    out["static_cci"] = D.Deck(dims=dims, spacing=2.0, horizon=6.0, total_time=1.0, total_step=10, fixed_dt=1e-3,
                               materials=[(1.0e5, 1e14, 6e10, 2e-6)], cci=(1, 0))
    dims = (9, 7, 3)
    out["static_hole"] = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=1.0, total_step=10,
                                fixed_dt=1e-8, intg_point=1,
                                deletion_spaces=[D.Space(0, (1.6e-3, 0.0, 0.0, -1.0, 1.0), geo=2)])
    return out


def make_static():
    out_dir = os.path.join(HERE, "static")
    os.makedirs(out_dir, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="pdgolden_static_")
    for name, deck in static_cases().items():
        ddir = os.path.join(out_dir, "decks", name)
        deck.write(ddir)
        wd = os.path.join(tmp, name)
        os.makedirs(wd, exist_ok=True)
        shutil.copy(os.path.join(ddir, "pds_input.txt"), os.path.join(wd, "pds_input.txt"))
        run("damp", wd, os.path.join(wd, "damp.bin"), STATIC_DT)
        f = read_pdb(os.path.join(wd, "damp.bin"))
        keep = ("n", "coords", "mat", "fam_ptr", "fam_col", "broken", "spring", "mat_density", "params", "iparams",
                "absK", "damp_coeff", "damp_dt", "u_field_0", "u_field_1", "u_field_2")
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), **{k: f[k] for k in keep})
        print(name, int(f["n"][0]), "nodes", "damping coefficients", f["damp_coeff"])
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__" and "--static" in sys.argv:
    make_static()


# ---- the reference's output files (tests/golden/outputs/) ----
#
# pdSolve::SolveDynamic (pdSolve.cpp:24-130) writes the pds_output.dat log
# (the deck echo of ReadInputFile and one line per step), the pds_steps.dat
# probe of the node at (dx/2, dx/2, dx/2) and pds_tecplot_<step>.dat at the
# first, the last and every dump step (pdSolve.cpp:708-774, pdNode.cpp:418-
# 433).  The harness runs it on two small decks (Gauss points with MLS and a
# shortened last step; CCI with a ramped displacement gradient) and the files
# are kept under outputs/<case>/ with a ref_ prefix.

def output_cases():
    h = 1e-3
    out = {}
    dims = (8, 6, 4)
    out["out_fgi"] = D.Deck(dims=dims, spacing=h, horizon=3.015 * h, total_time=6.5e-8, total_step=7, dump=3,
                            fixed_dt=1e-8, damping=0.01, bdry_eff=1, intg_point=2,
                            bcs=[D.BC(D.DISPL, (1, 1, 1), (0.0, 0.0, 0.0), 1.0, 2.0),
                                 D.BC(D.VELOC, (1, 0, 0), (0.05, 0.0, 0.0), 1.0, 2.0)],
                            bc_spaces=[D.Space(1, D.face_box(dims, h, 0, -1)), D.Space(2, D.face_box(dims, h, 0, +1))],
                            title="output check gauss")
    dims = (6, 6, 4)
    out["out_cci"] = D.Deck(dims=dims, spacing=2.0, horizon=6.0, total_time=2.0, total_step=5, dump=2, safety=1.1,
                            materials=[(1.0e5, 1e14, 6e10, 2e-6)], damping=0.06, bdry_eff=1, cci=(1, 0),
                            bcs=[D.BC(D.DISPLGRAD, (1, 1, 1), (-2.5e-5, 0, 0, 0, 1e-4, 0, 0, 0, -2.5e-5), 8e-4, 1.0)],
                            bc_spaces=[D.Space(1, D.face_box(dims, 2.0, 1, -1)), D.Space(1, D.face_box(dims, 2.0, 1, +1))],
                            title="output check cci")
    return out


# PostAFD's console answers per case: the Tecplot step to read, then planes
# (1, normal, location) and single nodes (2, id), "y" between runs, "n" last
AFD_SCRIPTS = {
    "out_fgi": ("7", [("1", "1", "0.0005"), ("1", "2", "-0.0005"), ("1", "3", "0.0005"), ("2", "10"), ("2", "100")]),
    "out_cci": ("5", [("1", "1", "1"), ("1", "2", "-1"), ("1", "3", "1"), ("2", "20")]),
}


def afd_script(case):
    step, runs = AFD_SCRIPTS[case]
    lines = [step]
    for k, r in enumerate(runs):
        lines += list(r)
        lines.append("y" if k + 1 < len(runs) else "n")
    return "\n".join(lines) + "\n"


def make_outputs():
    import glob
    out_dir = os.path.join(HERE, "outputs")
    tmp = tempfile.mkdtemp(prefix="pdgolden_out_")
    for name, deck in output_cases().items():
        cdir = os.path.join(out_dir, name)
        deck.write(cdir)
        wd = os.path.join(tmp, name)
        deck.write(wd)
        r = subprocess.run([HARNESS, "solve", wd], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"harness solve {name} failed: {r.stderr[-400:]}")
        for old in glob.glob(os.path.join(cdir, "ref_*")):
            os.remove(old)
        files = sorted(glob.glob(os.path.join(wd, "pds_*.dat")))
        for f in files:
            shutil.copy(f, os.path.join(cdir, "ref_" + os.path.basename(f)))
        print(name, [os.path.basename(f) for f in files])
        # PostAFD on the last Tecplot dump (the answers it reads from the console)
        with open(os.path.join(wd, "afd_script.txt"), "w") as f:
            f.write(afd_script(name))
        r = subprocess.run([HARNESS, "afd", wd, os.path.join(wd, "afd_script.txt")], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"harness afd {name} failed: {r.stderr[-400:]}")
        step = AFD_SCRIPTS[name][0]
        shutil.copy(os.path.join(wd, f"pds_AFD_{step}.dat"), os.path.join(cdir, f"ref_afd_pds_AFD_{step}.dat"))
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__" and "--outputs" in sys.argv:
    make_outputs()


if __name__ == "__main__" and "--ai" in sys.argv:
    make_ai()
