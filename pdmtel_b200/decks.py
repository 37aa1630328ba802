"""Writers for pdMTEL input decks (``pds_input.txt``).

The keyword grammar is the reference's (pdDataManager.cpp:4-758): a keyword on
its own line, its values on the next line, 1-based ids.  ``write_deck`` emits
exactly that grammar, and the ``config_*`` helpers build the synthetic lattices
this package benchmarks and tests on (uniform cubic lattices; no external
datasets are involved).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

# boundary-condition types, pdDataManager.h:231
DISPL, VELOC, DISPLGRAD, TRACTION = 1, 2, 3, 4


@dataclass
class BC:
    type: int
    dirs: Sequence[int]
    values: Sequence[float]  # 3 values, or 9 for DISPLGRAD
    end_time: float = 1.0
    load_type: float = 2.0  # 1 = ramp, otherwise step

    def line(self) -> str:
        vals = " ".join(repr(float(v)) for v in self.values)
        d = " ".join(str(int(x)) for x in self.dirs)
        return f"{self.type} {d} {vals} {self.end_time!r} {self.load_type!r}"


@dataclass
class Space:
    """Cuboid (geo 1) or cylinder (geo 2) region; ``ref`` is the 1-based
    material or boundary-condition id it carries."""
    ref: int
    box: Sequence[float]  # x1lo x1hi x2lo x2hi x3lo x3hi, or rad x1c x2c x3lo x3hi
    geo: int = 1

    def line(self) -> str:
        return f"{self.geo} {self.ref} " + " ".join(repr(float(v)) for v in self.box)


@dataclass
class Deck:
    dims: Sequence[int]
    spacing: float
    horizon: Optional[float] = None
    center: Sequence[float] = (0.0, 0.0, 0.0)
    total_time: float = 1.0
    total_step: int = 100
    dump: int = 100000
    fixed_dt: Optional[float] = None
    safety: Optional[float] = None
    # (ymod, sigmay, ecrit, density) per material, bond-based (type 1)
    materials: List[Sequence[float]] = field(default_factory=lambda: [(72e9, 1e20, 1e20, 2440.0)])
    material_spaces: List[Space] = field(default_factory=list)
    bcs: List[BC] = field(default_factory=list)
    bc_spaces: List[Space] = field(default_factory=list)
    deletion_spaces: List[Space] = field(default_factory=list)
    slits: List[Sequence[float]] = field(default_factory=list)
    damping: float = 0.0
    bdry_eff: int = 0
    cci: Optional[Sequence[int]] = None  # (on, modified); None -> FGI
    intg_point: int = 2
    support_domain: Optional[float] = None
    ai_mls: Optional[int] = None  # adaptive trapezoid (ai_on 1 <mls>); intg_point is its trapezoid index
    title: str = "pdmtel_b200 synthetic deck"

    def text(self) -> str:
        L: List[str] = []

        def kv(k: str, v: str) -> None:
            L.append(k)
            L.append(" " + v)

        kv("problem_title", self.title.replace(" ", "_"))
        kv("grid_center", " ".join(repr(float(c)) for c in self.center))
        kv("grid_dimension", " ".join(str(int(d)) for d in self.dims))
        kv("grid_spacing", repr(float(self.spacing)))
        if self.horizon is not None:
            kv("horizon", repr(float(self.horizon)))
        kv("total_time", repr(float(self.total_time)))
        kv("total_step", str(int(self.total_step)))
        kv("step_dump_frequency", str(int(self.dump)))
        if self.safety is not None:
            kv("safety_factor", repr(float(self.safety)))
        if self.fixed_dt is not None:
            kv("fixed_time_step", repr(float(self.fixed_dt)))
        kv("number_of_materials", str(len(self.materials)))
        for i, m in enumerate(self.materials):
            kv(f"material_{i + 1}", "1 " + " ".join(repr(float(x)) for x in m))
        spaces = self.material_spaces or [Space(1, (-1e9, 1e9, -1e9, 1e9, -1e9, 1e9))]
        kv("number_of_material_spaces", str(len(spaces)))
        for i, s in enumerate(spaces):
            kv(f"material_space_{i + 1}", s.line())
        if self.deletion_spaces:
            kv("number_of_deletion_spaces", str(len(self.deletion_spaces)))
            for i, s in enumerate(self.deletion_spaces):
                kv(f"deletion_space_{i + 1}", f"{s.geo} " + " ".join(repr(float(v)) for v in s.box))
        kv("number_of_boundary_conditions", str(len(self.bcs)))
        for i, b in enumerate(self.bcs):
            kv(f"boundary_condition_{i + 1}", b.line())
        kv("number_of_boundary_spaces", str(len(self.bc_spaces)))
        for i, s in enumerate(self.bc_spaces):
            kv(f"boundary_space_{i + 1}", s.line())
        if self.slits:
            kv("number_of_slits", str(len(self.slits)))
            for i, s in enumerate(self.slits):
                kv(f"slit_{i + 1}", "1 " + " ".join(repr(float(v)) for v in s))
        kv("damping_coeff", repr(float(self.damping)))
        kv("bdryEff_on", str(int(self.bdry_eff)))
        if self.cci is not None:
            kv("cci_on", f"{int(self.cci[0])} {int(self.cci[1])}")
        elif self.ai_mls is not None:
            kv("cci_on", "0 0")
            kv("fgi_on", "0")
            kv("ai_on", f"1 {int(self.ai_mls)}")
            kv("intg_point", str(int(self.intg_point)))
            if self.support_domain is not None:
                kv("support_domain_size", repr(float(self.support_domain)))
        else:
            kv("cci_on", "0 0")
            kv("fgi_on", "1")
            kv("intg_point", str(int(self.intg_point)))
            if self.support_domain is not None:
                kv("support_domain_size", repr(float(self.support_domain)))
        return "\n".join(L) + "\n"

    def write(self, directory: str) -> str:
        os.makedirs(directory, exist_ok=True)
        path = os.path.join(directory, "pds_input.txt")
        with open(path, "w") as f:
            f.write(self.text())
        return path


def face_box(dims: Sequence[int], spacing: float, axis: int, side: int, layers: int = 1,
             center: Sequence[float] = (0.0, 0.0, 0.0)) -> List[float]:
    """Cuboid covering ``layers`` node layers on the low (side=-1) or high
    (side=+1) face normal to ``axis``; node coordinates follow
    pdDataManager.cpp:851-853."""
    box: List[float] = []
    for a in range(3):
        n = dims[a]
        lo = (1 - (n + 1) * 0.5) * spacing + center[a]
        hi = (n - (n + 1) * 0.5) * spacing + center[a]
        if a == axis:
            if side < 0:
                box += [lo - 0.5 * spacing, lo + (layers - 0.5) * spacing]
            else:
                box += [hi - (layers - 0.5) * spacing, hi + 0.5 * spacing]
        else:
            box += [lo - 0.5 * spacing, hi + 0.5 * spacing]
    return box


def config_bar(dims=(20, 10, 10), spacing=1e-3, traction=1e6, dt=1e-8, steps=100,
               bdry_eff=1, traction_as_veloc: Optional[float] = None) -> Deck:
    """The small plain-FP64 case: a bar on a cubic lattice, left face fixed
    (DISPL 0 in xyz), right face under a uniform tensile traction (type 4,
    applied as a body-force density traction/spacing on the face layer)."""
    bcs = [BC(DISPL, (1, 1, 1), (0.0, 0.0, 0.0), 1.0, 2.0)]
    if traction_as_veloc is None:
        bcs.append(BC(TRACTION, (1, 0, 0), (traction, 0.0, 0.0), 1.0, 2.0))
    else:
        bcs.append(BC(VELOC, (1, 0, 0), (traction_as_veloc, 0.0, 0.0), 1.0, 2.0))
    return Deck(dims=dims, spacing=spacing, horizon=3.015 * spacing, total_time=1.0,
                total_step=steps, fixed_dt=dt, bcs=bcs,
                bc_spaces=[Space(1, face_box(dims, spacing, 0, -1)), Space(2, face_box(dims, spacing, 0, +1))],
                bdry_eff=bdry_eff, intg_point=2)


def config_plate(dims=(400, 400, 4), spacing=5e-4, slit_half_length=0.02, vel=0.05, dt=5e-9,
                 steps=2000, layers=1) -> Deck:
    """The pre-cracked plate: a central slit along x in the plane y=0 through
    the full thickness, and +-vel in y on the top and bottom node layers."""
    bcs = [BC(VELOC, (0, 1, 0), (0.0, vel, 0.0), 1.0, 2.0), BC(VELOC, (0, 1, 0), (0.0, -vel, 0.0), 1.0, 2.0)]
    return Deck(dims=dims, spacing=spacing, horizon=3.015 * spacing, total_time=1.0, total_step=steps,
                fixed_dt=dt, bcs=bcs,
                bc_spaces=[Space(1, face_box(dims, spacing, 1, +1, layers)),
                           Space(2, face_box(dims, spacing, 1, -1, layers))],
                slits=[(-slit_half_length, slit_half_length, 0.0, 0.0, -1.0, 1.0)],
                bdry_eff=0, intg_point=2)


def config_identify(dims=(64, 64, 8), spacing=1e-3, vel=0.02, dt=5e-8, steps=1000) -> Deck:
    """The identification specimen: low-x face fixed (DISPL 0 in xyz), the
    high-x face pulled at vel along x (VELOC), Gauss-point integration with
    2x2x2 points and MLS."""
    bcs = [BC(DISPL, (1, 1, 1), (0.0, 0.0, 0.0), 1.0, 2.0), BC(VELOC, (1, 0, 0), (vel, 0.0, 0.0), 1.0, 2.0)]
    return Deck(dims=dims, spacing=spacing, horizon=3.015 * spacing, total_time=1.0, total_step=steps,
                fixed_dt=dt, bcs=bcs,
                bc_spaces=[Space(1, face_box(dims, spacing, 0, -1)), Space(2, face_box(dims, spacing, 0, +1))],
                bdry_eff=0, intg_point=2)


def config_cube(n=128, spacing=1e-3, traction=1e6, intg_point=2) -> Deck:
    """The static cube: bottom face (low z) clamped, top face under a shear
    traction along x.  The static operator uses the family only, so
    intg_point=1 (no MLS) skips the Gauss-point setup."""
    dims = (n, n, n)
    bcs = [BC(DISPL, (1, 1, 1), (0.0, 0.0, 0.0), 1.0, 2.0), BC(TRACTION, (1, 0, 0), (traction, 0.0, 0.0), 1.0, 2.0)]
    return Deck(dims=dims, spacing=spacing, horizon=3.015 * spacing, total_time=1.0, total_step=1, fixed_dt=1.0,
                bcs=bcs, bc_spaces=[Space(1, face_box(dims, spacing, 2, -1)), Space(2, face_box(dims, spacing, 2, +1))],
                bdry_eff=0, intg_point=intg_point)
