"""GPU parity: the CUDA path, called through the C ABI, against the
reference's golden vectors (bit for bit in FP64) and against the oracle."""
import numpy as np
import pytest

import pdmtel_b200 as P
from conftest import deck_dir, kat, load_golden, CASES
from golden_model import model_from_golden, params
from pdmtel_b200 import decks as D

pytestmark = pytest.mark.gpu


def gpu_model(name_or_dir, init=True):
    dm = P.pdDataManager(deck_dir(name_or_dir) if name_or_dir in CASES else name_or_dir)
    if init:
        P.pdSolve.InitialProblem(dm)
    return dm


@pytest.mark.parametrize("name", CASES)
def test_device_bond_search_is_the_reference_family(name):
    g = load_golden(name)
    dm = gpu_model(name)
    rp, col, br = dm.family()
    assert np.array_equal(rp, g["fam_ptr"])
    assert np.array_equal(col, g["fam_col"])
    assert np.array_equal(br.astype(np.int32), g["broken"])
    assert dm.info().min_bond_length == g["min_bond"][0]
    assert np.array_equal(dm.bdry_eff(), g["bdry_eff"])
    if dm.info().mls:
        assert np.array_equal(dm.mls()[2], g["coeff"])


@pytest.mark.parametrize("name", CASES)
def test_force_stage_bit_exact(name):
    g = load_golden(name)
    t, dts = g["force_args"]
    dm = gpu_model(name)
    ctx = dm.context()
    ctx.set_state(g["u_test"], g["v_test"])
    ctx.init_dynamic()
    ctx.gather(t, g["u_test"])
    if len(g["ug"]):
        assert np.array_equal(ctx.get_gauss_displ(), g["ug"])
    k = ctx.force_stage(dts, t, g["u_test"])
    assert np.array_equal(k, g["k"])
    assert np.array_equal(ctx.get_vbuf(), g["vbuf"])
    U, _ = ctx.get_state()
    assert np.array_equal(U, g["U_after"])
    assert np.array_equal(ctx.get_energy_density(), g["eed"])


@pytest.mark.parametrize("name", CASES)
def test_rk4_trajectory_bit_exact(name):
    g = load_golden(name)
    dm = gpu_model(name)
    ctx = dm.context()
    dt = g["dt"][0]
    for it, t in enumerate(g["traj_times"], start=1):
        ke, ee = ctx.rk4_step(dt, t)
        # energies are sums over nodes: a tree sum on the device
        assert ke == pytest.approx(g["traj_ke"][it - 1], rel=1e-12, abs=1e-300)
        assert ee == pytest.approx(g["traj_ee"][it - 1], rel=1e-12, abs=1e-300)
        if f"traj_U_{it}" in g:
            U, V = ctx.get_state()
            assert np.array_equal(U, g[f"traj_U_{it}"])
            assert np.array_equal(V, g[f"traj_V_{it}"])
            if len(g[f"traj_ug_{it}"]):
                assert np.array_equal(ctx.get_gauss_displ(), g[f"traj_ug_{it}"])


def test_graph_replay_equals_single_steps():
    g = load_golden("fgi_slit")
    dt = g["dt"][0]
    a = gpu_model("fgi_slit").context()
    b = gpu_model("fgi_slit").context()
    t = 0.0
    for _ in range(5):
        t += dt
        a.rk4_step(dt, t)
    b.rk4_steps(dt, 0.0, 5)
    b.sync()
    Ua, Va = a.get_state()
    Ub, Vb = b.get_state()
    assert np.array_equal(Ua, Ub) and np.array_equal(Va, Vb)


def test_host_buffer_steps_equal_device_steps():
    g = load_golden("fgi_velo")
    dt = g["dt"][0]
    a = gpu_model("fgi_velo").context()
    a.rk4_steps(dt, 0.0, 3)
    a.sync()
    b = gpu_model("fgi_velo").context()
    n3 = 3 * b.n
    U0, V0 = np.zeros(n3), np.zeros(n3)
    U1, V1 = np.zeros(n3), np.zeros(n3)
    b.rk4_steps_host(dt, 0.0, 3, U0, V0, U1, V1)
    Ua, Va = a.get_state()
    assert np.array_equal(Ua, U1) and np.array_equal(Va, V1)


@pytest.mark.parametrize("prec", [P.PREC_FP64, P.PREC_FP32C])
def test_host_buffer_steps_continue_from_an_uploaded_state(prec):
    """A context handed a mid-run state through host buffers steps exactly
    like the context that reached that state by stepping: the uploaded U
    replaces the Gauss-point displacements (and FP32 node blocks) too, not
    only the nodal state."""
    g = load_golden("fgi_velo")
    dt = g["dt"][0]
    a = gpu_model("fgi_velo").context()
    a.set_precision(prec)
    a.rk4_steps(dt, 0.0, 4)
    a.sync()
    Ua, Va = a.get_state()
    a.rk4_steps(dt, 4 * dt, 2)
    a.sync()
    Ua6, Va6 = a.get_state()
    b = gpu_model("fgi_velo").context()  # at rest: its Gauss points are all zero
    b.set_precision(prec)
    n3 = 3 * b.n
    U1, V1 = np.zeros(n3), np.zeros(n3)
    b.rk4_steps_host(dt, 4 * dt, 1, Ua, Va, U1, V1)
    # second call: a round trip of the first call's output
    U2, V2 = np.zeros(n3), np.zeros(n3)
    b.rk4_steps_host(dt, 5 * dt, 1, U1, V1, U2, V2)
    assert np.array_equal(U2, Ua6) and np.array_equal(V2, Va6)
    assert np.abs(Ua).max() > 0


def test_sample_like_deck_known_answers():
    """The reference sample deck's parameters: 1,655,072 bonds and the
    energies of the first two steps (CCI, displacement-gradient layers)."""
    K = kat()["sample_like"]
    dm = gpu_model(deck_dir("sample_like"))
    assert dm.info().num_halves == 2 * K["bonds"]
    assert dm.CalcStableTimeStep() == K["dt"]
    ctx = dm.context()
    t = 0.0
    for it in range(2):
        t += K["dt"]
        ke, ee = ctx.rk4_step(K["dt"], t)
        assert ke == pytest.approx(K["ke"][it], rel=1e-12)
        assert ee == pytest.approx(K["ee"][it], rel=1e-12)
    U, V = ctx.get_state()
    assert np.abs(U).sum() == pytest.approx(K["u2_sum_abs"], rel=1e-12)
    assert np.abs(V).sum() == pytest.approx(K["v2_sum_abs"], rel=1e-12)


def test_bond_counts_of_larger_lattices(tmp_path):
    for dims, bonds in (((20, 10, 10), 168392), ((64, 64, 8), 3196784)):
        d = D.config_bar(dims=dims, traction_as_veloc=0.01)
        d.write(str(tmp_path / f"{dims[0]}"))
        dm = P.pdDataManager(str(tmp_path / f"{dims[0]}"))
        dm.InitNode()
        dm.InitBond()
        assert dm.info().num_halves == 2 * bonds


def test_traction_bar_matches_oracle(tmp_path):
    """The traction load (a project rule; the reference only parses it) on
    the full 20x10x10 bar: device and oracle agree bit for bit."""
    d = D.config_bar(dims=(20, 10, 10), traction=1e6, bdry_eff=1)
    d.write(str(tmp_path))
    dm = gpu_model(str(tmp_path))
    x, mat, bc = dm.nodes()
    rp, col, br = dm.family()
    cp, ci, co = dm.mls()
    I = dm.info()
    import oracle_lib as O
    xg, gw = O.gauss_points(x, I.grid_spacing, 2)
    spring = 18 * (72e9 / (3.0 * (1.0 - 2.0 * 0.25))) / (np.arccos(-1.0) * I.horizon ** 4.0)
    m = O.Model(n=I.num_nodes, x=x, dx=I.grid_spacing, delta=I.horizon, mls=1, npt=8, xg=xg, gw=gw,
                fam_ptr=rp, fam_col=col, broken=br, cb_ptr=cp, cb_idx=ci, coeff=co, bdry_eff=dm.bdry_eff(),
                mat=mat, mat_spring=np.array([spring]), mat_ecrit=np.array([1e20]), mat_density=np.array([2440.0]),
                mat_ymod=np.array([72e9]), bc=bc, bc_type=[1, 4], bc_dir=[1, 1, 1, 1, 0, 0],
                bc_val=[0] * 9 + [1e6] + [0] * 8, bc_end=[1.0, 1.0], bc_load=[2.0, 2.0])
    ctx = dm.context()
    t = 0.0
    for _ in range(3):
        t += 1e-8
        m.rk4_step(1e-8, t)
        ctx.rk4_step(1e-8, t)
    U, V = ctx.get_state()
    # the oracle's spring constant is formed in numpy here, so allow for one
    # ulp of difference in it
    assert np.linalg.norm(U - m.U) <= 1e-12 * np.linalg.norm(m.U)
    assert np.linalg.norm(V - m.V) <= 1e-12 * np.linalg.norm(m.V)
    assert np.abs(U).max() > 0


@pytest.mark.parametrize("name", ["fgi_velo", "fgi_slit", "fgi3_ramp", "cci_mdf"])
def test_fp32c_within_1e6_of_fp64(name):
    g = load_golden(name)
    dt = g["dt"][0]
    a = gpu_model(name).context()
    b = gpu_model(name)
    b.SetPrecision(P.PREC_FP32C)
    b = b.context()
    a.rk4_steps(dt, 0.0, 50)
    b.rk4_steps(dt, 0.0, 50)
    Ua, Va = a.get_state()
    Ub, Vb = b.get_state()
    eu = np.linalg.norm(Ub - Ua) / np.linalg.norm(Ua)
    ev = np.linalg.norm(Vb - Va) / np.linalg.norm(Va)
    assert eu <= 1e-6, eu
    assert ev <= 1e-5, ev


def test_static_operator_matches_oracle(tmp_path):
    d = D.config_bar(dims=(10, 6, 6), traction=1e6, bdry_eff=0)
    d.write(str(tmp_path))
    dm = gpu_model(str(tmp_path))
    x, mat, bc = dm.nodes()
    rp, col, br = dm.family()
    I = dm.info()
    import oracle_lib as O
    spring = 18 * (72e9 / 1.5) / (np.arccos(-1.0) * I.horizon ** 4.0)
    m = O.Model(n=I.num_nodes, x=x, dx=I.grid_spacing, delta=I.horizon, mls=0, npt=1, fam_ptr=rp, fam_col=col,
                broken=br, mat=mat, mat_spring=np.array([spring]), mat_ecrit=np.array([1e20]),
                mat_density=np.array([2440.0]), mat_ymod=np.array([72e9]), bc=bc, bc_type=[1, 4],
                bc_dir=[1, 1, 1, 1, 0, 0], bc_val=[0] * 9 + [1e6] + [0] * 8, bc_end=[1.0, 1.0], bc_load=[2.0, 2.0])
    ctx = dm.context()
    rng = np.random.default_rng(3)
    xv = rng.standard_normal(3 * I.num_nodes) * 1e-7
    y_gpu = ctx.static_matvec(1e-8, xv)
    y_or = m.static_apply(1e-8, xv)
    assert np.linalg.norm(y_gpu - y_or) <= 1e-12 * np.linalg.norm(y_or)
    b_gpu = ctx.static_rhs(1e-8)
    b_or = m.static_rhs(1e-8)
    assert np.linalg.norm(b_gpu - b_or) <= 1e-12 * np.linalg.norm(b_or)
    u64, it64, r64 = ctx.static_solve(1e-8, P.PREC_FP64, 1e-10)
    assert r64 <= 1e-10
    res = np.linalg.norm(m.static_apply(1e-8, u64) - b_or) / np.linalg.norm(b_or)
    assert res <= 2e-10
    u32, it32, r32 = ctx.static_solve(1e-8, P.PREC_FP32C, 1e-10)
    assert r32 <= 1e-10
    assert np.linalg.norm(u32 - u64) <= 1e-8 * np.linalg.norm(u64)


@pytest.mark.parametrize("dims", [(14, 8, 6), (16, 12, 10)])
def test_static_stencil_equals_family_kernel(tmp_path, dims):
    """On a complete box the static operator runs as a lattice stencil: the
    split form (D_i x_i - sum W_o x_j; 2, 4 or 8 nodes per thread) and the
    difference form agree with the family-list kernel, and the solvers
    converge.  The larger box has interior nodes (the shared diagonal block),
    the smaller one none."""
    d = D.config_bar(dims=dims, traction=1e6, bdry_eff=0)
    d.write(str(tmp_path))
    dm = gpu_model(str(tmp_path))
    ctx = dm.context()
    assert ctx.static_prepare()
    assert ctx.get_option(P.OPT_STATIC_SPLIT) == 4
    n3 = 3 * ctx.n
    xv = np.random.default_rng(5).standard_normal(n3) * 1e-7
    ys = {}
    for split in (4, 2, 8, 0):
        ctx.set_option(P.OPT_STATIC_SPLIT, split)
        ys[split] = ctx.static_matvec(1e-8, xv)
    # a rigid translation of the free nodes: no force on nodes away from the
    # clamped face, in the split form too (D_i matches its neighbour sums)
    ctx.set_option(P.OPT_STATIC_SPLIT, 4)
    t = np.repeat([1e-6, -2e-6, 3e-6], ctx.n)
    yt = ctx.static_matvec(1e-8, t)
    ctx.set_option(P.OPT_STATIC_STENCIL, 0)
    y_fl = ctx.static_matvec(1e-8, xv)
    yt_fl = ctx.static_matvec(1e-8, t)
    for split, y in ys.items():
        assert np.linalg.norm(y - y_fl) <= 1e-13 * np.linalg.norm(y_fl), split
    assert np.linalg.norm(yt - yt_fl) <= 1e-12 * np.linalg.norm(y_fl)
    u_fl, it_fl, r_fl = ctx.static_solve(1e-8, P.PREC_FP64, 1e-10)
    ctx.set_option(P.OPT_STATIC_STENCIL, 1)
    u64, it64, r64 = ctx.static_solve(1e-8, P.PREC_FP64, 1e-10)
    u32, it32, r32 = ctx.static_solve(1e-8, P.PREC_FP32C, 1e-10)
    assert r64 <= 1e-10 and r32 <= 1e-10
    assert np.linalg.norm(u64 - u_fl) <= 1e-8 * np.linalg.norm(u_fl)
    assert np.linalg.norm(u32 - u64) <= 1e-8 * np.linalg.norm(u64)
    # FP64 iterations until the residual is below 0.1, FP32 after: the
    # mixed-precision CG keeps close to the FP64 count
    assert it32 <= 1.2 * it64 + 10, (it32, it64)
    # FP32 from the first iteration still converges (with more iterations)
    ctx.set_option(P.OPT_STATIC_F32_BELOW, 0)
    u32a, it32a, r32a = ctx.static_solve(1e-8, P.PREC_FP32C, 1e-10)
    assert r32a <= 1e-10
    assert np.linalg.norm(u32a - u64) <= 1e-8 * np.linalg.norm(u64)


def test_static_operator_without_stencil_shape_matches_oracle():
    """A specimen with a hole (deleted nodes) keeps the family-list kernel."""
    g = load_golden("fgi1_hole")
    dm = gpu_model("fgi1_hole")
    x, mat, bc = dm.nodes()
    rp, col, br = dm.family()
    I = dm.info()
    m = model_from_golden(g)
    ctx = dm.context()
    assert not ctx.static_prepare()
    xv = np.random.default_rng(9).standard_normal(3 * I.num_nodes) * 1e-7
    y_gpu = ctx.static_matvec(1e-8, xv)
    y_or = m.static_apply(1e-8, xv)
    assert np.linalg.norm(y_gpu - y_or) <= 1e-12 * np.linalg.norm(y_or)
    u32, it32, r32 = ctx.static_solve(1e-8, P.PREC_FP32C, 1e-10)
    assert r32 <= 1e-10
    res = np.linalg.norm(m.static_apply(1e-8, u32) - m.static_rhs(1e-8)) / np.linalg.norm(m.static_rhs(1e-8))
    assert res <= 2e-10


@pytest.mark.parametrize("name", ["fgi_slit", "fgi3_ramp"])
def test_fp32c_gather_variants_agree(name):
    """The FP32-form gather per four points and per point: the same FMAs in
    the same contributor order, so the same trajectory bit for bit."""
    g = load_golden(name)
    dt = g["dt"][0]
    out = []
    for per_point in (0, 1):
        dm = gpu_model(name)
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        ctx.set_option(P.OPT_GATHER_PER_POINT, per_point)
        ctx.rk4_steps(dt, 0.0, 20)
        ctx.sync()
        out.append(ctx.get_state())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name,tiles", [("fgi_slit", [(8, 8, 3), (4, 8, 3)]), ("fgi_velo", [(8, 8, 4), (4, 4, 4)])])
def test_fp32c_tiled_force_equals_pair_kernel(name, tiles):
    """The FP32 force with shared-memory lattice tiles: the same arithmetic
    per node as the global-memory pair kernel, so the same trajectory."""
    g = load_golden(name)
    dt = g["dt"][0]

    def run(tile):
        dm = gpu_model(name)
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        if tile:
            ctx.set_option(P.OPT_FORCE_TILE, tile[0] | (tile[1] << 8) | (tile[2] << 16))
            assert ctx.get_option(P.OPT_FORCE_TILE) != 0
        ctx.rk4_steps(dt, 0.0, 20)
        ctx.sync()
        return ctx.get_state()

    U0, V0 = run(None)
    assert np.abs(U0).max() > 0
    for t in tiles:
        U1, V1 = run(t)
        assert np.array_equal(U0, U1) and np.array_equal(V0, V1), t


def test_fp32c_tiled_force_rejects_bad_shapes():
    dm = gpu_model("fgi_velo")
    dm.SetPrecision(P.PREC_FP32C)
    ctx = dm.context()
    with pytest.raises(P.PdError):
        ctx.set_option(P.OPT_FORCE_TILE, 3 | (8 << 8) | (4 << 16))  # odd x
    with pytest.raises(P.PdError):
        ctx.set_option(P.OPT_FORCE_TILE, 2 | (2 << 8) | (2 << 16))  # fewer than 32 pairs
    d3 = gpu_model("fgi3_ramp")  # 3x3x3 points: the pair kernels do not apply
    d3.SetPrecision(P.PREC_FP32C)
    with pytest.raises(P.PdError):
        d3.context().set_option(P.OPT_FORCE_TILE, 8 | (8 << 8) | (4 << 16))


@pytest.mark.parametrize("name", ["fgi_slit", "fgi_velo"])
def test_fp32c_quad_force_equals_pair_kernel(name):
    """Four nodes per thread in the FP32 force: the same arithmetic per node
    as two per thread, so the same trajectory bit for bit."""
    g = load_golden(name)
    dt = g["dt"][0]
    out = []
    for quad in (0, 1):
        dm = gpu_model(name)
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        ctx.set_option(P.OPT_FORCE_QUAD, quad)
        ctx.rk4_steps(dt, 0.0, 20)
        ctx.sync()
        out.append(ctx.get_state())
    assert np.abs(out[0][0]).max() > 0
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name", ["fgi_slit", "fgi_velo"])
def test_fp32c_sell_gather_equals_csr_gather(name):
    """The FP32 gather from its SELL copy (16 nodes side by side per
    contributor slot): the same sums in the same order as from the CSR lists,
    also after the work order changes and the copy is rebuilt."""
    g = load_golden(name)
    dt = g["dt"][0]

    def run(sell, tile=None):
        dm = gpu_model(name)
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        ctx.set_option(P.OPT_GATHER_SELL, sell)
        if tile is not None:
            ctx.set_option(P.OPT_TILE, tile)
        ctx.rk4_steps(dt, 0.0, 20)
        ctx.sync()
        return ctx.get_state()

    U0, V0 = run(0)
    for sell, tile in ((1, None), (1, 2 | (1 << 8) | (1 << 16))):
        U1, V1 = run(sell, tile)
        assert np.array_equal(U0, U1) and np.array_equal(V0, V1), (sell, tile)


def _fp32c_state(make_dm, dt, steps, stencil=0, sfac=None):
    dm = make_dm()
    dm.SetPrecision(P.PREC_FP32C)
    ctx = dm.context()
    if sfac is not None:
        ctx.set_spring_factor(sfac)
    if stencil:
        ctx.set_option(P.OPT_FORCE_STENCIL, stencil)
        assert ctx.get_option(P.OPT_FORCE_STENCIL) == stencil
    ctx.rk4_steps(dt, 0.0, steps)
    ctx.sync()
    return ctx.get_state()


@pytest.mark.parametrize("name", ["fgi_slit", "fgi_velo"])
def test_fp32c_stencil_force_equals_pair_kernel(name):
    """The FP32 force on the lattice stencil (family as a bit mask over one
    offset list, geometric terms from a per-offset table, chunk-major node
    blocks): the same terms in the same order per node as the pair kernel,
    so the same trajectory bit for bit, in every block shape."""
    g = load_golden(name)
    dt = g["dt"][0]
    U0, V0 = _fp32c_state(lambda: gpu_model(name), dt, 20)
    assert np.abs(U0).max() > 0
    for shape in (1, 2, 3, 4):
        U1, V1 = _fp32c_state(lambda: gpu_model(name), dt, 20, stencil=shape)
        assert np.array_equal(U0, U1) and np.array_equal(V0, V1), shape


def _stencil_decks():
    # odd row length (the last node of a row has no pair partner), a slit
    yield "odd_rows_slit", D.config_plate(dims=(35, 22, 3), spacing=5e-4, slit_half_length=2.5e-3, dt=5e-9,
                                           vel=5.0), None
    # boundary-effect factors
    d = D.config_plate(dims=(20, 16, 4), spacing=5e-4, slit_half_length=1.5e-3, dt=5e-9, vel=5.0)
    d.bdry_eff = 1
    yield "bdry", d, None
    # a critical stretch that the loaded layers exceed
    d = D.config_plate(dims=(20, 16, 4), spacing=5e-4, slit_half_length=1.5e-3, dt=5e-9, vel=5.0)
    d.materials = [(72e9, 1e20, 2e-5, 2440.0)]
    yield "ecrit", d, None
    # per-node spring factors
    d = D.config_plate(dims=(24, 12, 4), spacing=5e-4, slit_half_length=1.5e-3, dt=5e-9, vel=5.0)
    yield "sfac", d, np.exp(0.2 * np.random.default_rng(3).standard_normal(24 * 12 * 4))


@pytest.mark.parametrize("case", list(range(4)))
def test_fp32c_stencil_force_variants_equal_pair_kernel(tmp_path, case):
    """Odd rows, boundary factors, a critical stretch within reach and
    spring factors: every template variant of the stencil kernel against
    the pair kernel, bit for bit.  With a critical stretch the pair kernel
    runs its general variant, which forms bond vectors from FP32 hi/lo
    splits of the coordinates instead of lattice offsets; there the two
    agree to 1e-6 (the FP32 form's bar against FP64)."""
    name, deck, sfac = list(_stencil_decks())[case]
    deck.write(str(tmp_path))
    dt = 5e-9
    make = lambda: gpu_model(str(tmp_path))  # noqa: E731
    U0, V0 = _fp32c_state(make, dt, 30, sfac=sfac)
    assert np.abs(U0).max() > 0
    for shape in (1, 3):
        U1, V1 = _fp32c_state(make, dt, 30, stencil=shape, sfac=sfac)
        if name == "ecrit":
            assert np.linalg.norm(U1 - U0) <= 1e-6 * np.linalg.norm(U0), shape
            assert np.linalg.norm(V1 - V0) <= 1e-6 * np.linalg.norm(V0), shape
        else:
            assert np.array_equal(U0, U1) and np.array_equal(V0, V1), (name, shape)


@pytest.mark.parametrize("shape", [1, 3])
def test_fp32c_stencil_force_exact_pass_on_large_strains(tmp_path, shape):
    """Points whose bond strain leaves the series range (|eps| >= 1/64) send
    their tile of the stencil kernel to its exact pass.  With large random
    displacements in one end of a plate (some tiles marked, most not) and
    three RK4 steps from that state, the stencil trajectory still equals the
    pair kernel's bit for bit."""
    D.config_plate(dims=(40, 24, 4), spacing=5e-4, slit_half_length=2.5e-3, dt=5e-9, vel=5.0).write(str(tmp_path))
    dt, h = 5e-9, 5e-4
    dm0 = gpu_model(str(tmp_path))
    x = dm0.nodes()[0].reshape(-1, 3)
    U = np.zeros_like(x)
    end = x[:, 0] < x[:, 0].min() + 8 * h
    U[end] = 0.02 * h * np.random.default_rng(11).standard_normal((int(end.sum()), 3))
    # nearest-neighbour stretches in the loaded end reach well past 1/128
    # (eps is about twice the stretch, so points leave the series range)
    i = np.flatnonzero(end)[:200]
    j = i + 1
    ok = np.isclose(x[j, 0] - x[i, 0], h)
    s = (np.linalg.norm(x[j] + U[j] - x[i] - U[i], axis=1) - h) / h
    assert np.abs(s[ok]).max() > 1.0 / 64

    def run(stencil):
        dm = gpu_model(str(tmp_path))
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        if stencil:
            ctx.set_option(P.OPT_FORCE_STENCIL, stencil)
        ctx.set_state(U.reshape(-1), np.zeros(U.size))
        ctx.rk4_steps(dt, 0.0, 3)
        ctx.sync()
        return ctx.get_state()

    U0, V0 = run(0)
    U1, V1 = run(shape)
    assert np.abs(V0).max() > 0
    assert np.array_equal(U0, U1) and np.array_equal(V0, V1)


def test_fp32c_stencil_force_rejects_and_resets(tmp_path):
    """Problems off a complete box lattice are refused (deleted nodes, 3x3x3
    points, CCI); a new bond search turns the stencil force off."""
    d = D.config_plate(dims=(20, 16, 4), spacing=5e-4, slit_half_length=1.5e-3, dt=5e-9)
    d.deletion_spaces = [D.Space(0, (1.2e-3, 0.0, 0.0, -1.0, 1.0), geo=2)]
    hole = tmp_path / "hole"
    d.write(str(hole))
    for dm in (gpu_model(str(hole)), gpu_model("fgi3_ramp"), gpu_model("cci_grad")):
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        with pytest.raises(P.PdError):
            ctx.set_option(P.OPT_FORCE_STENCIL, 1)
        assert ctx.get_option(P.OPT_FORCE_STENCIL) == 0
    dm = gpu_model("fgi_velo")
    ctx = dm.context()
    with pytest.raises(P.PdError):
        ctx.set_option(P.OPT_FORCE_STENCIL, 5)
    ctx.set_option(P.OPT_FORCE_STENCIL, 2)
    ctx.bond_search()
    assert ctx.get_option(P.OPT_FORCE_STENCIL) == 0


@pytest.mark.parametrize("name", ["fgi_slit", "fgi_velo"])
def test_fp32c_pattern_gather_equals_list_gather(name):
    """The FP32 gather taking contributors from shared id-offset patterns:
    the same contributors in the same order as the lists, so the same
    trajectory bit for bit, with and without the SELL copy, and after the
    MLS data are set again (the patterns are rebuilt)."""
    g = load_golden(name)
    dt = g["dt"][0]

    def run(pat, sell, reset_mls=False):
        dm = gpu_model(name)
        dm.SetPrecision(P.PREC_FP32C)
        ctx = dm.context()
        ctx.set_option(P.OPT_GATHER_SELL, sell)
        ctx.set_option(P.OPT_GATHER_STENCIL, pat)
        assert ctx.get_option(P.OPT_GATHER_STENCIL) == pat
        if reset_mls:
            ctx.set_mls(*dm.mls())
            assert ctx.get_option(P.OPT_GATHER_STENCIL) == pat
        ctx.rk4_steps(dt, 0.0, 20)
        ctx.sync()
        return ctx.get_state()

    U0, V0 = run(0, 0)
    assert np.abs(U0).max() > 0
    for pat, sell, reset in ((1, 0, False), (1, 1, False), (1, 1, True)):
        U1, V1 = run(pat, sell, reset)
        assert np.array_equal(U0, U1) and np.array_equal(V0, V1), (pat, sell, reset)


def test_autotune_on_a_box_lattice_changes_no_result(tmp_path):
    """The tuner's trials on a plate (node orders, every gather variant, the
    stencil force, the persistent launch) keep the state and leave a choice
    whose trajectory equals the untuned one bit for bit."""
    D.config_plate(dims=(48, 40, 4), spacing=5e-4, slit_half_length=3e-3, dt=5e-9, vel=5.0).write(str(tmp_path))
    dt = 5e-9
    U0, V0 = _fp32c_state(lambda: gpu_model(str(tmp_path)), dt, 12)
    dm = gpu_model(str(tmp_path))
    dm.SetPrecision(P.PREC_FP32C)
    ctx = dm.context()
    r = ctx.autotune(dt, 2)
    assert r["trials"] >= 10
    U1, V1 = ctx.get_state()
    assert not U1.any() and not V1.any()
    if r["persistent"]:
        ctx.rk4_steps_persistent(dt, 0.0, 12)
    else:
        ctx.rk4_steps(dt, 0.0, 12)
    ctx.sync()
    U2, V2 = ctx.get_state()
    assert np.array_equal(U0, U2) and np.array_equal(V0, V2), r
