"""Batching form: many specimens in one context.

CPU: the host assembly (placement on one lattice, offsets, tables, family and
per-specimen MLS) against the specimens' own models, with the oracle's bond
search standing in for the device search.  GPU: the device search over the
batch, and stepping the batch (graph-captured or in one persistent launch)
against the same specimens stepped one context at a time, bit for bit."""
import os

import numpy as np
import pytest

import pdmtel_b200 as P
from pdmtel_b200 import batch as B

SPACING = 1e-3


def _small_spec(count=5, seed=3, nmin=200, nmax=2000):
    return B.BatchSpec(dims=B.draw_dims(count, seed, nmin, nmax), spacing=SPACING, seed=seed)


def _open_specimens(tmp, spec):
    from pdmtel_b200.adjoint import gaussian_random_field
    from pdmtel_b200.decks import config_identify
    out = []
    for k, dims in enumerate(spec.dims):
        d = os.path.join(tmp, f"s{k}")
        config_identify(dims=tuple(dims), spacing=SPACING, vel=spec.vel, dt=spec.dt, steps=1).write(d)
        m = P.pdDataManager(d)
        m.InitNode()
        x, _, _ = m.nodes()
        m.SetSpringFactor(np.exp(0.15 * gaussian_random_field(x, SPACING, 4 * SPACING, 1.0, seed=k)))
        out.append(m)
    return out


def test_draw_dims_counts_and_aspects():
    dims = B.draw_dims(400, 1)
    n = np.array([a * b * c for a, b, c in dims], dtype=float)
    assert n.min() >= 0.7 * 1000 and n.max() <= 1.3 * 60000
    # log-uniform: the median node count sits near the geometric mean
    assert abs(np.log(np.median(n)) - 0.5 * (np.log(1000) + np.log(60000))) < 0.35
    r = np.array([max(d) / min(d) for d in dims])
    assert r.max() <= 4.0 * 1.5 and r.min() >= 1.0


def test_batch_placement_offsets_and_tables(tmp_path):
    spec = _small_spec()
    sp = _open_specimens(str(tmp_path), spec)
    bm = P.pdDataManager.batch(str(tmp_path / "batch"), sp)
    off = bm.batch_offsets()
    counts = [s.info().num_nodes for s in sp]
    assert list(np.diff(off)) == counts
    xb, mb, bb = bm.nodes()
    xb = xb.reshape(-1, 3)
    I = bm.info()
    # the specimens share one material, merged into one entry
    assert I.num_nodes == sum(counts) and I.num_materials == 1 and I.num_bcs == 2 * len(sp)
    boxes = []
    for k, s in enumerate(sp):
        xs, ms, bs = s.nodes()
        xs = xs.reshape(-1, 3)
        seg = xb[off[k]:off[k + 1]]
        shift = seg - xs
        # one rigid shift per specimen, a whole number of lattice steps from
        # the first specimen's lattice
        assert np.allclose(shift, shift[0], rtol=0, atol=1e-12)
        steps = (seg[0] - xb[0]) / SPACING
        assert np.allclose(steps, np.rint(steps), atol=1e-6)
        assert np.array_equal(mb[off[k]:off[k + 1]], ms)
        assert np.array_equal(bb[off[k]:off[k + 1]], np.where(bs >= 0, bs + 2 * k, -1))
        boxes.append((seg.min(axis=0), seg.max(axis=0)))
    # every pair of specimens is further apart than the horizon plus a cell
    for a in range(len(boxes)):
        for b in range(a + 1, len(boxes)):
            gap = np.maximum(boxes[b][0] - boxes[a][1], boxes[a][0] - boxes[b][1]).max()
            assert gap > I.horizon + 1.5 * SPACING
    mats, bcs, ab, wt = bm.tables()
    assert len(mats) == 1 and len(bcs) == 2 * len(sp)
    assert np.allclose(ab, [1 / np.sqrt(3), -1 / np.sqrt(3)], rtol=1e-15) and np.all(wt == 1.0)


def test_batch_family_and_mls_equal_the_specimens(tmp_path):
    """With the oracle's bond search as the family, the batch's per-specimen
    MLS equals each specimen model's own, bit for bit."""
    import oracle_lib as O
    spec = _small_spec(count=4, seed=5, nmin=150, nmax=900)
    sp = _open_specimens(str(tmp_path), spec)
    bm = P.pdDataManager.batch(str(tmp_path / "batch"), sp)
    I = bm.info()
    xb, _, _ = bm.nodes()
    rp, col, mb = O.bond_search(xb, SPACING, I.horizon)
    bm.SetFamily(rp, col, None, mb)
    bm.InitIntegrationPoint()
    off = bm.batch_offsets()
    cpb, cib, cob = bm.mls()
    npt = I.num_gauss
    for k, s in enumerate(sp):
        xs, _, _ = s.nodes()
        r2, c2, m2 = O.bond_search(xs, SPACING, I.horizon)
        a, b = off[k], off[k + 1]
        # block-diagonal batch family = the specimen's own family, offset
        assert np.array_equal(rp[a:b + 1] - rp[a], r2)
        assert np.array_equal(col[rp[a]:rp[b]] - a, c2)
        s.SetFamily(r2, c2, None, m2)
        s.InitIntegrationPoint()
        cp, ci, co = s.mls()
        assert np.array_equal(cpb[a:b + 1] - cpb[a], cp)
        assert np.array_equal(cib[cpb[a]:cpb[b]] - a, ci)
        assert np.array_equal(cob[cpb[a] * npt:cpb[b] * npt], co)


def test_batch_rejects_mismatched_specimens(tmp_path):
    from pdmtel_b200.decks import config_identify
    d1, d2 = str(tmp_path / "a"), str(tmp_path / "b")
    config_identify(dims=(6, 5, 4), spacing=1e-3).write(d1)
    config_identify(dims=(6, 5, 4), spacing=2e-3).write(d2)
    a, b = P.pdDataManager(d1), P.pdDataManager(d2)
    with pytest.raises(P.PdError):
        P.pdDataManager.batch(str(tmp_path / "batch"), [a, b])


# ------------------------------------------------------------------ GPU


@pytest.mark.gpu
def test_device_bond_search_of_a_batch(tmp_path):
    spec = _small_spec(count=6, seed=7, nmin=300, nmax=3000)
    sp = _open_specimens(str(tmp_path), spec)
    bm = P.pdDataManager.batch(str(tmp_path / "batch"), sp)
    bm.InitBond()
    rp, col, _ = bm.family()
    off = bm.batch_offsets()
    for k, s in enumerate(sp):
        s.InitBond()
        r2, c2, _ = s.family()
        a, b = off[k], off[k + 1]
        assert np.array_equal(rp[a:b + 1] - rp[a], r2)
        assert np.array_equal(col[rp[a]:rp[b]] - a, c2)


def _state(ctx):
    U, V = ctx.get_state()
    return U.reshape(-1, 3), V.reshape(-1, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [P.PREC_FP64, P.PREC_FP32C])
def test_batch_steps_equal_specimen_steps(tmp_path, precision):
    spec = _small_spec(count=6, seed=11, nmin=300, nmax=4000)
    bt = B.Batch(str(tmp_path), spec, precision=precision)
    nsteps = 20
    bt.run(nsteps, persistent=False)
    Ub, Vb = _state(bt.ctx)
    assert np.abs(Ub).max() > 0
    for k, ctx in enumerate(bt.specimen_contexts(precision)):
        ctx.rk4_steps(spec.dt, 0.0, nsteps)
        ctx.sync()
        U, V = _state(ctx)
        a, b = bt.offsets[k], bt.offsets[k + 1]
        assert np.array_equal(U, Ub[a:b]) and np.array_equal(V, Vb[a:b]), k


@pytest.mark.gpu
def test_persistent_launch_equals_graph_steps(tmp_path):
    spec = _small_spec(count=8, seed=13, nmin=300, nmax=6000)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C)
    nsteps = 25
    bt.run(nsteps, persistent=False)
    Ug, Vg = _state(bt.ctx)
    bt.ctx.reset_state()
    bt.run(nsteps, persistent=True)
    Up, Vp = _state(bt.ctx)
    assert np.array_equal(Ug, Up) and np.array_equal(Vg, Vp)
    # odd node count, small chunks, one block per SM
    bt.ctx.set_option(P.OPT_PERSIST_BLOCKS_PER_SM, 1)
    bt.ctx.set_option(P.OPT_PERSIST_FORCE_CHUNK, 128)
    bt.ctx.set_option(P.OPT_PERSIST_GATHER_CHUNK, 128)
    bt.ctx.reset_state()
    bt.run(nsteps, persistent=True)
    Up, Vp = _state(bt.ctx)
    assert np.array_equal(Ug, Up) and np.array_equal(Vg, Vp)


@pytest.mark.gpu
def test_autotune_changes_no_result(tmp_path):
    spec = _small_spec(count=5, seed=17, nmin=500, nmax=5000)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C)
    bt.run(10, persistent=False)
    U0, V0 = _state(bt.ctx)
    bt.ctx.reset_state()
    r = bt.tune(steps=2)
    assert r["trials"] >= 7 and r["ms_per_step"] > 0
    # tuning leaves the state where it was
    U1, V1 = _state(bt.ctx)
    assert not U1.any() and not V1.any()
    bt.run(10)
    U2, V2 = _state(bt.ctx)
    assert np.array_equal(U0, U2) and np.array_equal(V0, V2)


@pytest.mark.gpu
def test_persistent_launch_refuses_unsupported_setups(tmp_path):
    spec = _small_spec(count=2, seed=19)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP64)
    with pytest.raises(P.PdError):
        bt.ctx.rk4_steps_persistent(spec.dt, 0.0, 2)
    bt.ctx.set_precision(P.PREC_FP32C)
    bt.ctx.set_energy(True)
    with pytest.raises(P.PdError):
        bt.ctx.rk4_steps_persistent(spec.dt, 0.0, 2)


def test_batch_keeps_distinct_materials_apart(tmp_path):
    """Identical materials of different specimens merge into one entry;
    different ones stay distinct and each node keeps its own."""
    from pdmtel_b200.decks import config_identify
    sp = []
    for k, E in enumerate((72e9, 72e9, 50e9)):
        deck = config_identify(dims=(6, 5, 4), spacing=1e-3)
        deck.materials = [(E, 1e20, 1e20, 2440.0)]
        d = str(tmp_path / f"s{k}")
        deck.write(d)
        m = P.pdDataManager(d)
        m.InitNode()
        sp.append(m)
    bm = P.pdDataManager.batch(str(tmp_path / "batch"), sp)
    mats, _, _, _ = bm.tables()
    assert len(mats) == 2
    _, mb, _ = bm.nodes()
    off = bm.batch_offsets()
    assert set(mb[off[0]:off[2]]) == {0} and set(mb[off[2]:off[3]]) == {1}
    assert mats[1]["spring"] < mats[0]["spring"]


@pytest.mark.gpu
def test_persistent_barrier_wait_runs_out_and_the_context_recovers(tmp_path):
    """The persistent launch's grid barriers give up after their wait limit:
    with block 0 held back from the first barrier every wait runs out, the
    call returns PD_ERR_TIMEOUT instead of hanging, and the next launch on the
    same context runs normally."""
    import time
    spec = _small_spec(count=3, seed=23)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C)
    bt.run(5, persistent=False)
    Ug, Vg = _state(bt.ctx)
    bt.ctx.set_option(P.OPT_PERSIST_WAIT_US, 200000)
    bt.ctx.set_option(P.OPT_PERSIST_TEST_STALL, 1)
    bt.ctx.reset_state()
    t0 = time.time()
    with pytest.raises(P.PdError) as e:
        bt.ctx.rk4_steps_persistent(spec.dt, 0.0, 5)
    assert e.value.code == -4  # PD_ERR_TIMEOUT
    assert time.time() - t0 < 30
    bt.ctx.set_option(P.OPT_PERSIST_TEST_STALL, 0)
    bt.ctx.reset_state()
    bt.run(5, persistent=True)
    Up, Vp = _state(bt.ctx)
    assert np.array_equal(Ug, Up) and np.array_equal(Vg, Vp)


@pytest.mark.gpu
def test_batch_stencil_force_equals_pair_force(tmp_path):
    """Specimens that are complete boxes run the lattice-stencil force box by
    box (pd_set_boxes, called by the batch setup): every block shape gives the
    trajectory of the general pair kernel bit for bit, thin boxes (narrower
    than the family reach) included."""
    dims = [(12, 9, 5), (10, 8, 8), (20, 10, 4), (4, 7, 6), (16, 3, 3), (9, 12, 3)]
    spec = B.BatchSpec(dims=dims, spacing=SPACING, seed=23)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C)
    assert bt.ctx.get_option(P.OPT_FORCE_STENCIL) == 0
    nsteps = 20
    bt.run(nsteps, persistent=False)
    U0, V0 = _state(bt.ctx)
    assert np.abs(U0).max() > 0
    for shape in (1, 2, 3, 4):
        bt.ctx.reset_state()
        bt.ctx.set_option(P.OPT_FORCE_STENCIL, shape)
        assert bt.ctx.get_option(P.OPT_FORCE_STENCIL) == shape
        bt.run(nsteps, persistent=False)
        U1, V1 = _state(bt.ctx)
        assert np.array_equal(U0, U1) and np.array_equal(V0, V1), shape


@pytest.mark.gpu
def test_batch_stencil_force_refuses_undeclared_boxes(tmp_path):
    spec = B.BatchSpec(dims=[(12, 9, 5), (10, 8, 8)], spacing=SPACING, seed=31)
    bt = B.Batch(str(tmp_path), spec, precision=P.PREC_FP32C)
    n0 = bt.offsets[1]
    # ranges that are not boxes are refused
    with pytest.raises(P.PdError):
        bt.ctx.set_boxes([0, n0 - 5, bt.offsets[2]])
    with pytest.raises(P.PdError):
        bt.ctx.set_boxes([0, n0])
    # without boxes the batch is no box lattice
    bt.ctx.set_boxes([])
    with pytest.raises(P.PdError):
        bt.ctx.set_option(P.OPT_FORCE_STENCIL, 1)
    assert bt.ctx.get_option(P.OPT_FORCE_STENCIL) == 0
    bt.ctx.set_boxes(bt.offsets)
    bt.ctx.set_option(P.OPT_FORCE_STENCIL, 1)
    assert bt.ctx.get_option(P.OPT_FORCE_STENCIL) == 1
