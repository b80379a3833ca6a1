"""Tile shapes, the tile autotuner and batched stepping, through librn.so.

None of these change the arithmetic of a cell: every cell and cut-cell group
computes the same float operations whatever tile or batch block it lands in.
So in exact precision the results must be bit-identical to single-handle
stepping with the default tile, and that to the CPU oracle (where the tests
check it)."""
import numpy as np
import pytest

from helpers import run_oracle

pytestmark = pytest.mark.gpu


def make(rn, s, precision="exact", tile=None):
    g = rn.GPUSolver(s.Nx, s.Nr)
    g.setPrecision(precision)
    if tile:
        g.setTile(tile)
    g.setGeometry(s.geo)
    init = s.initialState()
    g.setState(init["A"], init["B"])
    if s.injector is not None:
        rn.GPUSpray(g).resize()
        g.spray.setInjector(s.injector)
    return g


def identical(a, b):
    return np.array_equal(a["A"], b["A"]) and np.array_equal(a["B"], b["B"])


def setups(rn, kind, sizes):
    from rocket_nozzle_cfd_solver_b200 import configs
    f = {"plain": configs.plain_small, "viscous": configs.viscous_plume, "spray": configs.injector_spray}[kind]
    return [rn.build_sim_setup(f(Nx, Nr)[0]) for Nx, Nr in sizes]


@pytest.mark.parametrize("kind", ["plain", "viscous"])
def test_tile_shapes_bit_identical(rn, oracle, kind):
    s = setups(rn, kind, [(160, 60)])[0]
    outs = []
    for tile in ("16x16", "16x8", "16x15", "32x15", "14x16"):
        g = make(rn, s, tile=tile)
        assert g.tile == tile
        g.step(40, s.P)
        outs.append((g.readAll(), g.readStepInfo()))
        g.close()
    for o in outs[1:]:
        assert identical(outs[0][0], o[0]) and np.array_equal(outs[0][1], o[1])
    assert identical(outs[0][0], run_oracle(oracle, s, 40).readAll())


def test_fast_tile_shapes_agree(rn):
    """Fast precision: every shape computes the same operations too, but
    the compiler contracts multiply-adds per kernel, and the 14x16 shape's
    kernels (which stage the cell geometry and keep the raw halo block in
    shared memory) are compiled apart from the others; so shapes agree to a
    few rounding steps, not bit for bit (exact precision is bit-identical
    across shapes: test_tile_shapes_bit_identical)."""
    from helpers import state_rel_l2
    s = setups(rn, "viscous", [(256, 96)])[0]
    outs = []
    for tile in ("16x16", "16x8", "16x15", "32x15", "14x16"):
        g = make(rn, s, precision="fast", tile=tile)
        g.step(60, s.P)
        outs.append(g.readAll())
        g.close()
    for tile, o in zip(("16x8", "16x15", "32x15", "14x16"), outs[1:]):
        e = state_rel_l2(o, outs[0])
        print(tile, "vs 16x16, fast precision:", {k: float(f"{v:.2e}") for k, v in e.items()})
        assert max(e.values()) <= 1e-5, (tile, e)


def test_autotune_restores_state(rn):
    s = setups(rn, "spray", [(128, 48)])[0]
    g = make(rn, s)
    ref = make(rn, s)
    g.step(12, s.P)
    ref.step(12, s.P)
    before, si = g.readAll(), g.readStepInfo()
    launches = g.kernelLaunches()
    chosen = g.autotune(s.P, steps=4)
    assert chosen in ("16x16", "16x8", "16x15", "32x15", "14x16") and g.tile == chosen
    assert identical(g.readAll(), before) and np.array_equal(g.readStepInfo(), si)
    assert g.kernelLaunches() == launches
    g.step(9, s.P)
    ref.step(9, s.P)
    assert identical(g.readAll(), ref.readAll())
    assert np.array_equal(g.spray.readParcels()["PA"], ref.spray.readParcels()["PA"])
    g.close()
    ref.close()


@pytest.mark.parametrize("kind,sizes,calls", [
    ("plain", [(96, 36), (160, 60), (256, 96)], [13, 5, 1, 6]),
    ("viscous", [(128, 48), (200, 76)], [7, 6, 12]),
    ("spray", [(128, 48), (96, 36)], [5, 4]),
])
def test_batch_matches_single_handles(rn, kind, sizes, calls):
    """Members of uneven sizes, call lengths that start and end inside the
    6-step graph period: every member ends bit-identical to a handle stepped
    on its own."""
    ss = setups(rn, kind, sizes)
    batch = rn.SolverBatch()
    members = [make(rn, s) for s in ss]
    singles = [make(rn, s) for s in ss]
    for g, s in zip(members, ss):
        batch.add(g, s.P)
    assert batch.size() == (len(ss), sum(s.Nx * s.Nr for s in ss))
    for n in calls:
        batch.step(n)
        for g, s in zip(singles, ss):
            g.step(n, s.P)
        # reads in between go through the member handles
        for g, h in zip(members, singles):
            assert identical(g.readAll(), h.readAll())
            assert np.array_equal(g.readStepInfo(), h.readStepInfo())
    if kind == "spray":
        for g, h in zip(members, singles):
            assert np.array_equal(g.spray.readParcels()["PB"], h.spray.readParcels()["PB"])
    batch.close()
    for g in members + singles:
        g.close()


def test_batch_member_leaves_and_steps_alone(rn):
    ss = setups(rn, "plain", [(96, 36), (128, 48)])
    batch = rn.SolverBatch()
    a, b = make(rn, ss[0]), make(rn, ss[1])
    ref = make(rn, ss[1])
    batch.add(a, ss[0].P)
    batch.add(b, ss[1].P)
    batch.step(8)
    with pytest.raises(rn.RnError):
        b.step(1, ss[1].P)                                  # stepped by the batch
    batch.remove(b)
    b.step(5, ss[1].P)
    ref.step(13, ss[1].P)
    assert identical(b.readAll(), ref.readAll())
    # rescale a member between batch steps: the batch picks up its new ring slot
    a2 = make(rn, ss[0])
    a2.step(8, ss[0].P)
    a.rescaleAmbient(0.9, 1.0, 0.0, ss[0].P)
    a2.rescaleAmbient(0.9, 1.0, 0.0, ss[0].P)
    batch.step(7)
    a2.step(7, ss[0].P)
    assert identical(a.readAll(), a2.readAll())
    batch.close()
    for g in (a, b, ref, a2):
        g.close()


def test_batch_rejects_mismatched_members(rn):
    plain = setups(rn, "plain", [(96, 36)])[0]
    visc = setups(rn, "viscous", [(96, 36)])[0]
    batch = rn.SolverBatch()
    a = make(rn, plain)
    batch.add(a, plain.P)
    v = make(rn, visc)
    with pytest.raises(rn.RnError):
        batch.add(v, visc.P)                                # flags differ
    f = make(rn, plain, precision="fast")
    with pytest.raises(rn.RnError):
        batch.add(f, plain.P)                               # precision differs
    with pytest.raises(rn.RnError):
        batch.add(a, plain.P)                               # already a member
    batch.close()
    for g in (a, v, f):
        g.close()


def test_batch_launches_and_tile(rn, oracle):
    ss = setups(rn, "plain", [(96, 36), (160, 60)])
    batch = rn.SolverBatch()
    gs = [make(rn, s) for s in ss]
    for g, s in zip(gs, ss):
        batch.add(g, s.P)
    batch.setTile("16x15")
    assert all(g.tile == "16x15" for g in gs)
    n0 = batch.kernelLaunches()
    batch.step(20)
    batch.sync()
    assert batch.kernelLaunches() - n0 == 2 * 20             # stage 1 + stage 2 for every member at once
    for g, s in zip(gs, ss):
        assert identical(g.readAll(), run_oracle(oracle, s, 20).readAll())
    batch.close()
    for g in gs:
        g.close()


def test_batch_autotune_restores_members(rn):
    ss = setups(rn, "viscous", [(128, 48), (256, 96), (96, 36)])
    batch = rn.SolverBatch()
    members = [make(rn, s) for s in ss]
    singles = [make(rn, s) for s in ss]
    for g, s in zip(members, ss):
        batch.add(g, s.P)
    batch.step(5)
    for g, s in zip(singles, ss):
        g.step(5, s.P)
    snaps = [(g.readAll(), g.readStepInfo()) for g in members]
    n0 = batch.kernelLaunches()
    chosen = batch.autotune(steps=6)
    assert chosen in ("16x16", "16x8", "16x15", "32x15", "14x16") and batch.tile == chosen
    assert batch.kernelLaunches() == n0
    for g, (st, si) in zip(members, snaps):
        assert identical(g.readAll(), st) and np.array_equal(g.readStepInfo(), si)
    batch.step(7)
    for g, s in zip(singles, ss):
        g.step(7, s.P)
    for g, h in zip(members, singles):
        assert identical(g.readAll(), h.readAll())
    batch.close()
    for g in members + singles:
        g.close()


def test_heavy_tiles_run_in_their_own_launch(rn):
    """With 16x16 tiles a 1024x384 bell has wall tiles listing more out-of-tile
    group members than the common fused launch holds. On a grid of many waves
    those tiles run in a launch of their own, on a side stream beside the main
    one. Results stay bit-identical to the 16x15 tiling (whose lists are all
    short), alone and in a batch."""
    s = setups(rn, "viscous", [(1024, 384)])[0]
    small = setups(rn, "viscous", [(128, 48)])[0]
    outs = []
    for tile in ("16x15", "16x16"):
        g = make(rn, s, tile=tile)
        g.step(12, s.P)
        outs.append(g.readAll())
        g.close()
    assert identical(outs[0], outs[1])
    batch = rn.SolverBatch()
    bigs = [make(rn, s) for _ in range(2)]
    little = make(rn, small)
    for g in bigs:
        batch.add(g, s.P)
    batch.add(little, small.P)
    batch.setTile("16x16")                                    # 2 x 1,536 + 24 blocks: split
    n0 = batch.kernelLaunches()
    batch.step(12)
    batch.sync()
    assert batch.kernelLaunches() - n0 == 3 * 12
    ref = make(rn, small)
    ref.step(12, small.P)
    assert all(identical(g.readAll(), outs[0]) for g in bigs) and identical(little.readAll(), ref.readAll())
    batch.close()
    for g in bigs + [little, ref]:
        g.close()


def test_default_tile_by_grid_size(rn):
    """A new handle takes 14x16 tiles (compiled for 3 blocks per SM) when the
    grid's 14x16 tiles number at most 3 per SM, and 16x15 otherwise."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for Nx, Nr in ((128, 48), (512, 192), (1024, 384), (2048, 768)):
        g = rn.GPUSolver(Nx, Nr)
        tiles = -(-Nx // 14) * -(-Nr // 16)
        assert g.tile == ("14x16" if tiles <= 3 * sms else "16x15"), (Nx, Nr, g.tile)
        g.close()


def loop_to(g, s, t_end, chunk):
    """The plain form of a run to a stop time: `while t < t_end: step(chunk)`."""
    steps = 0
    while float(g.readStepInfo()[2]) < t_end:
        g.step(chunk, s.P)
        steps += chunk
    return steps


@pytest.mark.parametrize("kind,sizes,chunk", [
    ("viscous", [(320, 120), (200, 76), (96, 36)], 7),
    ("plain", [(320, 120), (160, 60), (128, 48)], 12),
    ("spray", [(320, 120), (96, 36), (112, 40)], 5),
])
def test_batch_run_matches_host_loops(rn, kind, sizes, chunk):
    """rn_batch_run stops each member on the device before the chunk at which
    its simulated time reaches its own t_end: every member takes the steps of
    the host loop run alone and ends bit-identical to it. The first member
    stops at once (t_end 0): its 160 blocks (16 x 15 tiles) are more than an
    SM's worth, so they leave the launch at the first chunk; the second stops
    after 3 chunks, and its blocks then return early until the run ends. A
    capped run (max_steps) and plain batch steps afterwards continue from the
    same ring positions."""
    ss = setups(rn, kind, sizes)
    # stop times: 0, and the probe's time after 2 chunks + 3 and 5 chunks
    probe = [make(rn, s) for s in ss]
    t_end = [0.0]
    for g, s, n in zip(probe[1:], ss[1:], (2 * chunk + 3, 5 * chunk)):
        g.step(n, s.P)
        t_end.append(float(g.readStepInfo()[2]))
    for g in probe:
        g.close()
    batch = rn.SolverBatch()
    members = [make(rn, s) for s in ss]
    singles = [make(rn, s) for s in ss]
    for g, s in zip(members, ss):
        batch.add(g, s.P)
    steps = batch.run(t_end, chunk=chunk)
    want = [loop_to(h, s, te, chunk) for h, s, te in zip(singles, ss, t_end)]
    assert steps == want and steps[0] == 0 and steps[1] == 3 * chunk and steps[2] >= 5 * chunk, (steps, want)
    for g, h in zip(members, singles):
        assert g.stepCount == h.stepCount
        assert identical(g.readAll(), h.readAll()) and np.array_equal(g.readStepInfo(), h.readStepInfo())
    # a capped run: every member takes max_steps steps
    steps = batch.run([1e30] * len(ss), chunk=chunk, max_steps=2 * chunk + 1)
    assert steps == [2 * chunk + 1] * len(ss)
    for h, s in zip(singles, ss):
        h.step(2 * chunk + 1, s.P)
    batch.step(9)
    for h, s in zip(singles, ss):
        h.step(9, s.P)
    for g, h in zip(members, singles):
        assert identical(g.readAll(), h.readAll()) and np.array_equal(g.readStepInfo(), h.readStepInfo())
    if kind == "spray":
        for g, h in zip(members, singles):
            assert np.array_equal(g.spray.readParcels()["PA"], h.spray.readParcels()["PA"])
    batch.close()
    for g in members + singles:
        g.close()


def test_batch_run_rejects_bad_arguments_and_empty_batches(rn):
    """A chunk below 1 or a negative step cap is refused before anything is
    queued; an empty batch runs no steps; a t_end list of the wrong length is
    refused by the host wrapper."""
    ss = setups(rn, "plain", [(96, 36)])
    batch = rn.SolverBatch()
    assert batch.run([], chunk=6) == []
    g = make(rn, ss[0])
    batch.add(g, ss[0].P)
    for kw in ({"chunk": 0}, {"chunk": 6, "max_steps": -1}):
        with pytest.raises(rn.RnError):
            batch.run([1.0], **kw)
    with pytest.raises(ValueError):
        batch.run([1.0, 2.0], chunk=6)
    assert g.stepCount == 0
    assert batch.run([0.0], chunk=6) == [0]                  # already at its stop time
    batch.close()
    g.close()
