"""The GA move kernel (pk_moves) against the oracle restatement of
core/pack_move.py: same Philox draws, same moves, same trees."""
import dataclasses

import numpy as np
import pytest
import torch

from oracle import moves as MV

pytestmark = pytest.mark.gpu
F = np.float32


def _pop(E, n, side, seed, kind="square", offset=(0.0, 0.0)):
    rng = np.random.default_rng(seed)
    xyt = np.zeros((E, n, 3), F)
    lo = -side / 2
    hi_x = 0.0 if kind in ("sym90", "sym180") else side / 2
    hi_y = 0.0 if kind == "sym90" else side / 2
    xyt[:, :, 0] = rng.uniform(lo, hi_x, (E, n)) + offset[0]
    xyt[:, :, 1] = rng.uniform(lo, hi_y, (E, n)) + offset[1]
    xyt[:, :, 2] = rng.uniform(-np.pi, np.pi, (E, n))
    h = np.tile(np.array([side, offset[0], offset[1]], F), (E, 1))
    h[:, 0] += rng.uniform(-0.2, 0.2, E).astype(F)
    return xyt, h


def _oracle_geno(g):
    from packing_b200.pack_move import EdgeSpacerBasic
    sp = g.edge_spacer
    return {"kind": g.kind, "filter": g.filter_move_locations_with_edge_spacer,
            "margin": g.filter_move_locations_margin,
            "spacer": dataclasses.asdict(sp) if isinstance(sp, EdgeSpacerBasic) else None}


def _run(cuda, entries, kind="square", mate_kind=None, E=40, n=36, side=6.0, spacer=None, filt=False, seed=11,
         call=0, offset=(0.0, 0.0), rows=None, exact=True, min_equal=0.99):
    from packing_b200 import pack_move as PM
    xyt, h = _pop(E, n, side, seed, kind, offset)
    mkind = mate_kind or kind
    mxyt, mh = _pop(E, n, side * 1.05, seed + 1, mkind, offset)
    pop = PM.Genotype(torch.from_numpy(xyt.copy()).to(cuda), torch.from_numpy(h).to(cuda), kind=kind,
                      edge_spacer=spacer or PM.EdgeSpacerDummy(), filter_move_locations_with_edge_spacer=filt)
    mate = PM.Genotype(torch.from_numpy(mxyt).to(cuda), torch.from_numpy(mh).to(cuda), kind=mkind)
    rows = np.arange(0, E, 2) if rows is None else np.asarray(rows)
    inds_mate = (rows * 7 + 3) % E
    sel = PM.MoveSelector(moves=[[m, type(m).__name__, w] for m, w in entries])
    gen = PM.MoveGenerator(seed=0x1234_5678_9ABC + seed)
    gen.call = call
    chosen = sel.do_move_vec(pop, torch.from_numpy(rows).to(cuda), mate, torch.from_numpy(inds_mate).to(cuda), gen)
    got = pop.xyt.cpu().numpy()
    ora_entries = [(type(m).__name__, dataclasses.asdict(m), w) for m, w in entries]
    want, want_chosen = MV.apply(ora_entries, _oracle_geno(pop), xyt, h, list(rows), mxyt, mh, list(inds_mate),
                                 gen.seed, call, mate_kind=mkind)
    np.testing.assert_array_equal(chosen.cpu().numpy(), want_chosen)
    untouched = np.setdiff1d(np.arange(E), rows)
    np.testing.assert_array_equal(got[untouched], xyt[untouched])
    if exact:
        np.testing.assert_array_equal(got, want)
    else:   # cos / sin of the GPU and the host may differ in the last bit
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-6)
        assert (got == want).mean() > min_equal
    assert (got[rows] != xyt[rows]).any()
    return got, want


def test_draws_match_oracle(cuda):
    from packing_b200.pack_move import move_draws
    for seed, call, row in [(0, 0, 0), (2 ** 40 + 5, 3, 17), (123456789, 2 ** 33 + 1, 4095)]:
        got = move_draws(seed, call, row, 5, 64, cuda).cpu().numpy()
        s = MV.Stream(seed, call, row)
        np.testing.assert_array_equal(got, np.array([s.draw(5 + k) for k in range(64)]))


def test_random_tree_and_jiggles(cuda):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.MoveRandomTree(), 1.0)])
    _run(cuda, [(PM.JiggleRandomTree(max_xy_move=0.05, max_theta_move=np.pi / 6), 1.0)], offset=(0.4, -0.3))
    _run(cuda, [(PM.JiggleCluster(max_xy_move=0.1, max_theta_move=np.pi), 1.0)])
    _run(cuda, [(PM.JiggleCluster(min_N_trees=3, max_N_trees=40), 1.0)], n=12)


def test_translate(cuda):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.Translate(), 1.0)], offset=(0.25, 0.5))


def test_twist(cuda):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.Twist(), 1.0)], exact=False)


@pytest.mark.parametrize("simple", [True, False])
def test_crossover(cuda, simple):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.Crossover(simple_mate_location=simple), 1.0)], exact=False)


@pytest.mark.parametrize("kw", [{}, {"distance_function": "square"},
                                {"distance_function": "square", "decouple_mate_location": True},
                                {"decouple_mate_location": True, "use_edge_clearance_when_decoupled": False},
                                {"do_90_rotation": False, "max_N_trees_ratio": 0.45}])
def test_crossover2_square_population(cuda, kw):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.Crossover2(**kw), 1.0)], exact=False)


def test_crossover2_symmetric(cuda):
    from packing_b200 import pack_move as PM
    _run(cuda, [(PM.Crossover2(distance_function="square90"), 1.0),
                (PM.Crossover2(distance_function="square90", decouple_mate_location=True), 1.0)],
         kind="sym90", n=20, side=8.0, exact=False)
    _run(cuda, [(PM.Crossover2(distance_function="square180", max_N_trees_ratio=0.45), 1.0),
                (PM.Crossover2(distance_function="square180", decouple_mate_location=True, max_N_trees_ratio=0.45),
                 1.0)], kind="sym180", n=24, side=7.0, exact=False)


def test_symmetric_move_centres(cuda):
    from packing_b200 import pack_move as PM
    for kind in ("sym90", "sym180"):
        _run(cuda, [(PM.MoveRandomTree(), 1.0), (PM.JiggleCluster(), 1.0)], kind=kind, n=20, side=7.0)


def test_edge_spacer_filter(cuda):
    """The tesselated configuration (pack_ga3.py:1770-1830): EdgeSpacerBasic,
    filtered move locations, Crossover2 without 90-degree turns."""
    from packing_b200 import pack_move as PM
    sp = PM.EdgeSpacerBasic(dist_x=0.75, dist_y=0.5, dist_corner=0.0)
    moves = [(PM.MoveRandomTree(), 1.0), (PM.JiggleRandomTree(), 1.0), (PM.JiggleCluster(), 1.0),
             (PM.Twist(), 1.0),
             (PM.Crossover2(do_90_rotation=False, use_edge_clearance_when_decoupled=False), 2.0),
             (PM.Crossover2(distance_function="square", decouple_mate_location=True, do_90_rotation=False,
                            use_edge_clearance_when_decoupled=False, max_N_trees_ratio=0.45), 2.0),
             (PM.JiggleRandomTree(respect_edge_spacer_filter=False), 1.0)]
    _run(cuda, moves, spacer=sp, filt=True, E=96, exact=False)
    # corner clearance: the analytic samplers give way to rejection sampling
    sp2 = PM.EdgeSpacerBasic(dist_x=0.75, dist_y=0.5, dist_corner=0.6)
    _run(cuda, moves[:3], spacer=sp2, filt=True, E=64)
    _run(cuda, [(PM.MoveRandomTree(), 1.0), (PM.JiggleRandomTree(), 1.0)], kind="sym180", spacer=sp, filt=True,
         n=24, side=7.0)


def test_reference_ga_move_set(cuda):
    """The GA's default MoveSelector (pack_ga3.py:1084-1115) on 512 rows."""
    from packing_b200 import pack_move as PM
    moves = [(PM.MoveRandomTree(), 1.0),
             (PM.JiggleRandomTree(max_xy_move=0.05, max_theta_move=np.pi / 6), 1.0),
             (PM.JiggleRandomTree(max_xy_move=0.1, max_theta_move=np.pi), 1.0),
             (PM.JiggleCluster(max_xy_move=0.05, max_theta_move=np.pi / 6), 1.0),
             (PM.JiggleCluster(max_xy_move=0.1, max_theta_move=np.pi), 1.0),
             (PM.Translate(), 1.0), (PM.Twist(), 1.0), (PM.Crossover(), 2.0), (PM.Crossover2(), 2.0)]
    got, _ = _run(cuda, moves, E=1024, n=50, side=7.5, rows=np.arange(0, 1024, 2), call=7, exact=False)
    assert np.isfinite(got).all()


def test_calls_draw_fresh_numbers_and_replay(cuda):
    from packing_b200 import pack_move as PM
    xyt, h = _pop(8, 20, 5.0, 0)
    outs = []
    for call in (0, 1, 0):
        pop = PM.Genotype(torch.from_numpy(xyt.copy()).to(cuda), torch.from_numpy(h).to(cuda))
        gen = PM.MoveGenerator(seed=99)
        gen.call = call
        PM.JiggleRandomTree().do_move_vec(pop, torch.arange(8, device=cuda), None, None, gen)
        outs.append(pop.xyt.cpu().numpy())
    assert not np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])


def test_argument_errors(cuda):
    from packing_b200 import pack_move as PM
    xyt, h = _pop(4, 10, 5.0, 0)
    pop = PM.Genotype(torch.from_numpy(xyt).to(cuda), torch.from_numpy(h).to(cuda))
    with pytest.raises(ValueError):
        PM.Crossover().do_move_vec(pop, torch.arange(4, device=cuda), None, None, PM.MoveGenerator())
    with pytest.raises(ValueError):
        PM.Crossover2(distance_function="circle").do_move_vec(pop, torch.arange(4, device=cuda), pop,
                                                              torch.arange(4, device=cuda), PM.MoveGenerator())
    sym = PM.Genotype(pop.xyt, pop.h, kind="sym90", filter_move_locations_with_edge_spacer=True,
                      edge_spacer=PM.EdgeSpacerBasic())
    with pytest.raises(ValueError):   # the reference asserts: no edge-spacer filter on 90-degree genotypes
        PM.MoveRandomTree().do_move_vec(sym, torch.arange(4, device=cuda), None, None, PM.MoveGenerator())


def test_out_of_range_rows_are_reported(cuda):
    """Row and mate indices are checked in the kernel: a bad one is reported
    and its row left alone; the other rows still move."""
    from packing_b200 import pack_move as PM
    xyt, h = _pop(4, 10, 5.0, 0)
    pop = PM.Genotype(torch.from_numpy(xyt.copy()).to(cuda), torch.from_numpy(h).to(cuda))
    with pytest.raises(IndexError):
        PM.JiggleRandomTree().do_move_vec(pop, torch.tensor([0, 7], device=cuda), None, None, PM.MoveGenerator())
    got = pop.xyt.cpu().numpy()
    assert (got[0] != xyt[0]).any()
    np.testing.assert_array_equal(got[1:], xyt[1:])
    mate = PM.Genotype(torch.from_numpy(xyt.copy()).to(cuda), torch.from_numpy(h).to(cuda))
    with pytest.raises(IndexError):
        PM.Crossover().do_move_vec(pop, torch.tensor([1], device=cuda), mate, torch.tensor([-1], device=cuda),
                                   PM.MoveGenerator())


def test_generation_step(cuda):
    """Clone, the GA's default moves, and the rough relaxation on the GA's
    fitness cost (exact-separation LUT) in one call."""
    from packing_b200 import pack_move as PM
    from packing_b200.ga_step import default_moves, fitness_spec, generation_step
    from packing_b200.pack_cuda_lut import LookupTable
    P, n = 32, 24
    rng = np.random.default_rng(2)
    side = float(np.sqrt(n * 0.2456875) * 1.6)
    xyt = np.zeros((P, n, 3), F)
    xyt[:, :, :2] = rng.uniform(-side / 2, side / 2, (P, n, 2))
    xyt[:, :, 2] = rng.uniform(-np.pi, np.pi, (P, n))
    h = np.tile(np.array([side, 0, 0], F), (P, 1))
    pop, hh = torch.from_numpy(xyt).to(cuda), torch.from_numpy(h).to(cuda)
    parents = torch.arange(P, device=cuda).flip(0)
    mates = (parents + 1) % P
    spec = fitness_spec(LookupTable.build_exact_separation(N_x=200, N_y=200, N_theta=180, device=cuda))
    out, hout, loss, chosen = generation_step(pop, hh, parents, mates, PM.MoveGenerator(3), spec, default_moves())
    assert out.shape == (P, n, 3) and torch.isfinite(out).all() and torch.isfinite(loss).all()
    assert ((chosen >= 0) & (chosen < 9)).all()
    np.testing.assert_array_equal(pop.cpu().numpy(), xyt)      # the old population is untouched


@pytest.mark.parametrize("n", [1, 2, 3])
def test_tiny_packings(cuda, n):
    """Every move on packings of 1 to 3 trees (cluster and crossover sizes
    clamp to n) matches the oracle."""
    from packing_b200 import pack_move as PM
    moves = [(PM.MoveRandomTree(), 1.0), (PM.JiggleRandomTree(), 1.0), (PM.JiggleCluster(), 1.0),
             (PM.Translate(), 1.0), (PM.Twist(), 1.0), (PM.Crossover(), 1.0), (PM.Crossover2(), 1.0),
             (PM.Crossover2(distance_function="square", decouple_mate_location=True), 1.0)]
    _run(cuda, moves, E=64, n=n, side=2.0, exact=False, min_equal=0.9)
