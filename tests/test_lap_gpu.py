"""Batched Hungarian: bit-exact against the float32 restatement of the
reference kernel (lap_batch.py:62-196), optimal against scipy."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.workloads import poses

pytestmark = pytest.mark.gpu


def _solve(C, dev):
    from packing_b200.lap_batch import solve_lap_batch
    rm, tot = solve_lap_batch(torch.from_numpy(C).to(dev))
    return rm.cpu().numpy(), tot.cpu().numpy()


@pytest.mark.parametrize("N", [1, 2, 5, 31, 32, 33, 64, 100, 129, 200, 256])
def test_random_bitexact(cuda, N):
    rng = np.random.default_rng(N)
    C = rng.random((24, N, N)).astype(np.float32)
    rm, tot = _solve(C, cuda)
    orm, otot = O.hungarian(C)
    assert np.array_equal(rm, orm)
    assert np.array_equal(tot.view(np.int32), otot.view(np.int32))


def test_staged_and_l2_forms_bitexact(cuda):
    """The solver stages each matrix in shared memory when every problem of
    the batch can be resident at once (600 of 100 x 100 on a B200), and
    reads it from L2 otherwise (1000): both give the oracle's answer.  An odd
    side and a base one float past a 16-byte boundary take the scalar copy."""
    rng = np.random.default_rng(5)
    for B, N in ((600, 100), (1000, 100), (9, 37)):
        C = rng.random((B, N, N)).astype(np.float32)
        rm, tot = _solve(C, cuda)
        orm, otot = O.hungarian(C)
        assert np.array_equal(rm, orm)
        assert np.array_equal(tot.view(np.int32), otot.view(np.int32))
    from packing_b200.lap_batch import solve_lap_batch
    flat = rng.random(1 + 7 * 36 * 36).astype(np.float32)
    view = torch.from_numpy(flat).to(cuda)[1:].view(7, 36, 36)
    assert view.data_ptr() % 16 != 0
    rm, tot = solve_lap_batch(view)
    orm, otot = O.hungarian(flat[1:].reshape(7, 36, 36))
    assert np.array_equal(rm.cpu().numpy(), orm)
    assert np.array_equal(tot.cpu().numpy(), otot)


def test_ties_bitexact(cuda):
    """Integer costs with many equal slacks: ties must go to the lowest column."""
    rng = np.random.default_rng(1)
    for N in (8, 50, 100):
        C = rng.integers(0, 4, size=(32, N, N)).astype(np.float32)
        rm, tot = _solve(C, cuda)
        orm, otot = O.hungarian(C)
        assert np.array_equal(rm, orm)
        assert np.array_equal(tot, otot)
    C = np.zeros((3, 17, 17), np.float32)
    rm, tot = _solve(C, cuda)
    orm, _ = O.hungarian(C)
    assert np.array_equal(rm, orm)


def test_config3_diversity_matrices_bitexact(cuda):
    """2048 problems of 100x100: squared centre distance + |wrapped angle
    difference| between seeded packings."""
    a = poses(2048, 100, seed=3).astype(np.float64)
    b = poses(2048, 100, seed=4).astype(np.float64)
    d2 = ((a[:, :, None, :2] - b[:, None, :, :2]) ** 2).sum(-1)
    dt = np.abs(np.remainder(a[:, :, None, 2] - b[:, None, :, 2] + np.pi, 2 * np.pi) - np.pi)
    C = (d2 + dt).astype(np.float32)
    rm, tot = _solve(C, cuda)
    orm, otot = O.hungarian(C)
    assert np.array_equal(rm, orm)
    assert np.array_equal(tot, otot)


def test_optimal_vs_scipy(cuda):
    from scipy.optimize import linear_sum_assignment
    rng = np.random.default_rng(9)
    C = rng.random((16, 120, 120)).astype(np.float32)
    rm, tot = _solve(C, cuda)
    for b in range(16):
        r, c = linear_sum_assignment(C[b].astype(np.float64))
        assert C[b][np.arange(120), rm[b]].astype(np.float64).sum() == pytest.approx(
            C[b][r, c].astype(np.float64).sum(), abs=1e-4)


def test_heuristics_and_limits(cuda):
    from packing_b200.lap_batch import LAPConfig, solve_lap_batch
    rng = np.random.default_rng(2)
    C = torch.from_numpy(rng.random((5, 9, 9)).astype(np.float32)).to(cuda)
    rm, tot = solve_lap_batch(C, LAPConfig("min_cost_row"))
    assert torch.all(rm == -1)
    assert torch.allclose(tot, C.amin(2).sum(1))
    rm, tot = solve_lap_batch(C, LAPConfig("min_cost_col"))
    assert torch.allclose(tot, C.amin(1).sum(1))
    with pytest.raises(AssertionError):
        solve_lap_batch(torch.zeros((1, 257, 257), device=cuda))
    rm, tot = solve_lap_batch(torch.zeros((0, 4, 4), device=cuda))
    assert rm.shape == (0, 4) and tot.shape == (0,)
    # a row of +inf everywhere has no finite slack: reported, not a hang
    C = torch.ones((2, 4, 4), device=cuda)
    C[1, 2, :] = float("inf")
    rm, tot, st = solve_lap_batch(C, return_status=True)
    assert st.tolist() == [0, 1]
    assert torch.all(rm[1] == -1) and torch.isnan(tot[1])


def test_genetic_diversity_matrix(cuda):
    """Fused transform + assignment + min over the 8 symmetries equals the
    materialised matrices solved one by one, and the oracle on them."""
    from packing_b200.lap_batch import genetic_diversity_cost_matrices, genetic_diversity_matrix, solve_lap_batch
    pop = torch.from_numpy(poses(4, 30, seed=11)).to(cuda)
    ref = torch.from_numpy(poses(3, 30, seed=12)).to(cuda)
    D = genetic_diversity_matrix(pop, ref).cpu().numpy()
    M = genetic_diversity_cost_matrices(pop, ref)
    _, tot = solve_lap_batch(M)
    T = tot.reshape(8, 4, 3).amin(0).cpu().numpy()
    assert np.array_equal(D, T)
    _, otot = O.hungarian(M.cpu().numpy())
    assert np.array_equal(T, otot.reshape(8, 4, 3).min(0))
    # against a float64 numpy restatement of kaggle_support.py:2061-2112
    P, R = pop.cpu().numpy().astype(np.float64), ref.cpu().numpy().astype(np.float64)
    for t, (ang, mir) in enumerate([(0, 0), (np.pi / 2, 0), (np.pi, 0), (3 * np.pi / 2, 0),
                                    (0, 1), (np.pi / 2, 1), (np.pi, 1), (3 * np.pi / 2, 1)]):
        rx, ry, rt = R[..., 0], R[..., 1], R[..., 2]
        if mir:
            ry, rt = -ry, np.pi - rt
        if ang:
            rx, ry, rt = rx * np.cos(ang) - ry * np.sin(ang), rx * np.sin(ang) + ry * np.cos(ang), rt + ang
        rt = np.remainder(rt + np.pi, 2 * np.pi) - np.pi
        dx = P[:, :, None, None, 0] - rx[None, None]
        dy = P[:, :, None, None, 1] - ry[None, None]
        dth = np.remainder(P[:, :, None, None, 2] - rt[None, None] + np.pi, 2 * np.pi) - np.pi
        C64 = np.sqrt(dx ** 2 + dy ** 2 + dth ** 2).transpose(0, 2, 1, 3).reshape(-1, 30, 30)
        np.testing.assert_allclose(M[t * 12:(t + 1) * 12].cpu().numpy(), C64, rtol=1e-5, atol=1e-5)


def _diversity_costs_f32(P, R):
    """The diversity cost matrices (kaggle_support.py:2061-2112, torch float32:
    remainder = fmod, plus the divisor when the sign differs) restated in
    float32 numpy with the kernel's rounding order, stacked (transform, pop,
    ref) -> (n, n)."""
    f = np.float32
    PI = f(np.pi)
    T = f(2) * PI
    ca, sa = [f(1), f(0), f(-1), f(0)], [f(0), f(1), f(0), f(-1)]
    ang = [f(0), f(1.5707963267948966), f(3.141592653589793), f(4.71238898038469)]

    def rem(x):
        m = np.fmod(x, T)
        return np.where(m < 0, m + T, m)

    out = []
    for t in range(8):
        x, y, th = R[..., 0], R[..., 1], R[..., 2]
        if t >= 4:
            y, th = -y, PI - th
        r = t & 3
        if r:
            x, y = x * ca[r] - y * sa[r], x * sa[r] + y * ca[r]
            th = th + ang[r]
        th = rem(th + PI) - PI
        dx = P[:, None, :, None, 0] - x[None, :, None, :]
        dy = P[:, None, :, None, 1] - y[None, :, None, :]
        dt = rem((P[:, None, :, None, 2] - th[None, :, None, :]) + PI) - PI
        out.append(np.sqrt((dx * dx + dy * dy) + dt * dt).astype(f))
    return np.stack(out).reshape(-1, P.shape[1], P.shape[1])


def test_diversity_costs_bitexact_wide_angles(cuda):
    """Cost matrices equal the float32 restatement bit for bit for angles far
    outside [0, 2 pi) as well, so every branch of the kernel's remainder
    (|x| < 2 pi, 2 pi <= |x| < 4 pi, beyond) meets the general fmod."""
    from packing_b200.lap_batch import genetic_diversity_cost_matrices, genetic_diversity_matrix, solve_lap_batch
    rng = np.random.default_rng(17)
    P = poses(3, 40, seed=21)
    R = poses(2, 40, seed=22)
    P[..., 2] = rng.uniform(-25.0, 25.0, P.shape[:2])
    R[..., 2] = rng.uniform(-25.0, 25.0, R.shape[:2])
    P[0, :4, 2] = [0.0, -0.0, np.float32(2 * np.pi), -np.float32(4 * np.pi)]
    M = genetic_diversity_cost_matrices(torch.from_numpy(P).to(cuda), torch.from_numpy(R).to(cuda)).cpu().numpy()
    ref = _diversity_costs_f32(P.astype(np.float32), R.astype(np.float32))
    assert np.array_equal(M.view(np.int32), ref.view(np.int32))
    D = genetic_diversity_matrix(torch.from_numpy(P).to(cuda), torch.from_numpy(R).to(cuda)).cpu().numpy()
    _, tot = solve_lap_batch(torch.from_numpy(ref).to(cuda))
    assert np.array_equal(D, tot.reshape(8, 3, 2).amin(0).cpu().numpy())


def test_diversity_shortcut(cuda):
    from packing_b200.lap_batch import compute_diversity_shortcut_kernel
    pop = poses(5, 40, seed=13)
    ref = poses(4, 40, seed=14)
    for ca, sa, mir in [(1.0, 0.0, False), (0.0, 1.0, True), (np.cos(2.0), np.sin(2.0), False)]:
        D = compute_diversity_shortcut_kernel(torch.from_numpy(pop).to(cuda), torch.from_numpy(ref).to(cuda),
                                              ca, sa, mir).cpu().numpy()
        OD = O.diversity_shortcut(pop, ref, ca, sa, mir)
        np.testing.assert_allclose(D, OD, rtol=1e-5, atol=1e-5)


def test_matched_crossover_generation(cuda):
    """The matched-crossover generation: each parent's trees are assigned to
    its partner's by the batched Hungarian (a permutation, equal to the
    float32 restatement's), then crossover, jitter and relaxation give
    finite children."""
    from packing_b200.ga_step import crossover_jitter_step, matching_costs
    P, n = 16, 20
    x = torch.from_numpy(poses(P, n, seed=9)).to(cuda)
    h = torch.zeros((P, 3), device=cuda)
    h[:, 0] = float(np.sqrt(n * 0.2456875) * 1.3)
    partners = torch.roll(torch.arange(P, device=cuda), 1)
    g = torch.Generator(device=cuda)
    g.manual_seed(1)
    out, loss, rm = crossover_jitter_step(x, partners, h, g, iterations=20)
    rm = rm.cpu().numpy()
    assert all(np.array_equal(np.sort(r), np.arange(n)) for r in rm)
    orm, _ = O.hungarian(matching_costs(x, x[partners]).cpu().numpy())
    assert np.array_equal(rm, orm)
    assert torch.isfinite(out).all() and torch.isfinite(loss).all()
