"""This package against the reference's OWN CUDA kernels, compiled from the
reference source by oracle/build_ref.py and launched with the reference's
launch shapes, on the same inputs.  Hungarian: bit-identical.  Cost kernels:
both are FP32 evaluations of the same quantity; they must agree within the
sum of their tolerances against FP64 (cost 2e-5 relative, gradient 2e-4)."""
import time

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import ref_kernels as R
from tests.workloads import poses, square_h

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="reference cubins not built (oracle/build_ref.py)")]


def _ours_overlap(x, sep):
    from packing_b200 import pack_cuda
    c = torch.empty(x.shape[0], device=x.device)
    g = torch.empty_like(x)
    pack_cuda.overlap_multi_ensemble(x, x, sep, out_cost=c, out_grads=g)
    return c, g


@pytest.mark.parametrize("sep", [False, True])
@pytest.mark.parametrize("E,n,seed", [(64, 20, 0), (8, 200, 1), (32, 50, 2)])
def test_pair_cost_vs_reference_kernel(cuda, sep, E, n, seed):
    """Costs agree within 2e-5 relative.  Gradients: both FP32 kernels are
    compared with the FP64 oracle; ours must be within the reference test's
    1e-4 and no further from FP64 than the reference kernel is (the
    reference's clip-stage backward pass loses more FP32 accuracy near
    degenerate clips than the single-pass boundary assembly)."""
    x = torch.from_numpy(poses(E, n, seed=seed)).to(cuda)
    rc, rg = R.overlap(x, sep)
    oc, og = _ours_overlap(x, sep)
    torch.cuda.synchronize()
    np.testing.assert_allclose(oc.cpu().numpy(), rc.cpu().numpy(), rtol=2e-5, atol=2e-6)
    fc, fg = O.pair_cost(x.cpu().numpy().astype(np.float64), sep)
    err_ours = np.abs(og.cpu().numpy() - fg).max()
    err_ref = np.abs(rg.cpu().numpy() - fg).max()
    print(f"\nmax |grad - FP64|: ours {err_ours:.3g}, reference kernel {err_ref:.3g}")
    np.testing.assert_allclose(og.cpu().numpy(), fg, rtol=1e-4, atol=1e-4)
    assert err_ours <= err_ref + 1e-5


def test_boundary_vs_reference_kernel(cuda):
    from packing_b200 import pack_cuda
    x = torch.from_numpy(poses(16, 100, seed=3)).to(cuda)
    h = torch.from_numpy(square_h(16, 100) * 0.8).to(cuda)
    h[:, 1] = 0.1
    h[:, 2] = -0.2
    rc, rg, rgh = R.boundary(x, h)
    c = torch.empty(16, device=cuda)
    g = torch.empty_like(x)
    gh = torch.empty_like(h)
    pack_cuda.boundary_distance_multi_ensemble(x, h, out_cost=c, out_grads=g, out_grad_h=gh)
    torch.cuda.synchronize()
    np.testing.assert_allclose(c.cpu().numpy(), rc.cpu().numpy(), rtol=2e-5)
    np.testing.assert_allclose(g.cpu().numpy(), rg.cpu().numpy(), rtol=2e-4, atol=2e-4)
    np.testing.assert_allclose(gh.cpu().numpy(), rgh.cpu().numpy(), rtol=2e-4, atol=2e-3)


@pytest.mark.parametrize("quad", [False, True])
def test_lut_vs_reference_kernel(cuda, quad):
    from packing_b200 import pack_cuda_lut
    from packing_b200.pack_cuda_lut import LookupTable
    lut = LookupTable.build_from_kernel("area", N_x=96, N_y=96, N_theta=72, trim_zeros=False,
                                        apply_quadratic_transform=quad, device=cuda)
    x = torch.from_numpy(poses(24, 80, seed=4)).to(cuda)
    b = (lut.X_min, lut.X_max, lut.Y_min, lut.Y_max, lut.theta_min, lut.theta_max)
    rc, rg = R.lut_overlap(x, lut.lut_d, b, quad)
    c = torch.empty(24, device=cuda)
    g = torch.empty_like(x)
    pack_cuda_lut.overlap_multi_ensemble(x, c, lut, g)
    torch.cuda.synchronize()
    np.testing.assert_allclose(c.cpu().numpy(), rc.cpu().numpy(), rtol=1e-5, atol=1e-6)
    # Gradients: the two FP32 kernels sum a tree's pair terms in different
    # orders (the reference with float atomics, here exactly in fixed point),
    # so they are each held to the FP64 evaluation of the same table at the
    # reference's own gradient tolerance (pack_test.py:286-297), and ours
    # must be no further from it than the reference kernel is.
    _, og = O.lut_cost(list(x.cpu().numpy().astype(np.float64)), lut.lut_d.cpu().numpy(), b, quad,
                       O.geometry()[3])
    og = np.stack(og)
    err_ours = np.abs(g.cpu().numpy() - og).max()
    err_ref = np.abs(rg.cpu().numpy() - og).max()
    print(f"\nLUT max |grad - FP64|: ours {err_ours:.3g}, reference kernel {err_ref:.3g}")
    np.testing.assert_allclose(g.cpu().numpy(), og, rtol=1e-4, atol=1e-4)
    assert err_ours <= err_ref + 1e-6


@pytest.mark.parametrize("N", [3, 33, 100, 200])
def test_hungarian_bit_identical_to_reference_kernel(cuda, N):
    from packing_b200.lap_batch import solve_lap_batch
    rng = np.random.default_rng(N)
    for C in (rng.random((64, N, N)), rng.integers(0, 5, size=(64, N, N))):
        Ct = torch.from_numpy(C.astype(np.float32)).to(cuda)
        rrm, rtot = R.hungarian(Ct)
        rm, tot = solve_lap_batch(Ct)
        torch.cuda.synchronize()
        assert torch.equal(rm, rrm)
        assert torch.equal(tot, rtot)


def _time(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_timing_against_reference_kernels(cuda):
    """Same inputs, same GPU: reference kernels vs this package (printed)."""
    from packing_b200 import pack_cuda
    from packing_b200.lap_batch import solve_lap_batch
    x = torch.from_numpy(poses(4096, 200, seed=0)).to(cuda)
    c = torch.empty(4096, device=cuda)
    g = torch.empty_like(x)
    lines = []
    for sep in (False, True):
        tr = _time(lambda: R.overlap(x, sep))
        to = _time(lambda: pack_cuda.overlap_multi_ensemble(x, x, sep, out_cost=c, out_grads=g))
        lines.append(f"overlap {'sep ' if sep else 'area'} 4096 x n=200: reference {tr:.3f} ms, ours {to:.3f} ms, "
                     f"x{tr / to:.2f}")
    from packing_b200 import pack_cuda_lut
    from packing_b200.pack_cuda_lut import LookupTable
    r0 = 0.5796198
    X = np.linspace(-2 * r0, 2 * r0, 510, dtype=np.float32)[254:]
    Y = np.linspace(-2 * r0, 2 * r0, 256, dtype=np.float32)
    T = np.linspace(-np.pi, np.pi, 360, dtype=np.float32)
    lut = LookupTable.build_from_kernel("area", X=X, Y=Y, theta=T, trim_zeros=False, device=cuda)
    b = (lut.X_min, lut.X_max, lut.Y_min, lut.Y_max, lut.theta_min, lut.theta_max)
    tr = _time(lambda: R.lut_overlap(x, lut.lut_d, b, False))
    to = _time(lambda: pack_cuda_lut.overlap_multi_ensemble(x, c, lut, g))
    lines.append(f"LUT 256 x 256 x 360, 4096 x n=200: reference {tr:.3f} ms, ours {to:.3f} ms, x{tr / to:.2f}")
    C = torch.rand((2048, 100, 100), device=cuda)
    tr = _time(lambda: R.hungarian(C), reps=3)
    to = _time(lambda: solve_lap_batch(C), reps=3)
    lines.append(f"hungarian 2048 x 100^2: reference {tr:.3f} ms, ours {to:.3f} ms, x{tr / to:.2f}")
    print("\n" + "\n".join(lines))
