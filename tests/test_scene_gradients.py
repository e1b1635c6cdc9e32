"""SceneGradients on the GPU: hashed scratch rows filled by the
warp-aggregated atomics the adjoint kernels use (atomic_add_grad =
fpt_scene_gradients_atomic_add, SceneGradients.slang:50-57), then aggregated.

The first test is the reference's own AggregateGradients case
(Tools/FalcorTest/Tests/DiffRendering/SceneGradientsTest.cpp:36-78, the check
the CPU oracle passes in tests/test_oracle_pinning.py): 1024 additions of 10^i
to element i at hash row j % 64, aggregated, equal 1024 * 10^i within 1e-6
relative.  The second adds random contributions, runs of 16 to the same
element as neighbouring lanes of a warp do, and compares with a float64 sum.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scene_gradients(dim, hash_size):
    from falcor_b200.diff import GradConfig, GradientType, SceneGradients
    return SceneGradients.create(None, [GradConfig(GradientType.Material, dim, hash_size)])


def test_aggregate_gradients_reference_case(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.diff import GradientType
    dim, count, hash_size = 3, 1024, 64
    sg = _scene_gradients(dim, hash_size)
    sg.clear_grads(None, GradientType.Material)
    gi, j = np.meshgrid(np.arange(dim), np.arange(count), indexing="ij")
    vals = (10.0 ** gi).astype(np.float32)
    sg.atomic_add_grad(GradientType.Material, torch.from_numpy(gi.ravel()), torch.from_numpy(j.ravel() % hash_size),
                       torch.from_numpy(vals.ravel()))
    sg.aggregate_grads(None, GradientType.Material)
    res = sg.get_grads_buffer(GradientType.Material).cpu().numpy()
    for i in range(dim):
        ref = count * 10.0 ** i
        assert abs(res[i] - ref) / ref <= 1e-6, (i, res[i], ref)


def test_warp_aggregated_atomics_random(fpt):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200.diff import GradientType
    rng = np.random.default_rng(3)
    dim, hash_size, count = 5120, 8, 2_000_000
    sg = _scene_gradients(dim, hash_size)
    sg.clear_grads(None, GradientType.Material)
    # Runs of equal targets mixed with scattered ones, plus out-of-range
    # element indices and hash rows that must be ignored.
    gi = np.repeat(rng.integers(0, dim + 16, count // 16), 16)
    hi = rng.integers(0, hash_size + 1, count)
    vals = rng.standard_normal(count).astype(np.float32)
    sg.atomic_add_grad(GradientType.Material, torch.from_numpy(gi), torch.from_numpy(hi), torch.from_numpy(vals))
    sg.aggregate_grads(None, GradientType.Material)
    res = sg.get_grads_buffer(GradientType.Material).cpu().numpy().astype(np.float64)
    keep = (gi < dim) & (hi < hash_size)
    ref = np.zeros(dim)
    np.add.at(ref, gi[keep], vals[keep].astype(np.float64))
    err = np.abs(res - ref)
    assert err.max() <= 1e-4 * max(1.0, np.abs(ref).max()), err.max()
