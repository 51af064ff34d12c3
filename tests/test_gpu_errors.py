"""Error returns of the C ABI on a GPU (the reference prints and continues or
asserts; here every refusal is an ``a2a_status``, checked on the host before
anything is launched): transform lengths with no compiled kernel, transforms
before ``make_plans``, NULL and misaligned data pointers.  No case hands a
kernel an invalid buffer."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("P,shape", [(8, 40), (4, 20), (8, (64, 40, 64)), (4, (32, 32, 80))])
def test_length_without_a_kernel_is_unsupported(pkg, cuda, P, shape):
    """Decomposable grids whose transform length (40, 20, 80: a factor 5)
    has no compiled plan."""
    with pytest.raises(pkg.A2AError, match="UNSUPPORTED") as e:
        pkg.a2aDistribution(P, shape, 64, precision="c64")
    assert "no compiled transform of length" in str(e.value)


def test_grid_above_32_bit_indices_is_unsupported(pkg, cuda):
    with pytest.raises(pkg.A2AError, match="UNSUPPORTED"):
        pkg.a2aDistribution(8, 2048, 64, precision="c64")


def test_transform_before_make_plans(pkg, cuda):
    dist = pkg.a2aDistribution(4, 32, 64, precision="c64")
    f = pkg.a2adfft(dist)
    x = dist.empty()
    with pytest.raises(pkg.A2AError, match="NO_PLANS"):
        f.forward(x)
    f.make_plans()
    f.forward(x)  # then it runs


def test_null_and_misaligned_data(pkg, oracle, cuda):
    import torch

    P, ng = 4, 32
    dist = pkg.a2aDistribution(P, ng, 64, precision="c64")
    f = pkg.a2adfft(dist)
    f.make_plans()
    x = dist.empty()
    with pytest.raises(pkg.A2AError, match="INVALID_VALUE"):
        f.forward(0)
    with pytest.raises(pkg.A2AError, match="MISALIGNED"):
        f.forward(x.data_ptr() + 8)  # refused before any launch
    # the plan is unharmed: a correct transform follows
    d = oracle.Decomp(ng, P)
    g = oracle.make_input("uniform", (ng,) * 3, seed=9, dtype=np.complex64)
    x.copy_(torch.from_numpy(oracle.global_to_bricks(g, d).ravel()))
    f.forward(x)
    fwd = oracle.bricks_to_global(x.cpu().numpy().reshape(P, -1), d)
    assert oracle.rel_l2(fwd, oracle.fft3_global(g)) <= 1e-6
    f.check_device()
