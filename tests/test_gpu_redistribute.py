"""GPU tests of the redistribution transposes (rgf_permute_c16): each of the
four RESHAPE(..., ORDER=) transposes of energies_to_ijs_2 /
ijs_to_energies_2 (green_rgf.f90:243-329) bit-exact against the oracle, and
the one-rank round trip through liteqt_b200.redistribute on the GPU."""
import numpy as np
import pytest

from oracle.redistribute import fortran_reshape_order

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rgf():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from liteqt_b200 import build, rgf as R
    build.build()
    R.load()
    return R


@pytest.mark.parametrize("shape,order", [((64, 4, 10, 8, 4), (1, 5, 2, 3, 4)), ((64, 10, 8, 4, 4), (5, 4, 1, 3, 2)),
                                         ((8, 4, 4, 10, 64), (3, 5, 4, 2, 1)), ((64, 10, 8, 4, 4), (1, 3, 4, 5, 2)),
                                         ((3, 5, 7), (2, 3, 1)), ((37, 5, 70), (3, 1, 2)), ((300, 3), (1, 2)),
                                         ((33, 65, 2), (2, 1, 3)), ((7,), (1,))])
def test_permute_matches_oracle(rgf, shape, order):
    import torch
    rng = np.random.default_rng(1)
    n = int(np.prod(shape))
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    src = torch.from_numpy(x).cuda()
    dst = torch.empty_like(src)
    with rgf.Context(rgf.Options()) as ctx:
        ctx.permute(src, dst, shape, order)
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy(), fortran_reshape_order(x, shape, order))


def test_one_rank_round_trip(rgf):
    import torch
    from liteqt_b200 import redistribute as RD
    nij, nx, ne, nk = 64, 6, 12, 2
    rng = np.random.default_rng(2)
    x = rng.normal(size=nij * nx * ne * nk) + 1j * rng.normal(size=nij * nx * ne * nk)
    buf = torch.from_numpy(x).cuda()
    tmp0, tmp1 = torch.empty_like(buf), torch.empty_like(buf)
    with rgf.Context(rgf.Options()) as ctx:
        RD.energies_to_ijs_2(buf, tmp0, tmp1, nx, nk, nij, ne, 1, ctx=ctx)
        torch.cuda.synchronize()
        want = np.transpose(x.reshape((nij, nx, ne, nk), order="F"), (2, 3, 1, 0)).reshape(-1, order="F")
        assert np.array_equal(buf.cpu().numpy(), want)
        RD.ijs_to_energies_2(buf, tmp0, tmp1, nx, nk, nij, ne, 1, ctx=ctx)
        torch.cuda.synchronize()
    assert np.array_equal(buf.cpu().numpy(), x)
