"""GPU tests of the texture-fetch loader, sgemm_b200_texld -- the B200 form of
the reference's pre-Ampere path (src/sgemm.cuh:49-89,
src/kernels/128x128x8_texld.cuh): A and B read as float4 texels through
linear texture objects when aligned, the plain kernels otherwise.  Either way
the result must equal the oracle's restatement of the reference's arithmetic
bit for bit."""
import numpy as np
import pytest

import oracle
import sgemm_b200 as sg

pytestmark = pytest.mark.gpu


def _dev(x, ld=None, offset=0):
    """CUDA view of x with row stride ld, starting `offset` floats into its
    allocation (a base that is 16-byte but not texture-aligned)."""
    import torch
    r, c = x.shape
    ld = ld or c
    big = torch.full((r * ld + offset + 8,), float("nan"), device="cuda")
    v = big[offset:offset + r * ld].view(r, ld)
    v[:, :c] = torch.from_numpy(x).cuda()
    return v[:, :c]


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (64, 64, 64), (300, 520, 1001), (129, 257, 33),
                                   (1000, 1000, 1000), (77, 1031, 263), (2048, 512, 30)])
@pytest.mark.parametrize("ab", [(1.5, 0.5), (1.0, 0.0)], ids=["a1.5b0.5", "a1b0"])
def test_texld_bit_exact(m, n, k, ab):
    import torch
    alpha, beta = ab
    A = oracle.fill(m, k, 31, 1, 0)
    B = oracle.fill(k, n, 31, 2, 0)
    C = oracle.fill(m, n, 31, 3, 0)
    # padded strides (multiples of 4: the texture path) and bases 16 bytes
    # past a texture-aligned address
    lda, ldb = (k + 3) // 4 * 4 + 4, (n + 3) // 4 * 4
    dA, dB = _dev(A, lda, offset=4), _dev(B, ldb, offset=8)
    dC = _dev(C)
    if beta == 0.0:
        dC.fill_(float("nan"))  # never read
    sg.sgemm_texld(dA, dB, dC, alpha, beta)
    torch.cuda.synchronize()
    assert sg.device_status() == sg.OK
    assert np.array_equal(dC.cpu().numpy(), oracle.sgemm_basic(A, B, C, alpha, beta, basic=False))


def test_texld_unaligned_operands_fall_back():
    # lda not a multiple of 4: the reference's condition fails, the plain
    # kernels run, same bits
    import torch
    m, n, k = 200, 136, 101
    A = oracle.fill(m, k, 32, 1, 0)
    B = oracle.fill(k, n, 32, 2, 0)
    C = oracle.fill(m, n, 32, 3, 0)
    dA, dB, dC = _dev(A, k), _dev(B, n + 1), _dev(C)
    sg.sgemm_texld(dA, dB, dC, 1.5, 0.5)
    torch.cuda.synchronize()
    assert np.array_equal(dC.cpu().numpy(), oracle.sgemm_basic(A, B, C, 1.5, 0.5, basic=False))


def test_texld_many_calls_release_their_textures():
    # each call's texture objects are destroyed after its kernel: a long run
    # of calls on one stream keeps working and agrees with the plain path
    import torch
    m = n = k = 256
    A = torch.empty((m, k), device="cuda")
    B = torch.empty((k, n), device="cuda")
    sg.fill_random(A, 33, 1, 0)
    sg.fill_random(B, 33, 2, 0)
    C1 = torch.zeros((m, n), device="cuda")
    C2 = torch.zeros((m, n), device="cuda")
    for _ in range(2000):
        sg.sgemm_texld(A, B, C1, 1.0, 0.5)
        sg.sgemm(A, B, C2, 1.0, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(C1, C2)
