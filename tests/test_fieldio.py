"""The plugin's field gather and rate scatter on the device (gf_gather_states,
gf_scatter_rates; the reference does them on the host, getY0 in
gpuChemistryModel.C:33-53 and the RR_ loop of computeRRAndChemDeltaT,
:351-356).

CPU: the kernels' tile index arithmetic, restated loop for loop (grid-stride
tiles of 16 cells, 256 threads), against numpy transposes for ragged sizes —
every read and write checked to stay inside its array; the argument checks of
the C ABI. GPU: the kernels themselves, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from gpufoam_b200 import _native as N

TILE, THREADS = 16, 256


def emulate_gather(fields, T, p, n, nS, ld, grid):
    """gather_states_kernel's loops; returns y and asserts every index is in bounds."""
    ne = nS + 2
    y = np.full((n * ld,), np.nan)
    for b in range(grid):
        c0 = b * TILE
        while c0 < n:
            nc = min(TILE, n - c0)
            tile = np.full(TILE * ne, np.nan)
            for tid in range(THREADS):
                for t in range(tid, ne * TILE, THREADS):
                    e, j = divmod(t, TILE)
                    if j < nc:
                        src = fields[e] if e < nS else (T if e == nS else p)
                        assert 0 <= c0 + j < n and 0 <= j * ne + e < TILE * ne
                        tile[j * ne + e] = src[c0 + j]
            for tid in range(THREADS):
                for t in range(tid, nc * ne, THREADS):
                    j, e = divmod(t, ne)
                    assert 0 <= (c0 + j) * ld + e < n * ld
                    y[(c0 + j) * ld + e] = tile[j * ne + e]
            c0 += grid * TILE
    return y.reshape(n, ld)


def emulate_scatter(RR, n, nS, ld, grid):
    out = [np.full(n, np.nan) for _ in range(nS)]
    for b in range(grid):
        c0 = b * TILE
        while c0 < n:
            nc = min(TILE, n - c0)
            tile = np.full(TILE * nS, np.nan)
            for tid in range(THREADS):
                for t in range(tid, nc * nS, THREADS):
                    j, i = divmod(t, nS)
                    assert 0 <= (c0 + j) * ld + i < n * ld
                    tile[j * nS + i] = RR[(c0 + j) * ld + i]
            for tid in range(THREADS):
                for t in range(tid, nS * TILE, THREADS):
                    i, j = divmod(t, TILE)
                    if j < nc:
                        assert 0 <= c0 + j < n
                        out[i][c0 + j] = tile[j * nS + i]
            c0 += grid * TILE
    return out


@pytest.mark.parametrize("n, nS, ld, grid", [(1, 1, 3, 1), (15, 10, 12, 1), (17, 10, 13, 1), (33, 53, 55, 2),
                                             (40, 7, 9, 5), (5, 300, 302, 1)])
def test_tile_index_arithmetic(n, nS, ld, grid):
    rng = np.random.default_rng(n * 1000 + nS)
    fields = [rng.standard_normal(n) for _ in range(nS)]
    T, p = rng.uniform(300, 3000, n), rng.uniform(1e5, 4e6, n)
    y = emulate_gather(fields, T, p, n, nS, ld, grid)
    ref = np.column_stack(fields + [T, p])
    assert np.array_equal(y[:, :nS + 2], ref)
    RR = rng.standard_normal((n, ld)).ravel()
    out = emulate_scatter(RR, n, nS, ld, grid)
    assert all(np.array_equal(out[i], RR.reshape(n, ld)[:, i]) for i in range(nS))


def test_argument_checks():
    from gpufoam_b200 import build as B
    B.build()
    lib = N.load()
    one = (C.c_void_p * 1)(C.c_void_p(8))
    null1 = (C.c_void_p * 1)(None)
    # invalid before any device work
    assert lib.gf_gather_states(4, 0, one, None, None, None, 2, None) == 1
    assert lib.gf_gather_states(4, 301, one, None, None, None, 400, None) == 1
    assert lib.gf_gather_states(4, 1, one, None, None, None, 2, None) == 1      # ld_y < nS + 2
    assert lib.gf_gather_states(4, 1, null1, C.c_void_p(8), C.c_void_p(8), C.c_void_p(8), 3, None) == 1
    assert lib.gf_gather_states(0, 1, one, None, None, None, 3, None) == 0      # nothing to do
    assert lib.gf_scatter_rates(4, 1, C.c_void_p(8), 0, one, None) == 1         # ld_rr < nS
    assert lib.gf_scatter_rates(4, 1, None, 1, one, None) == 1
    assert lib.gf_scatter_rates(4, 1, C.c_void_p(8), 1, null1, None) == 1
    assert lib.gf_scatter_rates(0, 1, None, 1, one, None) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n, nS, ld", [(1, 1, 3), (17, 10, 12), (1000, 53, 55), (4099, 100, 104), (70, 300, 302)])
def test_gather_scatter_on_gpu(n, nS, ld):
    import torch

    from gpufoam_b200 import evaluator as E
    g = torch.Generator().manual_seed(n + nS)
    fields = [torch.randn(n, dtype=torch.float64, generator=g).cuda() for _ in range(nS)]
    T = (torch.rand(n, dtype=torch.float64, generator=g) * 2000 + 300).cuda()
    p = (torch.rand(n, dtype=torch.float64, generator=g) * 4e6).cuda()
    y = E.gather_states(fields, T, p, ld=ld)
    ref = torch.stack(fields + [T, p], dim=1)
    assert torch.equal(y[:, :nS + 2], ref) and bool((y[:, nS + 2:] == 0).all())
    RR = torch.randn((n, ld), dtype=torch.float64, generator=g).cuda()
    out = [torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(nS)]
    E.scatter_rates(RR, out)
    torch.cuda.synchronize()
    assert all(torch.equal(out[i], RR[:, i]) for i in range(nS))
