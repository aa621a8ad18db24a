"""The reference's own marker-exchange tests, run on the oracle's exchangeMarkers (MarkerExchange.jl:8-163) as the
reference runs them on MPI ranks: test/test_MarkerExchange_1P.jl, _9P.jl and _varP.jl.  The device exchange is
bit-identical to the oracle's (tests/test_domains_markers.py), so these pin it too.  Julia's rand is replaced by
a seeded numpy generator with the same distributions."""
import numpy as np
import pytest

import oracle


def test_exchange_1p_is_the_identity():
    """test/test_MarkerExchange_1P.jl:19-51: one rank, jittered markers (3 per cell), random properties."""
    Nx, Ny, L = 7, 11, 10.0
    dx, dy = L / (Nx - 1), L / (Ny - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    x, y = oracle.initialize_markers(3, lx, ly, dx, dy, Nx, Ny, 1.0, 0)
    rng = np.random.default_rng(0)
    rho, mu = rng.random(x.size), rng.random(x.size)
    out = oracle.exchange_markers({(0, 0): (x, y, rho, mu)}, (1, 1), lx, ly, dx, dy)[(0, 0)]
    for got, want in zip(out, (x, y, rho, mu)):
        assert np.array_equal(got, want)


def test_exchange_9p_known_answer():
    """test/test_MarkerExchange_9P.jl:18-107: 3 x 3 ranks, each with a marker in all eight directions and one in
    the centre (local domain 1 x 1, dx = dy = 0.4), properties encoding the source rank; no marker is lost and
    the centre rank holds exactly the nine expected markers with their source ranks."""
    dims, dx, dy = (3, 3), 0.4, 0.4
    markers = {}
    for cx in range(3):
        for cy in range(3):
            i = np.arange(9)
            markers[(cx, cy)] = (0.1 + 0.4 * (i % 3), 0.1 + 0.4 * (i // 3), np.full(9, float(cx)), np.full(9, float(cy)))
    out = oracle.exchange_markers(markers, dims, 1.0, 1.0, dx, dy)
    for c in markers:
        assert all(v.size == 9 for v in out[c])                                       # :59-62
    m = np.stack(out[(1, 1)], axis=1)
    m = m[np.lexsort((m[:, 3], m[:, 2], m[:, 1], m[:, 0]))]                           # sortslices, :67
    want = [(0.3, 0.3, 0, 0), (0.3, 0.5, 0, 1), (0.3, 0.7, 0, 2), (0.5, 0.3, 1, 0), (0.5, 0.5, 1, 1),
            (0.5, 0.7, 1, 2), (0.7, 0.3, 2, 0), (0.7, 0.5, 2, 1), (0.7, 0.7, 2, 2)]    # :69-104
    for row, (x, y, sx, sy) in zip(m, want):
        assert np.isclose(row[0], x) and np.isclose(row[1], y) and row[2] == sx and row[3] == sy


# test/test_MarkerExchange_varP.jl:12-51: the 26 x 32-point global grid on 1 to 9 ranks
VARP_GRIDS = [((1, 1), 26, 32), ((1, 2), 26, 17), ((2, 1), 14, 32), ((1, 3), 26, 12), ((3, 1), 10, 32),
              ((4, 1), 8, 32), ((2, 2), 14, 17), ((2, 3), 14, 12), ((3, 2), 10, 17), ((4, 2), 8, 17), ((3, 3), 10, 12)]


def _varp_markers(rng, Nx, Ny, dx, dy):
    """init_markers of test/test_MarkerExchange_varP.jl:53-84: 17 markers near the low (l) and high (h) edges,
    half a cell in from them, and in the middle (m)."""
    def l(N, d):
        return 0.005 * d + 0.49 * d * rng.random()

    def h(N, d):
        return (N - 1) * d - (0.005 * d + 0.49 * d * rng.random())

    def m(N, d):
        return 0.505 * d + ((N - 3) * d + 0.99 * d) * rng.random()

    x = [l(Nx, dx), l(Nx, dx), l(Nx, dx)]
    y = [l(Ny, dy), m(Ny, dy), h(Ny, dy)]
    x += [v + 0.5 * dx for v in (l(Nx, dx), l(Nx, dx), l(Nx, dx))]
    y += [l(Ny, dy) + 0.5 * dy, m(Ny, dy), h(Ny, dy) - 0.5 * dy]
    x += [m(Nx, dx) for _ in range(5)]
    y += [l(Ny, dy), l(Ny, dy) + 0.5 * dy, m(Ny, dy), h(Ny, dy) - 0.5 * dy, h(Ny, dy)]
    x += [v - 0.5 * dx for v in (h(Nx, dx), h(Nx, dx), h(Nx, dx))]
    y += [l(Ny, dy) + 0.5 * dy, m(Ny, dy), h(Ny, dy) - 0.5 * dy]
    x += [h(Nx, dx), h(Nx, dx), h(Nx, dx)]
    y += [l(Ny, dy), m(Ny, dy), h(Ny, dy)]
    n = len(x)
    return np.array(x), np.array(y), rng.random(n) * 1000, rng.random(n) * 100000


def _gather(markers, dims, lx, ly, dx, dy):
    """gather_markers! (GlobalGather.jl:10-48): rank order (x slowest), local -> global by coords * (l - d)."""
    coords = [(cx, cy) for cx in range(dims[0]) for cy in range(dims[1])]
    return (np.concatenate([markers[c][0] + c[0] * (lx - dx) for c in coords]),
            np.concatenate([markers[c][1] + c[1] * (ly - dy) for c in coords]),
            np.concatenate([markers[c][2] for c in coords]), np.concatenate([markers[c][3] for c in coords]))


@pytest.mark.parametrize("dims,Nx,Ny", VARP_GRIDS)
def test_exchange_varp(dims, Nx, Ny):
    """test/test_MarkerExchange_varP.jl:91-204: after the exchange every rank's markers lie inside its bounds
    (half a cell in from a shared edge in y), and the gathered markers before and after are the same set with
    the same properties."""
    n_ranks = dims[0] * dims[1]
    assert dims[0] * (Nx - 2) + 2 == 26 and dims[1] * (Ny - 2) + 2 == 32                 # :97
    dx, dy = 0.5, 0.4
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(10 * dims[0] + dims[1])
    while True:                                                                        # :119-132
        markers = {(cx, cy): _varp_markers(rng, Nx, Ny, dx, dy) for cx in range(dims[0]) for cy in range(dims[1])}
        g1 = _gather(markers, dims, lx, ly, dx, dy)
        crit = np.sort(g1[0] * lx * n_ranks + g1[1])
        if np.min(np.diff(crit)) > 1e-12 * np.max(crit):
            break
    out = oracle.exchange_markers(markers, dims, lx, ly, dx, dy)
    for (cx, cy), (x, y, _, _) in out.items():                                         # TEST 1, :149-173
        if cx == 0:
            assert np.all(x > 0)
        if cx == dims[0] - 1:
            assert np.all(x < (Nx - 1) * dx)
        assert np.all(y > 0) if cy == 0 else np.all(y > 0.5 * dy)
        assert np.all(y < (Ny - 1) * dy) if cy == dims[1] - 1 else np.all(y < (Ny - 1) * dy - 0.5 * dy)
    g2 = _gather(out, dims, lx, ly, dx, dy)                                            # TEST 2, :175-200
    assert g1[0].size == g2[0].size == 17 * n_ranks
    o1 = np.argsort(g1[0] * lx * n_ranks + g1[1])
    o2 = np.argsort(g2[0] * lx * n_ranks + g2[1])
    assert np.allclose(g1[0][o1], g2[0][o2]) and np.allclose(g1[1][o1], g2[1][o2])
    assert np.array_equal(g1[2][o1], g2[2][o2]) and np.array_equal(g1[3][o1], g2[3][o2])
