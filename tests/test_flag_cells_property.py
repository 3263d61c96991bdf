"""The boundary-flag cell neighbourhoods, restated in float64 (CPU only).

k_prep_flag (supertrack_b200/csrc/vcs_kernels.cu, cell_of / cell_nbr) puts a deposit in the flag
cell floor(RN(c * RN(1/s))) per axis, for a side s slightly above d (27 neighbour cells probed) or
slightly above 2d (8 probed: per axis the deposit's cell and the neighbour on the side of the half
of the cell it lies in, u - floor(u) < 1/2 choosing the lower one). A deposit within distance d
of another must lie in one of the probed cells of the other, or the flag of a sphere with hits in
two windows could be missed. numpy float64 products and subtractions round like the kernel's
st_dmul and st_dsub.
"""
import numpy as np


def _sides(d):
    return d * (1.0 + 2.0 ** -10), 2.0 * d * (1.0 + 2.0 ** -10)


def _cell_u(c, s):
    return c * (1.0 / s)


def _probed27(p, q, s):
    cp, cq = np.floor(_cell_u(p, s)), np.floor(_cell_u(q, s))
    return np.all(np.abs(cq - cp) <= 1, axis=-1)


def _probed8(p, q, s):
    u = _cell_u(p, s)
    cp = np.floor(u)
    side = np.where(u - cp < 0.5, -1.0, 1.0)
    cq = np.floor(_cell_u(q, s))
    return np.all((cq == cp) | (cq == cp + side), axis=-1)


def _pairs(rs, d, n, scale):
    p = rs.uniform(-scale, scale, size=(n, 3))
    v = rs.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    length = d * rs.random(n)
    length[: n // 4] = d
    q = p + v * length[:, None]
    # exactly d along one axis, from points on the centre planes and near the edges of cells
    s2 = 2.0 * d * (1.0 + 2.0 ** -10)
    m = n // 4
    frac = rs.choice([0.5, np.nextafter(0.5, 0), np.nextafter(0.5, 1), 0.0, 1e-12,
                      1.0 - 1e-12, 0.25], size=(m, 3))
    p[-m:] = (np.floor(_cell_u(p[-m:], s2)) + frac) * s2
    q[-m:] = p[-m:]
    axis = rs.integers(0, 3, m)
    q[np.arange(n - m, n), axis] += rs.choice([-d, d], m)
    return p, q


def test_every_deposit_within_d_is_in_a_probed_cell():
    rs = np.random.default_rng(7)
    for d in (2.0, 10.0, 100.0, 1000.0, 1.0, 0.1, 3.0, 1.0 / 3.0, 7.25):
        s1, s2 = _sides(d)
        for scale in (5.0 * d, 2500.0, 5000.0, 2.0 ** 18 * d):
            p, q = _pairs(rs, d, 40_000, scale)
            # within d up to the roundings of the coordinates (the sides' 2^-10 margin is far
            # larger)
            assert np.all(np.linalg.norm(q - p, axis=1) <= d + 1e-12 * (scale + d))
            assert np.all(_probed27(p, q, s1))
            assert np.all(_probed27(q, p, s1))
            assert np.all(_probed8(p, q, s2))
            assert np.all(_probed8(q, p, s2))


def test_eight_cells_are_fewer_probes_not_a_looser_test_of_distance():
    """Per axis the 8-cell neighbourhood is two cells: the point's own cell is always probed,
    and a point two sides away never is."""
    rs = np.random.default_rng(3)
    d = 2.0
    _, s2 = _sides(d)
    p = rs.uniform(-1000, 1000, size=(10_000, 3))
    assert np.all(_probed8(p, p, s2))
    far = p + np.array([2.0 * s2 + 1e-9, 0.0, 0.0])
    assert not np.any(_probed8(p, far, s2))
