"""The fused kernel's lattice index without a division per axis, restated in float64 (CPU only).

The kernel (supertrack_b200/csrc/vcs_kernels.cu, the geometry block of the superimposition loop)
forms q = RN(a * RN(1/d)), takes k = (q + 1.5*2^52) - 1.5*2^52 (rint, ties to even) and, when
|q - k| >= 0.5 - 2^-20, decides with the correctly rounded division instead. That must equal the
reference's llrint(a / d) (VoxelConstrainedSphereMethod.cu:249-258) for every in-box quotient
(|q| < 2^21, the largest lattice side). numpy float64 operations round each step like the
kernel's explicit __dmul_rn/__dadd_rn/__dsub_rn.
"""
import numpy as np

K_MAGIC = 1.5 * 2.0 ** 52
RISK_BAND = 0.5 - 2.0 ** -20
Q_MAX = 2.0 ** 21


def fast_index(a, d):
    inv_d = 1.0 / d
    q = a * inv_d
    k = (q + K_MAGIC) - K_MAGIC
    near = np.abs(q - k) >= RISK_BAND
    return np.where(near, np.rint(a / d), k), near


def _diameters(rs):
    fixed = [2.0, 10.0, 100.0, 1000.0, 3.0, 7.0, 0.1, 1.0 / 3.0, 4.0, 0.125]
    return fixed + list(np.exp(rs.uniform(np.log(1e-3), np.log(1e4), 20)))


def test_random_in_box_quotients():
    rs = np.random.default_rng(0)
    for d in _diameters(rs):
        a = rs.uniform(-Q_MAX, Q_MAX, 400_000) * d
        k, near = fast_index(a, d)
        assert np.array_equal(k, np.rint(a / d)), d
        assert near.mean() < 1e-4                 # the exact division is rare


def test_near_half_integers():
    """a = RN((m + 1/2) d) and its neighbours up to 16 ulps away, over the whole index range:
    the quotients closest to a tie, where q and a/d may round to different integers."""
    rs = np.random.default_rng(1)
    plain_wrong = 0
    for d in _diameters(rs):
        m = np.concatenate([np.arange(-64, 64),
                            rs.integers(-int(Q_MAX) + 1, int(Q_MAX) - 1, 20_000)]).astype(np.float64)
        base = (m + 0.5) * d
        for steps in range(-16, 17):
            a = base.copy()
            if steps:
                toward = np.inf if steps > 0 else -np.inf
                for _ in range(abs(steps)):
                    a = np.nextafter(a, toward)
            k, _ = fast_index(a, d)
            exact = np.rint(a / d)
            assert np.array_equal(k, exact), (d, steps)
            plain_wrong += int(((a * (1.0 / d) + K_MAGIC) - K_MAGIC != exact).sum())
    assert plain_wrong > 0      # the samples include quotients that need the exact division


def test_exact_ties_round_to_even():
    """With d a power of two, (m + 1/2) d is exact, a/d is an exact tie, and llrint rounds it to
    the even neighbour."""
    for d in (0.25, 1.0, 4.0, 1024.0):
        m = np.arange(-5000, 5000, dtype=np.float64)
        a = (m + 0.5) * d
        k, near = fast_index(a, d)
        assert near.all()
        assert np.array_equal(k, np.rint(a / d))
        assert np.all(k % 2 == 0)
