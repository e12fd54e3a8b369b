"""CPU restatement of the learned collision step's features and transform.

TEST INFRASTRUCTURE ONLY: the checker of picopic_b200's learned collision
kernels (pcg_learned.cu).  From the per-cell moment sums of
Domain.cell_moments it computes, in float64, the 13 features, the collision
scale S and, for given network outputs, the per-axis velocity scales of the
moment-matching transform, with the same definitions as the kernels.
"""
import numpy as np

PI, EPS0, E, LOGL = 3.1415926535897932, 8.85e-12, 1.6e-19, 10.0


def features(m, grid, dt, masses, charges):
    """(cells, 13) features (NaN where a list has fewer than 2 particles or
    no positive temperature), S (cells,), and the state per cell:
    T (cells, 2, 3), Tm (cells, 2), W (cells, 2), u (cells, 2, 3)."""
    cells = m.shape[0]
    i = np.arange(cells) // grid.nz
    vol = PI * grid.dz * grid.dr ** 2 * (2.0 * i + 1)
    T, u, W, N = np.zeros((cells, 2, 3)), np.zeros((cells, 2, 3)), m[:, [1, 9]], m[:, [0, 8]]
    with np.errstate(invalid="ignore", divide="ignore"):
        for l in (0, 1):
            ml = m[:, 8 * l:8 * l + 8]
            u[:, l] = ml[:, 2:5] / ml[:, 1:2]
            T[:, l] = masses[l] * (ml[:, 5:8] / ml[:, 1:2] - u[:, l] ** 2) / E
        Tm = T.mean(2)
        n = W / vol[:, None]

        def s_of(a, b):
            mab = masses[a] * masses[b] / (masses[a] + masses[b])
            v2 = 3.0 * E * (Tm[:, a] / masses[a] + Tm[:, b] / masses[b])
            qq = charges[a] * charges[b]
            return np.maximum(n[:, a], n[:, b]) * dt * LOGL * qq * qq / (4 * PI * (EPS0 * mab) ** 2 * v2 * np.sqrt(v2))

        see, sei, sii = s_of(0, 0), s_of(0, 1), s_of(1, 1)
        x = np.zeros((cells, 13))
        x[:, 0:3] = T[:, 0] / Tm[:, 0:1] - 1
        x[:, 3:6] = T[:, 1] / Tm[:, 1:2] - 1
        x[:, 6] = np.log(Tm[:, 1] / Tm[:, 0])
        x[:, 7], x[:, 8], x[:, 9] = np.log10(see), np.log10(sei), np.log10(sii)
        x[:, 10] = np.sqrt(((u[:, 0] - u[:, 1]) ** 2).sum(1) / (3 * E * Tm[:, 0] / masses[0]))
        x[:, 11] = np.log(n[:, 1] / n[:, 0])
        x[:, 12] = 1 / np.sqrt(N.sum(1))
    ok = (N >= 2).all(1) & (W > 0).all(1) & (Tm > 0).all(1)
    x[~ok] = np.nan
    S = np.where(ok, see + sei + sii, 0.0)
    return x, S, (T, Tm, W, u)


def transform_scales(y, S, state):
    """Per-axis velocity scales (cells, 2, 3) of the learned step for network
    outputs y (cells, 6) in physical units: T' = T + Tm S y, one factor per
    cell keeps sum_s W_s sum_a T_s,a, then sqrt(T' / T)."""
    T, Tm, W, _ = state
    Tn = T + (Tm * S[:, None])[:, :, None] * y.reshape(-1, 2, 3)
    e0 = (W[:, :, None] * T).sum((1, 2))
    e1 = (W[:, :, None] * Tn).sum((1, 2))
    f = np.where(e1 > 0, e0 / e1, 1.0)
    Tn = np.maximum(Tn * f[:, None, None], 1e-6 * Tm[:, :, None])
    return np.sqrt(Tn / T)
