"""Per-tet rest data for the SNK1 element kernel, as the reference prepares
it at load time (StiffGIPC/gl_main.cu:600-628): Dm^-1 (row-major), the rest
volume |det Dm| / 6 and the Lame rates u = 4/3 mu, r = lambda + 5/6 mu
(gl_main.cu:586-590, 618-624)."""
from __future__ import annotations

import numpy as np


def rest_data(tets, X, E, nu):
    T = np.asarray(tets, np.int64).reshape(-1, 4)
    Xr = np.asarray(X, np.float64).reshape(-1, 3)
    Dm = np.stack([Xr[T[:, c + 1]] - Xr[T[:, 0]] for c in range(3)], axis=2)
    E = np.broadcast_to(np.asarray(E, np.float64), (len(T),))
    mu, la = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    return np.linalg.inv(Dm).reshape(-1, 9), np.abs(np.linalg.det(Dm)) / 6.0, 4 * mu / 3, la + 5 * mu / 6
