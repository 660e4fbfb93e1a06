"""Data files of the reference's DSP-WENO trainer.

DSP-WENO_trainer/DSP-WENO_network_trainer.py:305-333 reads one sample per line,
comma-separated.  With ``tanh_theta`` (its default) a line holds 23 values:

    u0 u1 u2 u3 | theta- theta+ | tanh(theta-) tanh(theta+) del1 del2 del3 |
    vertex x 0..4 | vertex y 0..4 | target left, target right

and the trainer feeds columns 6-20 to the network (5 inputs, then the 10
vertex coordinates), compares its left / right interface values with columns
21-22, and takes the cell values from columns 0-3.  Without ``tanh_theta`` the
two tanh columns are absent (21 values; the network inputs are theta-, theta+,
del1..del3).  ``Trainer.export_rows`` produces rows in the 23-column order from
samples collected on the GPU; ``read_trainer_file`` returns the stencils and
targets of such a file for ``Trainer.set_data``.
"""
from __future__ import annotations

import numpy as np

COLUMNS = (["u0", "u1", "u2", "u3", "theta_m", "theta_p", "tanh_theta_m", "tanh_theta_p", "del1", "del2", "del3"]
           + [f"vx{k}" for k in range(5)] + [f"vy{k}" for k in range(5)] + ["target_left", "target_right"])
NCOLS = len(COLUMNS)          # 23
_TANH = (6, 7)


def width(tanh_theta: bool = True) -> int:
    return NCOLS if tanh_theta else NCOLS - len(_TANH)


def write_trainer_file(path, rows, tanh_theta: bool = True) -> int:
    """Write 23-column rows (``Trainer.export_rows``) as the trainer's data
    file; without tanh_theta the two tanh columns are left out.  Returns the
    number of lines."""
    rows = np.asarray(rows, dtype=np.float64)
    if rows.ndim != 2 or rows.shape[1] != NCOLS:
        raise ValueError(f"expected rows of {NCOLS} values, got shape {rows.shape}")
    if not tanh_theta:
        rows = np.delete(rows, _TANH, axis=1)
    np.savetxt(path, rows, delimiter=",", fmt="%.17g")
    return rows.shape[0]


def read_trainer_file(path, tanh_theta: bool = True):
    """(stencils (n, 4), targets (n, 2), all columns (n, width)) of a trainer
    data file."""
    a = np.loadtxt(path, delimiter=",", ndmin=2, dtype=np.float64)
    w = width(tanh_theta)
    if a.shape[1] != w:
        raise ValueError(f"{path}: {a.shape[1]} values per line, expected {w}")
    return a[:, 0:4].copy(), a[:, w - 2:w].copy(), a
