"""Data files of the reference's DSP-WENO trainer (dspw.traindata): the
column layout its reader slices (DSP-WENO_trainer/DSP-WENO_network_trainer.py:
305-333 and the batch slicing at :395-398), checked by parsing our files the way
that reader does; and (GPU) the rows the GPU trainer exports."""
import numpy as np
import pytest

import oracle as O
from dspw.traindata import COLUMNS, NCOLS, read_trainer_file, width, write_trainer_file


def _reference_reader(path, tanh_theta=True):
    """The trainer's view of a data file: per line a tag, the tokens, then the
    4 cell values again (unscaled copies); the network input columns start at
    7 (tanh_theta) or 5; the targets are the last two tokens."""
    size = 23 if tanh_theta else 21
    start = 7 if tanh_theta else 5
    out = []
    for count, line in enumerate(open(path).read().splitlines(), 1):
        tok = line.split(",")
        t = np.zeros(size + 1 + 4)
        t[0] = count
        for i in range(1, size + 1):
            t[i] = float(tok[i - 1])
            if i < 5:
                t[size + i] = float(tok[i - 1])
        out.append(t)
    d = np.array(out)
    return dict(inputs=d[:, start:start + 15], actual=d[:, size - 1:size + 1], orig=d[:, size + 1:size + 5])


def _rows(n, seed=3):
    return np.random.default_rng(seed).normal(size=(n, NCOLS))


@pytest.mark.parametrize("tanh_theta", [True, False])
def test_layout_as_the_trainer_reads_it(tmp_path, tanh_theta):
    rows = _rows(50)
    p = tmp_path / "data.dat"
    assert write_trainer_file(p, rows, tanh_theta) == 50
    v = _reference_reader(p, tanh_theta)
    np.testing.assert_array_equal(v["orig"], rows[:, 0:4])
    np.testing.assert_array_equal(v["actual"], rows[:, 21:23])
    if tanh_theta:   # tanh(theta-), tanh(theta+), del1..3, vertices
        np.testing.assert_array_equal(v["inputs"], rows[:, 6:21])
    else:            # theta-, theta+, del1..3, vertices
        np.testing.assert_array_equal(v["inputs"], np.concatenate([rows[:, 4:6], rows[:, 8:21]], axis=1))
    s, t, a = read_trainer_file(p, tanh_theta)
    np.testing.assert_array_equal(s, rows[:, 0:4])
    np.testing.assert_array_equal(t, rows[:, 21:23])
    assert a.shape == (50, width(tanh_theta))


def test_bad_files_are_rejected(tmp_path):
    with pytest.raises(ValueError):
        write_trainer_file(tmp_path / "x.dat", np.zeros((3, 22)))
    p = tmp_path / "y.dat"
    write_trainer_file(p, _rows(4))
    with pytest.raises(ValueError):
        read_trainer_file(p, tanh_theta=False)
    assert COLUMNS[6] == "tanh_theta_m" and COLUMNS[-1] == "target_right"


@pytest.mark.gpu
def test_trainer_export_rows(tmp_path):
    """Exported rows: the network inputs and vertices are those of the
    reference's forward (oracle or_nn_features) for the sample's cell values,
    which the trainer holds in FP32; the file reads back into a trainer."""
    from _common import net
    from dspw import Trainer
    rng = np.random.default_rng(7)
    st = rng.uniform(-2, 2, size=(3000, 4))
    st[:10, 2] = st[:10, 1]                      # flat middle pair: skipped by the trainer
    tg = rng.uniform(-2, 2, size=(3000, 2))
    tr = Trainer(net(), batch=512)
    tr.set_data(st, tg)
    rows = tr.export_rows()
    assert rows.shape == (2990, NCOLS)
    u = st[10:].astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(rows[:, 0:4], u)
    np.testing.assert_array_equal(rows[:, 21:23], tg[10:].astype(np.float32).astype(np.float64))
    for k in range(0, 2990, 97):
        f, vx, vy = O.nn_features(u[k])
        np.testing.assert_allclose(rows[k, 6:11], f, rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(rows[k, 11:16], vx, rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(rows[k, 16:21], vy, rtol=1e-14, atol=1e-15)
        np.testing.assert_allclose(np.tanh(rows[k, 4:6]), f[0:2], rtol=1e-13, atol=1e-15)
    p = tmp_path / "data.dat"
    write_trainer_file(p, rows)
    s2, t2, _ = read_trainer_file(p)
    tr2 = Trainer(net(), batch=512)
    tr2.set_data(s2, t2)
    # the mean loss is taken over all samples, skipped ones contributing 0
    assert abs(tr2.eval() * 2990 - tr.eval() * 3000) <= 1e-5 * abs(tr.eval() * 3000)
