"""bench.py's autotuner (CPU, with a stand-in for the library): it times
every (mode, CTAs per SM, W-scatter tiles, candidate tiles) of its grid on
the recorded batch, keeps the fastest, and leaves the batch cut and tuned to
that shape; a fixed CTAs-per-SM or mode narrows the grid."""
import bench


class FakeLib:
    def __init__(self):
        self.shape = None
        self.cps = None
        self.calls = []

    def batch_shape(self, w, l):
        self.shape = (w, l)
        return 1000 * w + l

    def batch_tune(self, cps):
        self.cps = cps


def fake_timer(lib, best):
    def time_mode(md, reps):
        key = (md, lib.cps, lib.shape)
        lib.calls.append(key)
        return 1.0 if key == best else 2.0 + 0.01 * len(lib.calls)
    return time_mode


def test_autotune_keeps_the_fastest_shape_and_mode():
    lib = FakeLib()
    best = (2, 4, (2, 1))
    tune, md, cps, gt, nitems = bench.autotune(lib, fake_timer(lib, best))
    assert (md, cps, gt) == (2, 4, (2, 1))
    assert lib.shape == (2, 1) and lib.cps == 4 and nitems == 2001
    n = sum(len(c) * len(w) * len(l) for c, w, l in bench.TUNE_GRID.values())
    assert len(tune) == n == len(lib.calls)
    assert tune["2:4x2x1"] == 1.0


def test_autotune_fixed_mode_and_ctas():
    lib = FakeLib()
    best = (1, 6, (1, 4))
    tune, md, cps, gt, _ = bench.autotune(lib, fake_timer(lib, best), fixed_cps=6, modes=(1,))
    assert (md, cps, gt) == (1, 6, (1, 4))
    assert all(k.startswith("1:6x") for k in tune)
