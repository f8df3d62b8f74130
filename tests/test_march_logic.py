"""The host-side march drivers of the warm-start study on a fake batch (CPU).

A fake case's residual follows a prescribed sequence per step; the drivers
must stop a case at its tolerance, at its FP32 rounding plateau (the
residual fell by less than 20% over 1000 steps below 1e-3) or when it
diverges, and the extrapolating driver must snapshot m + 2 iterates per
cycle, extrapolate only below `start`, and give up on a case whose
residual grew tenfold after an extrapolation.
"""
import numpy as np

from dgbgk._lib import DGBGK_ENONFINITE
from dgbgk.study import march_batch, march_batch_rre


class FakeCase:
    def __init__(self, res, ref=1.0):
        self.res = res          # function: step -> relative residual (nan: diverged)
        self.step = 0
        self.ref = ref
        self.snaps = []
        self.extrapolations = 0
        self.jump = None        # after an extrapolation, add this to the step count

    def residual_reference(self):
        return self.ref

    def snapshot(self, slot):
        if slot >= 0:
            self.snaps.append(slot)

    def extrapolate(self, n):
        assert n == len(self.snaps[-n:]) and self.snaps[-n:] == list(range(n))
        self.extrapolations += 1
        if self.jump:
            self.step += self.jump
        return np.ones(n - 1) / (n - 1)


class FakeBatch:
    """The library's batch semantics: cases left out by set_active, and
    cases stopped by a divergence, run no step and keep their status."""

    def __init__(self, cases):
        self.cases = cases
        self.active = np.ones(len(cases), dtype=bool)
        self.stopped = np.zeros(len(cases), dtype=bool)
        self.steps_run = np.zeros(len(cases), dtype=np.int64)

    def set_active(self, active):
        self.active = np.asarray(active, dtype=bool).copy()

    def advance(self, k, tol=0.0, raise_on_error=False):
        steps, last, status = [], [], []
        for i, c in enumerate(self.cases):
            if not self.active[i] or self.stopped[i]:
                steps.append(0)
                last.append(0.0)
                status.append(DGBGK_ENONFINITE if (self.active[i] and self.stopped[i]) else 0)
                continue
            n, r, st = 0, np.inf, 0
            for _ in range(k):
                c.step += 1
                n += 1
                r = c.res(c.step)
                if not np.isfinite(r):
                    st = DGBGK_ENONFINITE
                    self.stopped[i] = True
                    break
                if tol > 0 and r <= tol:
                    break
            self.steps_run[i] += n
            steps.append(n)
            last.append(r * c.ref)
            status.append(st)
        return {"steps": np.array(steps), "res_l2_last": np.array(last), "status": np.array(status, dtype=np.int32)}

    def last_ms(self):
        return 0.0

    def snapshot(self, slot, which=None):
        for i, c in enumerate(self.cases):
            if which is None or which[i]:
                c.snapshot(slot)

    def extrapolate(self, n, which=None):
        status = np.zeros(len(self.cases), dtype=np.int32)
        for i, c in enumerate(self.cases):
            if which is None or which[i]:
                c.extrapolate(n)
        return status, np.zeros((len(self.cases), n - 1))


def test_march_batch_stops_at_tolerance_plateau_and_divergence():
    fast = FakeCase(lambda k: 10 ** (-k / 500))                    # reaches 1e-8 at step 4000
    plateau = FakeCase(lambda k: max(10 ** (-k / 500), 2e-6))      # FP32 rounding plateau
    bad = FakeCase(lambda k: np.nan if k > 1500 else 1.0)
    cases = [fast, plateau, bad]
    b = FakeBatch(cases)
    steps, rel, status, _ = march_batch(b, cases, 1e-8, 60000)
    assert steps[0] == 4000 and rel[0] <= 1e-8
    assert status[1] == 0 and abs(rel[1] - 2e-6) < 1e-12 and steps[1] < 6000
    assert status[2] == DGBGK_ENONFINITE
    # finished cases are left out of later chunks: the diverged case ran
    # 1501 steps (its last one non-finite) and the converged ones no step
    # past their stop
    assert b.steps_run[2] == 1501 and steps[2] == 1501
    assert b.steps_run[0] == 4000 and b.steps_run[1] == steps[1]
    # and the batch is handed back with every case active
    assert b.active.all()


def test_rre_driver_cycles_and_guard():
    good = FakeCase(lambda k: 10 ** (-k / 1000))
    good.jump = 300                     # an extrapolation skips 300 steps of decay
    worse = FakeCase(lambda k: 10 ** (-k / 1000) * (20.0 if worse.extrapolations else 1.0))
    cases = [good, worse]
    steps, rel, status, _ = march_batch_rre(FakeBatch(cases), cases, 1e-8, 60000, stall_below=0.0)
    assert rel[0] <= 1e-8 and good.extrapolations > 3
    # no extrapolation above start = 1e-2 (residual 1e-2 at step 2000)
    assert steps[0] < 8000
    # the case whose residual grew tenfold after its first extrapolation stops extrapolating
    assert worse.extrapolations == 1 and rel[1] <= 1e-8
    # m + 2 = 10 snapshots per cycle
    assert len(good.snaps) == 10 * good.extrapolations


def test_rre_driver_confirms_a_warm_start_convergence():
    # a transient whose residual dips to 1e-8 at step 3000, rises to 1e-5 at
    # step 6000 and then decays for good (1e-8 again at step 9000)
    def dip(k):
        if k <= 3000:
            return 10 ** (-k / 375)
        if k <= 6000:
            return 1e-8 * 10 ** ((k - 3000) / 1000)
        return 1e-5 * 10 ** (-(k - 6000) / 1000)

    plain = FakeCase(lambda k: 10 ** (-k / 500))   # 1e-8 at step 4000, falling
    cases = [FakeCase(dip), FakeCase(dip), plain]
    # without the confirmation the dip counts as convergence
    steps, rel, status, _ = march_batch_rre(FakeBatch(cases[:1]), cases[:1], 1e-8, 60000, stall_below=0.0)
    assert rel[0] <= 1e-8 and 3000 <= steps[0] < 3100
    # with it the transient case marches on to its real convergence, and a
    # case whose residual keeps falling stops `confirm` steps after its hit
    steps, rel, status, _ = march_batch_rre(FakeBatch(cases[1:]), cases[1:], 1e-8, 60000, stall_below=0.0,
                                            confirm=200)
    assert rel[0] <= 1e-8 and 9000 <= steps[0] <= 9400
    assert rel[1] <= 1e-8 and 4000 <= steps[1] <= 4300
    assert (status == 0).all()
