"""The plain FP64 side of the time-to-equilibrium comparison
(multiphaselb_b200.ensemble.run_plain): every case runs on the tile the
autotuner keeps for its lattice, found on a throwaway handle before the timed
region, so the plain wall times hold no tuning.  CPU only: a stand-in for the
library handle records what the runner asks of it."""
import numpy as np

from multiphaselb_b200 import ensemble


class StandIn:
    made = []

    def __init__(self, case, path=None, precision=None, tile_config=0, **kw):
        self.case, self.tile_config = case, tile_config
        self.stepped, self.ran = 0, False
        StandIn.made.append(self)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def upload_case(self):
        pass

    def initialize(self):
        pass

    def sync(self):
        pass

    def step(self, n):
        self.stepped += n

    def info(self):
        # the tuner's pick on a tuned handle (0-based), the forced one otherwise
        return {"tile_config": 8 if self.tile_config == 0 else self.tile_config - 1}

    def run_to_equilibrium(self, max_steps, K, tol):
        self.ran = True
        return 3 * K, 1e-10

    def download(self):
        return {"rho": np.full(self.case.n, 0.3)}


def test_plain_runs_on_the_tuned_tile_outside_the_timing(monkeypatch):
    StandIn.made = []
    monkeypatch.setattr(ensemble, "Lattice", StandIn)
    specs = [dict(L=64, t_ratio=0.8, radius=12.0), dict(L=96, t_ratio=0.7, radius=20.0)]
    out = ensemble.run_plain(specs, 1000, 1e-9, 400000)
    assert [o["steps"] for o in out] == [3000, 3000]
    assert len(StandIn.made) == 2 * len(specs)
    for i in range(len(specs)):
        probe, timed = StandIn.made[2 * i], StandIn.made[2 * i + 1]
        # the throwaway handle is tuned (tile_config 0) by its first step and never run to equilibrium
        assert probe.tile_config == 0 and probe.stepped == 1 and not probe.ran
        # the timed handle takes the pick (1-based) and starts from the initial state
        assert timed.tile_config == 9 and timed.stepped == 0 and timed.ran
