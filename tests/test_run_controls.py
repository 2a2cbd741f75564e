"""The reference loop's cooperative controls on the host (src/gpe.f90:136-159,
src/io.f90:1566-1595): deleting RUNNING stops the run with an end_state,
creating SAVE produces one snapshot.  Driven with a stand-in for the solver
(host-side fault injection; no GPU)."""
import os

import numpy as np

from gpe_b200.restart import read_end_state, write_end_state
from gpe_b200.solver import GpeParams, run_loop


class FakeSolver:
    def __init__(self):
        self.prm = GpeParams(nx=4, ny=4, nz=4, eqn_to_solve=4, real_time=True)
        self.t, self.im_t, self.p, self.dt = 0.0, 0.0, 0, complex(0.1, 0.0)
        self.calls = 0
        self.hook = None

    def solver(self):
        self.calls += 1
        self.t += 0.1
        if self.hook:
            self.hook(self)

    def get_norm(self):
        return 1.0

    def save_end_state(self, path):
        write_end_state(path, np.full((4, 4, 4), complex(self.calls, 0)), self.p, self.t,
                        self.im_t, self.dt)


def test_deleting_running_stops_with_an_end_state(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()

    def stop_after_three(sv):
        if sv.calls == 3:
            os.remove(os.path.join(d, "RUNNING"))
    s.hook = stop_after_three
    out = run_loop(s, 10, run_dir=d)
    assert s.calls == 3 and len(out) == 3
    st = read_end_state(os.path.join(d, "end_state.dat"), expect=(4, 4, 4))
    assert st.p == 3 and st.psi[0, 0, 0] == 3


def test_save_file_gives_one_snapshot(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()

    def request_save(sv):
        if sv.calls == 2:
            open(os.path.join(d, "SAVE"), "w").close()
    s.hook = request_save
    run_loop(s, 5, run_dir=d)
    assert s.calls == 5
    snaps = sorted(f for f in os.listdir(d) if f.startswith("snapshot_"))
    assert snaps == ["snapshot_0000002.dat"] and not os.path.exists(os.path.join(d, "SAVE"))
    assert read_end_state(os.path.join(d, snaps[0])).psi[0, 0, 0] == 2
