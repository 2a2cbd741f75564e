"""The reference loop's cooperative controls and output cadence on the host
(src/gpe.f90:126-278, src/io.f90:1566-1595): deleting RUNNING stops the run
with an end_state, creating SAVE produces one IDL surface, and the io_params
cadence writes the reference's files.  Driven with a stand-in for the solver
(host-side fault injection; no GPU)."""
import os

import numpy as np

from gpe_b200 import output
from gpe_b200.restart import read_end_state, write_end_state
from gpe_b200.solver import GpeParams, OutputParams, run_loop


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

    def state(self):
        return np.full((4, 4, 4), complex(self.calls, 0))

    def save_end_state(self, path):
        write_end_state(path, self.state(), self.p, self.t, self.im_t, self.dt)

    def get_state(self):
        return self.state()

    def grid(self):
        g = np.linspace(-1.0, 1.0, 4)
        return g, g, g

    def energy(self):
        return 64.0 * (self.calls + 1), 0.0

    def get_site(self, i, j, k):
        return complex(self.calls, 0.5)

    def linelength(self):
        return 2.5 * self.calls

    def zeros(self):
        return np.array([1] + [0] * 11), np.array([[1.0, 2.0, 3.0]])

    def condensed_particles(self):
        from gpe_b200.spectral import Condensate
        row = dict(M_density=1.0, n0_over_V=0.5, M=8.0, n0=32.0, temp=0.1, temp2=0.2,
                   H_over_V=0.3)
        return Condensate(row, np.arange(7.0), np.arange(7), np.arange(2.0))


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
    st = read_end_state(os.path.join(d, "proc00", "end_state.dat"), expect=(4, 4, 4))
    assert st.p == 3 and st.psi[0, 0, 0] == 3


def test_save_file_gives_one_idl_surface(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()

    def request_save(sv):
        if sv.calls == 2:
            open(os.path.join(d, "SAVE"), "w").close()
    s.hook = request_save
    run_loop(s, 5, run_dir=d)
    assert s.calls == 5
    # save_run runs after the second solver call, before p is advanced to 2
    dens = sorted(os.listdir(os.path.join(d, "proc00")))
    assert dens == ["dens0000001.dat"] and not os.path.exists(os.path.join(d, "SAVE"))
    t, dims, _, _, field, x, _, _ = output.read_surface(os.path.join(d, "proc00", dens[0]))
    assert dims == (4, 4, 4) and field[0, 0, 0] == 2 and t == 0.2
    assert open(os.path.join(d, "p_saved.dat")).read() == "         1\n"


def test_output_cadence(tmp_path):
    """dt = 0.1, save_rate = 2 steps, save_rate3 = 0.3, save_rate2 = 0.5,
    p_save = 0.4, 6 steps from t = 0."""
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()
    io = OutputParams(save_rate=2, save_rate2=0.5, save_rate3=0.3, p_save=0.4)
    run_loop(s, 6, run_dir=d, outputs=io)
    # before the steps at t = 0, 0.2, 0.4 (modulo(t, 0.2) < 0.1, up to rounding)
    e = open(os.path.join(d, "energy.dat")).read().splitlines()
    ts = [float(line[:17]) for line in e]
    assert len(e) >= 3 and ts[:3] == [0.0, 0.2, 0.4]
    assert e[0] == output.e_line(0.0, 0.0, 1.0).rstrip("\n")
    psi_t = open(os.path.join(d, "psi_time.dat")).read().splitlines()
    assert len(psi_t) == len(e) and psi_t[0][34:51] == output.fortran_e(0.0)
    # condensed_particles at t >= 0, 0.3 (m = 0, 1) and 0.6 is past the last step
    m = open(os.path.join(d, "mass.dat")).read().splitlines()
    assert len(m) == 2 and len(m[0]) == 9 * 17
    assert sorted(os.listdir(os.path.join(d, "spectrum"))) == ["spectrum0000000.dat",
                                                                "spectrum0000003.dat"]
    # idl_surface at t >= 0 and 0.5; end_state at t >= 0 and 0.4
    dens = sorted(f for f in os.listdir(os.path.join(d, "proc00")) if f.startswith("dens"))
    assert dens == ["dens0000000.dat", "dens0000005.dat"]
    assert read_end_state(os.path.join(d, "proc00", "end_state.dat")).p == 4
    n = open(os.path.join(d, "norm.dat")).read().splitlines()
    assert len(n) >= 3 and all(len(line) == 4 * 17 for line in n)


def test_rk45_writes_timestep_every_save_rate_steps(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()
    s.prm.scheme = "rk45"
    run_loop(s, 7, run_dir=d, outputs=OutputParams(save_rate=3, save_rate2=1e9, save_rate3=1e9,
                                                    p_save=1e9))
    lines = open(os.path.join(d, "timestep.dat")).read().splitlines()
    # p = 0, 3, 6 when the step is taken (src/solve.f90:236)
    assert [int(line[51:]) for line in lines] == [0, 3, 6]
    assert all(len(line) == 3 * 17 + 10 for line in lines)
    assert lines[0][34:51] == output.fortran_e(0.1)


def test_line_length_and_zero_files(tmp_path):
    d = str(tmp_path)
    open(os.path.join(d, "RUNNING"), "w").close()
    s = FakeSolver()
    io = OutputParams(save_rate=2, save_rate2=0.25, save_rate3=1e9, p_save=1e9, save_3d=False,
                      save_ll=True, save_zeros=True)
    run_loop(s, 5, run_dir=d, outputs=io)
    ll = open(os.path.join(d, "linelength.dat")).read().splitlines()
    assert ll[0] == output.e_line(0.0, 0.0, 0.0).rstrip("\n")
    assert float(ll[1][34:51]) == 5.0  # before the third step: 2 calls so far
    zs = sorted(f for f in os.listdir(os.path.join(d, "proc00")) if f.startswith("zeros"))
    assert zs[0] == "zeros0000000.dat" and len(zs) >= 2
