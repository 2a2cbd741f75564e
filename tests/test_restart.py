"""end_state.dat checkpoint format (src/io.f90:840-862) and the restart
rules of state_restart (src/ic.f90:117-186): byte layout, round trip,
and clean errors for missing, truncated and mismatched files (host-side
fault injection; no GPU)."""
import os

import numpy as np
import pytest

from gpe_b200.restart import (EndState, RestartError, file_size, read_end_state,
                              restart_time_state, write_end_state)


def test_byte_layout_is_the_reference_stream_format(tmp_path):
    psi = (np.arange(2 * 3 * 4) + 1j * np.arange(24)[::-1]).reshape(2, 3, 4)
    f = str(tmp_path / "end_state.dat")
    write_end_state(f, psi, p=17, t=1.5, im_t=0.25, dt=complex(0.01, -0.02), pr_bytes=8)
    raw = open(f, "rb").read()
    assert len(raw) == file_size(4, 3, 2, 8) == 16 + 16 + 16 + 24 * 16
    assert list(np.frombuffer(raw[:16], "<i4")) == [4, 3, 2, 17]
    assert list(np.frombuffer(raw[16:32], "<f8")) == [1.5, 0.25]
    assert complex(np.frombuffer(raw[32:48], "<c16")[0]) == complex(0.01, -0.02)
    # x fastest: the second value is psi(x=1, y=0, z=0)
    assert complex(np.frombuffer(raw[64:80], "<c16")[0]) == psi[0, 0, 1]


@pytest.mark.parametrize("pr", [8, 4])
def test_round_trip(tmp_path, pr):
    rng = np.random.default_rng(pr)
    psi = rng.standard_normal((5, 6, 7)) + 1j * rng.standard_normal((5, 6, 7))
    f = str(tmp_path / "s.dat")
    write_end_state(f, psi, 3, 2.0, 0.0, complex(0.005, 0.0), pr)
    st = read_end_state(f, pr, expect=(7, 6, 5))
    assert (st.nx, st.ny, st.nz, st.p, st.t, st.im_t) == (7, 6, 5, 3, 2.0, 0.0)
    tol = 0 if pr == 8 else 1e-6
    np.testing.assert_allclose(st.psi, psi, rtol=tol, atol=tol)


def test_missing_truncated_and_mismatched_files_fail_cleanly(tmp_path):
    f = str(tmp_path / "s.dat")
    with pytest.raises(RestartError, match="does not exist"):
        read_end_state(f)
    write_end_state(f, np.ones((4, 4, 4), complex), 0, 0.0, 0.0, 0.01)
    with pytest.raises(RestartError, match="differs"):
        read_end_state(f, expect=(8, 4, 4))
    with pytest.raises(RestartError, match="expected"):
        read_end_state(f, pr_bytes=4)  # written with 8-byte reals
    raw = open(f, "rb").read()
    open(f, "wb").write(raw[:-10])
    with pytest.raises(RestartError, match="expected"):
        read_end_state(f)
    open(f, "wb").write(raw[:9])
    with pytest.raises(RestartError, match="truncated"):
        read_end_state(f)


def test_restart_time_rules():
    psi = np.ones((1, 1, 1), complex)
    # imaginary-time save, real-time run: dt rotated, im_t reset
    st = EndState(1, 1, 1, 10, 0.0, 0.5, complex(0.0, -0.01), psi)
    assert restart_time_state(st, True, "rk4", complex(0.01, 0)) == (10, 0.0, 0.0, complex(0.01, 0))
    # real-time save, imaginary-time run: t reset
    st = EndState(1, 1, 1, 10, 2.0, 0.0, complex(0.01, 0.0), psi)
    p, t, im_t, dt = restart_time_state(st, False, "rk4", complex(0.0, -0.01))
    assert (p, t, im_t, dt) == (10, 0.0, 0.0, complex(0.0, -0.01))
    # rk45 keeps the saved step
    st = EndState(1, 1, 1, 4, 1.0, 0.0, complex(0.0123, 0.0), psi)
    assert restart_time_state(st, True, "rk45", complex(0.005, 0))[3] == complex(0.0123, 0)
    # other schemes rescale p when dt changed
    st = EndState(1, 1, 1, 100, 1.0, 0.0, complex(0.01, 0.0), psi)
    assert restart_time_state(st, True, "rk4", complex(0.005, 0))[0] == 200
