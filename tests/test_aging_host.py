"""Host logic of the one-process aging workflow: the log schedule against the
oracle's restatement of main.cu:14-53, waiting-time steps, stdin protocol."""
import io

import pytest

from bd_aging_b200 import aging as A
from oracle import oracle as O


@pytest.mark.parametrize("md,rt,dt", [(1e-3, 10.0, 1e-4), (1e-3, 1.0, 1e-5), (1e-2, 100.0, 1e-3),
                                      (1e-4, 1.0, 1e-5), (1e-3, 10.0, 3e-5), (1e-3, 1e-1, 1e-4)])
def test_sampling_indexes_match_oracle(md, rt, dt):
    assert A.sampling_indexes(md, rt, dt) == list(O.sampling_indexes(md, rt, dt))


def test_waiting_time_steps_follow_decade_writes():
    idx = A.sampling_indexes(1e-3, 10.0, 1e-4)
    # decade k's configuration is written at sample 1 + 10 (k - 1) (main.cu:809-835)
    assert A.waiting_time_steps(idx, 3) == [0, idx[1] + 1, idx[11] + 1, idx[21] + 1]
    with pytest.raises(ValueError):
        A.waiting_time_steps(idx, 5)


def test_protocol_parser_reads_run_fself_data():
    data = ("linear\n1.0  0.25  0.0  0.0  1\n1.0e-4\nlog\n0.1  1.0e-3  1.0e1\n1  3  0\n8  8\n5\n"
            "400  15.0\n6.19\n12345\n")
    p = A._read_protocol(io.StringIO(data))
    assert p["protocol"] == "linear" and p["T0"] == 1.0 and p["Tf"] == 0.25 and p["dt"] == 1e-4
    assert (p["trans_time"], p["minimal_decade"], p["run_time"]) == (0.1, 1e-3, 10.0)
    assert (p["print_decades"], p["number_of_tws"], p["current_decade"]) == (1, 3, 0)
    assert p["n_configs"] == 5 and p["nbins_gder"] == 400 and p["range_gder"] == 15.0
    assert p["qmax"] == 6.19 and p["idum"] == 12345


def test_protocol_parser_rejects_linear_sampling():
    data = "linear\n1 1 0 0 1\n1e-4\nlinear\n0.1 1.0 10\n8 8\n1\n10 2.0\n6.19\n1\n"
    with pytest.raises(SystemExit):
        A._read_protocol(io.StringIO(data))
