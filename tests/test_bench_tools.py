"""The bench's own tooling, on CPU: the launch-list summariser that turns an
ncu --csv log into the tables under profiles/, and the percentile helper of
the latency figures."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

HEADER = ('"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream",'
          '"Block Size","Grid Size","Device","CC","Section Name","Metric Name","Metric Unit",'
          '"Metric Value"')


def row(launch, kernel, metric, unit, value):
    return (f'"{launch}","1","python3","127.0.0.1","{kernel}","1","13","(256, 1, 1)",'
            f'"(148, 1, 1)","0","10.0","Command line profiler metrics","{metric}","{unit}","{value}"')


def test_launch_list_summary(tmp_path, capsys):
    log = tmp_path / "launches.csv"
    lines = ["==PROF== Connected to process 1 (python3)", HEADER,
             row(0, "void k_route_scan<6, 0>(state)", "gpu__time_duration.sum", "usecond", "200"),
             row(0, "void k_route_scan<6, 0>(state)", "dram__bytes_read.sum", "Mbyte", "80"),
             row(1, "k_sweep(state)", "gpu__time_duration.sum", "ns", "50000"),
             row(1, "k_sweep(state)", "dram__bytes_read.sum", "Kbyte", "4"),
             row(2, "void k_route_scan<6, 0>(state)", "gpu__time_duration.sum", "usecond", "250"),
             row(2, "void k_route_scan<6, 0>(state)", "dram__bytes_read.sum", "Mbyte", "90"),
             "==PROF== Disconnected from process 1"]
    log.write_text("\n".join(lines) + "\n")
    bench.ncu_summary(str(log))
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "total 0.500 ms over 3 launches"
    scan = next(x for x in out if x.startswith("void k_route_scan<6, 0>")).split()
    # name (3 words), launches, total ms, share, mean us, DRAM bytes per launch
    assert scan[3:7] == ["2", "0.450", "90.00%", "225.0"]
    assert scan[7] == "85,000,000"
    sweep = next(x for x in out if x.startswith("k_sweep")).split()
    assert sweep[1:5] == ["1", "0.050", "10.00%", "50.0"]
    # the table is sorted by total time
    assert out.index(next(x for x in out if x.startswith("void k_route_scan"))) < \
        out.index(next(x for x in out if x.startswith("k_sweep")))


def test_percentile_picks_the_order_statistic():
    xs = list(range(1, 101))
    assert bench.percentile(xs, 0.5) == pytest.approx(50.5, abs=0.6)
    assert bench.percentile(xs, 0.99) == pytest.approx(99, abs=1.1)
    assert bench.percentile([7.0], 0.99) == 7.0
