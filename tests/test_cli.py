"""The command-line drop-in (partitioned_join_b200/bin/partitioned_join):
the reference binary's options (main.cu:100-188) and CSV columns
(scripts/bench_partitioned_join.sh:13)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle
from partitioned_join_b200 import build as pj_build

CLI = pj_build.CLI
CSV_HEADER = ("build size,probe size,key byte,tuple byte,selectivity,unique build key,num part P1,num part P2,"
              "max part size factor,skewed mode,zipf factor,joined size,combined histo [ms],part P1 [ms],"
              "part P2 [ms],handle skew [ms],join [ms],total [ms],num errors")


def run_cli(*args, timeout=300):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=timeout)


def test_cli_built_and_lists_reference_options():
    assert os.path.exists(CLI)
    r = run_cli("-h")
    assert r.returncode == 1  # as main.cu:180-188
    for flag in "b p s r u F B P v f R n N S V C Z z H".split():
        assert f"  -{flag}, --" in r.stdout, flag


def test_cli_rejects_partition_counts_like_the_reference():
    r = run_cli("-b", 1000, "-p", 1000, "-n", 100)
    assert r.returncode == 1 and "power of two" in r.stderr
    r = run_cli("-b", 1000, "-p", 1000, "-R", "-n", 64)
    assert r.returncode == 1 and "power of two" in r.stderr


def _csv_fields(stdout):
    lines = [l for l in stdout.strip().splitlines() if l.count(",") >= 18]
    assert len(lines) == 1, stdout
    f = lines[0].split(",")
    assert len(f) == len(CSV_HEADER.split(","))
    return f


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [[], ["-V"], ["-K", 8], ["-H"]])
def test_cli_csv_run_is_error_free(extra):
    # the reference bench script's form: -b B -p P -r 2B -R -n 256 -N 256 -u -C
    b = 1 << 21
    r = run_cli("-b", b, "-p", 2 * b, "-r", 2 * b, "-R", "-n", 256, "-N", 256, "-u", "-C", "-s", 0.5, *extra)
    assert r.returncode == 0, r.stderr
    f = _csv_fields(r.stdout)
    assert int(f[0]) == b and int(f[1]) == 2 * b and int(f[2]) == (8 if "-K" in extra else 4)
    joined = int(f[11])
    assert abs(joined / (2 * b) - 0.5) < 0.01
    assert int(f[18]) == 0
    assert float(f[17]) > 0


@pytest.mark.gpu
def test_cli_report_and_repeated_keys():
    r = run_cli("-b", 300000, "-p", 600000, "-r", 100000, "-n", 64, "-s", 0.8)
    assert r.returncode == 0, r.stderr
    assert "[*] Results:" in r.stdout and "number of errors     = 0" in r.stdout


@pytest.mark.gpu
def test_cli_reads_key_files(tmp_path):
    rng = np.random.default_rng(31)
    b = rng.permutation(200000).astype(np.int32)
    p = rng.integers(0, 300000, size=500000).astype(np.int32)
    bf, pf = tmp_path / "build.bin", tmp_path / "probe.bin"
    b.tofile(bf)
    p.tofile(pf)
    r = run_cli("-F", "-B", bf, "-P", pf, "-b", b.shape[0], "-p", p.shape[0], "-u", "-n", 128, "-C")
    assert r.returncode == 0, r.stderr
    f = _csv_fields(r.stdout)
    assert int(f[11]) == oracle.inner_join(b, p, True)[0].shape[0]
    assert int(f[18]) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("flags,parts,two", [(["-n", 64], "64 partitions (raw key bits), ", False),
                                             (["-n", 1024], "1024 partitions (raw key bits), ", False),
                                             (["-R", "-n", 256, "-N", 512], "256 partitions (raw key bits) x 512", True),
                                             (["-R", "-n", 32, "-N", 16, "-f", 1.5], "32 partitions (raw key bits) x 16",
                                              True)])
def test_cli_plans_from_the_reference_partition_flags(flags, parts, two):
    b = 1 << 22
    args = ["-b", b, "-p", b, "-r", 2 * b, "-u", "-s", 0.9, *flags]
    r = run_cli(*args)
    assert r.returncode == 0, r.stderr
    assert f"B200 plan            = {parts}" in r.stdout
    assert "number of errors     = 0" in r.stdout
    assert ("partition P2 time" in r.stdout) == two
    f = _csv_fields(run_cli(*args, "-C").stdout)
    assert int(f[18]) == 0 and abs(int(f[11]) / b - 0.9) < 0.01
    assert (float(f[14]) > 0) == two  # part P2 [ms]: the second pass's own time
    assert float(f[13]) > 0
