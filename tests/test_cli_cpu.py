"""Command-line handling that needs no device: usage errors are reported
before any CUDA call, with the reference's messages (CHostSetting.cu:14-44,
listenCommandLine.cpp)."""
from clast_b200 import api


def test_usage_errors():
    rc, err = api.run_clast(["-t", "x.fa", "-gap", "1", "-q", "y.fa", "-o", "z"])
    assert rc == 1 and "allowableGap" in err
    rc, err = api.run_clast(["-t", "x.fa", "-gap", "17", "-q", "y.fa", "-o", "z"])
    assert rc == 1 and "too large allowableGap" in err
    rc, err = api.run_clast(["-t", "x.fa", "-lMer", "32", "-q", "y.fa", "-o", "z"])
    assert rc == 1 and "lMerLength" in err
    rc, err = api.run_clast(["-q", "y.fa", "-o", "z"])
    assert rc == 1 and "target" in err
    rc, err = api.run_clast(["-t", "x.fa", "-o", "z"])
    assert rc == 1 and "query" in err
    rc, err = api.run_clast(["-t", "x.fa", "-q", "y.fa"])
    assert rc == 1 and "output" in err
    rc, err = api.run_clast(["bogus"])
    assert rc == 1 and "Odd parameter" in err
    rc, err = api.run_clast(["-t", "a", "-t"])
    assert rc == 1 and "\"-t\"" in err
    rc, err = api.run_clast(["-stride", "x5", "-t", "a", "-q", "b", "-o", "c"])
    assert rc == 1


def test_missing_file(tmp_path):
    rc, err = api.run_clast(["-t", str(tmp_path / "none.fa"), "-q", str(tmp_path / "none.fa"),
                             "-o", str(tmp_path / "o.tsv")])
    assert rc == 3 and "open failed" in err
