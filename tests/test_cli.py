"""The drop-in command line (gem_b200/bin/gem, the reference's `GEM`
executable, in-core/src/main.cu:23-275 and out-of-core/src/main.cu:334-460):
argument errors on the CPU; on a B200 its printed counts against the
library's in exact, hash, relaxed, directory-batch and out-of-core runs."""
import os
import re
import subprocess

import pytest

import gem_b200 as gem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gem_b200", "bin", "gem")
RESULT = re.compile(r"Relaxed Query ET ([01]{32}): (\d+) matches")


def run_cli(*args, timeout=300):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=timeout)


def bits(mask):
    return format(mask, "032b")


def test_cli_is_built():
    assert os.access(CLI, os.X_OK)


@pytest.mark.parametrize("args", [[], ["-q"], ["-q", "x"], ["--bogus"], ["-q", "a", "-d", "b", "-t", "11"],
                                  ["-q", "a", "-d", "b", "--ooc-stream", "sometimes"]])
def test_cli_rejects_bad_arguments(args):
    p = run_cli(*args)
    assert p.returncode == 1 and "usage:" in p.stderr


def test_cli_reports_a_missing_query_path(tmp_path):
    p = run_cli("-q", tmp_path / "none.in", "-d", tmp_path / "none.graph")
    assert p.returncode == 1 and "Query path is not a file or directory" in p.stderr


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("cli")
    g = gem.HostGraph.rmat(11, 8, seed=91).set_labels(4, seed=92)
    gp = str(d / "data.graph")
    g.write_text(gp)
    qd = d / "queries"
    qd.mkdir()
    qs = gem.gen_queries(g, 4, gem.ANY, 4, seed=93)
    for i, q in enumerate(qs):
        q.write_text(str(qd / f"Q_{i}.in"))
    with gem.Context(time_cap_ms=30000) as c:
        c.load_graph(g)
        exact = [c.run(q, mode=gem.MODE_HASH) for q in qs]
        relaxed = c.relaxed(qs[0], 1)
    return gp, qs, qd, exact, relaxed


@pytest.mark.gpu
def test_cli_exact_counts_and_hash_equal_the_library(files):
    gp, qs, qd, exact, _ = files
    for i, q in enumerate(qs):
        p = run_cli("-q", qd / f"Q_{i}.in", "-d", gp, "-t", 0, "--mode", "hash")
        assert p.returncode == 0, p.stderr
        for line in ("Filter time:", "construct time:", "Join Time:", "=== Final Results ==="):
            assert line in p.stdout
        assert RESULT.findall(p.stdout) == [(bits((1 << q.ne) - 1), str(exact[i]["count"]))]
        assert f"Embedding hash: {exact[i]['emb_hash']:016x}" in p.stdout


@pytest.mark.gpu
def test_cli_relaxed_lines_equal_the_library(files):
    gp, qs, qd, _, relaxed = files
    p = run_cli("-q", qd / "Q_0.in", "-d", gp, "-t", 1)
    assert p.returncode == 0, p.stderr
    assert RESULT.findall(p.stdout) == [(bits(et), str(r["count"])) for et, r in relaxed]


@pytest.mark.gpu
def test_cli_directory_batch(files):
    gp, qs, qd, exact, _ = files
    p = run_cli("-q", qd, "-d", gp, "-t", 0)
    assert p.returncode == 0, p.stderr
    assert [int(c) for _, c in RESULT.findall(p.stdout)] == [r["count"] for r in exact]
    assert "=== Batch Summary ===" in p.stdout and f"success={len(qs)} failed=0" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("stream", ["always", "never", "auto"])
def test_cli_out_of_core_counts(files, stream):
    gp, qs, qd, exact, _ = files
    p = run_cli("-q", qd / "Q_1.in", "-d", gp, "-t", 0, "--ooc", "--ooc-part-kib", 4, "--ooc-stream", stream)
    assert p.returncode == 0, p.stderr
    assert [int(c) for _, c in RESULT.findall(p.stdout)] == [exact[1]["count"]]
