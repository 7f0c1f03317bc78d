"""dcx_cli: the reference cli's flag surface (cli.cpp:149-305) over the C ABI."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import random_text

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "distributed_suffix_sorting_evaluation_b200", "lib", "dcx_cli")
README_FLAGS = ("--dcx dc39 --atomic-sorter ams --discarding-threshold 0.7 --ams-levels 2 --splitter-sampling random "
                "--splitter-sorting central --use-random-sampling-splitters --num-samples-splitters 20000 "
                "--buckets-sample-phase 16,16 --buckets-merging-phase 64,64,16 --use-binary-search-for-splitters "
                "--use-randomized-chunks --avg-chunks-pe 10000 --use-char-packing-samples "
                "--use-char-packing-merging --buckets-phase3 1 --samples-buckets-phase3 10000 "
                "--rearrange-buckets-balanced --use-compressed-buckets --pack-extra-words 0").split()


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        from distributed_suffix_sorting_evaluation_b200 import build
        build.build()
    return CLI


def run(cli, *args):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=600)


def test_readme_command_line_parses(cli):
    r = run(cli, "--input", "x", "--textsize", "1024", *README_FLAGS, "--json-output-path", "o", "--dry-run")
    assert r.returncode == 0, r.stderr
    cfg = json.loads(r.stdout)
    assert cfg["dcx"] == 39 and cfg["packing"] and cfg["sa_width"] == 40 and cfg["textsize"] == 1024
    assert "--atomic-sorter" in cfg["ignored"] and "--dcx" not in cfg["ignored"]


def test_unknown_flag_and_bad_values(cli):
    assert run(cli, "--no-such-flag").returncode == 1
    assert run(cli, "--dcx", "dc5", "--dry-run").returncode == 1
    assert run(cli, "--pack-extra-words", "1", "--dry-run").returncode == 1
    assert run(cli, "--sa-width", "48", "--dry-run").returncode == 1


def test_missing_file_exits_1(cli, tmp_path):
    r = run(cli, "--input", str(tmp_path / "nope.txt"), "--dcx", "dc3")
    assert r.returncode == 1 and "does not exist" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("width", [40, 64])
def test_cli_end_to_end(cli, oracle, tmp_path, width):
    t = random_text(300_000, 4, seed=5)
    f = tmp_path / "text.bin"
    t.tofile(f)
    out = tmp_path / "text.sa"
    args = ["--input", str(f), "--textsize", "250000", *README_FLAGS, "--check", "--output", str(out),
            "--json-output-path", str(tmp_path / "run")]
    if width == 64:
        args += ["--sa-width", "64"]
    r = run(cli, *args)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "SA_ok=1" in r.stdout
    raw = np.fromfile(out, np.uint8)
    from distributed_suffix_sorting_evaluation_b200 import unpack_sa
    sa = unpack_sa(raw, width, 250_000)
    assert np.array_equal(sa, oracle.libsais(t[:250_000]).astype(np.uint64))
    timer = json.load(open(str(tmp_path / "run") + "_timer.json"))
    assert "total_time" in timer[0]["data"]["root"]
    assert timer[0]["config"]["dcx"] == "dc39"
    json.load(open(str(tmp_path / "run") + "_counter.json"))


@pytest.mark.gpu
def test_cli_random_input(cli, tmp_path):
    r = run(cli, "--input", "random", "--textsize", "100000", "--alphabet_size", "8", "--seed", "3", "--dcx", "dc7",
            "--check")
    assert r.returncode == 0 and "SA_ok=1" in r.stdout


@pytest.mark.gpu
def test_checker_accepts_and_rejects(ctx, oracle):
    t = random_text(50_000, 4, seed=8)
    raw = ctx.build_sa_raw(t, dc=39, sa_width=40)
    assert ctx.check_sa(t, raw, 40)
    sa = oracle.libsais(t).astype(np.uint64)
    assert ctx.check_sa(t, sa, 64)
    bad = sa.copy()
    bad[[100, 101]] = bad[[101, 100]]  # a mistake planted on the CPU
    assert not ctx.check_sa(t, bad, 64)
    dup = sa.copy()
    dup[7] = dup[8]
    assert not ctx.check_sa(t, dup, 64)


def test_sa_input_flag(cli, tmp_path):
    f = tmp_path / "t.bin"
    f.write_bytes(b"ACGT" * 10)
    sa = str(tmp_path / "t.sa")
    r = run(cli, "--input", str(f), "--dcx", "dc3", "--sa-input", sa, "--check", "--dry-run")
    assert r.returncode == 0, r.stderr
    assert "--sa-input" not in json.loads(r.stdout)["ignored"]
    r = run(cli, "--input", str(f), "--dcx", "dc3", "--sa-input", sa, "--dry-run")
    assert r.returncode == 1 and "needs --check" in r.stderr
