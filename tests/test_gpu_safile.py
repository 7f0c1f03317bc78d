"""SA files in the reference's raw layout (mpi/io.hpp:80-98: entries back to
back, little endian; uint40 for 40-bit) streamed between the disk and device
memory, and checked on the GPU straight from the file (dcx_cli --sa-input)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import random_text
from distributed_suffix_sorting_evaluation_b200 import DCX_ERR_IO, DcxError

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "distributed_suffix_sorting_evaluation_b200", "lib", "dcx_cli")


def _raw(sa, width):
    sa = np.asarray(sa, np.uint64)
    if width == 32:
        return sa.astype(np.uint32).tobytes()
    if width == 64:
        return sa.tobytes()
    b = np.zeros((sa.size, 5), np.uint8)
    for i in range(5):
        b[:, i] = (sa >> np.uint64(8 * i)) & np.uint64(255)
    return b.tobytes()


@pytest.mark.parametrize("width", [32, 40, 64])
def test_write_and_read_stream(ctx, oracle, tmp_path, width):
    import torch
    t = random_text(3_000_001, 4, seed=21)
    n = t.size
    wb = width // 8
    d_text = torch.from_numpy(t).cuda()
    d_sa = torch.empty(n * wb, dtype=torch.uint8, device="cuda")
    ctx.build_sa_device(d_text.data_ptr(), n, d_sa.data_ptr(), dc=39, sa_width=width)
    torch.cuda.synchronize()
    path = str(tmp_path / f"t.sa{width}")
    ctx.write_sa_file(path, d_sa.data_ptr(), n, width, chunk_bytes=(1 << 20) + 7)  # chunks that do not divide it
    want = _raw(oracle.libsais(t), width)
    with open(path, "rb") as f:
        assert f.read() == want
    back = torch.zeros(n * wb, dtype=torch.uint8, device="cuda")
    ctx.read_sa_file(path, back.data_ptr(), n, width, chunk_bytes=(3 << 20) + 1)
    torch.cuda.synchronize()
    assert torch.equal(back, d_sa)


def test_check_sa_file(ctx, oracle, tmp_path):
    t = random_text(500_000, 4, seed=22)
    sa = oracle.libsais(t)
    good = tmp_path / "good.sa"
    good.write_bytes(_raw(sa, 40))  # what the reference cli's --output writes
    assert ctx.check_sa_file(t, str(good), 40)
    bad = sa.copy()
    bad[[10, 20]] = bad[[20, 10]]
    badf = tmp_path / "bad.sa"
    badf.write_bytes(_raw(bad, 40))
    assert not ctx.check_sa_file(t, str(badf), 40)
    short = tmp_path / "short.sa"
    short.write_bytes(_raw(sa[:-1], 40))
    with pytest.raises(DcxError):
        ctx.check_sa_file(t, str(short), 40)
    with pytest.raises(DcxError) as e:
        ctx.check_sa_file(t, str(tmp_path / "missing.sa"), 40)
    assert e.value.code == DCX_ERR_IO


def test_cli_checks_an_sa_file(oracle, tmp_path):
    t = random_text(200_000, 4, seed=23)
    tf = tmp_path / "text.bin"
    t.tofile(tf)
    sf = tmp_path / "text.sa"
    sf.write_bytes(_raw(oracle.libsais(t), 40))
    r = subprocess.run([CLI, "--input", str(tf), "--dcx", "dc39", "--sa-input", str(sf), "--check"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "SA_ok=1" in r.stdout
    bad = oracle.libsais(t)
    bad[[0, 1]] = bad[[1, 0]]
    sf.write_bytes(_raw(bad, 40))
    r = subprocess.run([CLI, "--input", str(tf), "--dcx", "dc39", "--sa-input", str(sf), "--check"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "SA_ok=0" in r.stdout
