"""XPIR's own TCP server and client over loopback, with the server answering on the GPU.

`pir_server` and `pir_client` are XPIR's apps (apps/server, apps/client, apps/optim)
compiled unchanged and linked with XPIR's pir library as built with the B200 engine
plugged in (xpir_b200/xpir/_build/): the server's PIRReplyGeneratorFactory("LWE") returns
PIRReplyGeneratorB200, so its sessions import the database into HBM and reply on the GPU,
and its optimizer service measures the GPU's costs.  The test follows XPIR's own
apps/tools/check-correctness.sh: a database directory of equal-size seeded files, the server
in server-driven mode (-z: the first client configures it and the imported database is kept
in HBM for the next clients), the client with forced crypto parameters, recursion level and
aggregation (-r ... --reclvl d --alpha a -c), run twice, and the retrieved file compared with
the database's first element (the directory's first entry, as DBDirectoryProcessor lists it).

The same loopback also runs without a GPU against XPIR's server built with the stock libpir
and factory (oracle/_ref/pir_server, the CPU reply generator): it checks the Boost
stand-ins of xpir_b200/xpir/compat and this harness on every CPU run.
"""
from __future__ import annotations

import os
import subprocess
import time
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
BUILD = ROOT / "xpir_b200" / "xpir" / "_build"
SERVER, CLIENT = BUILD / "pir_server", BUILD / "pir_client"
STOCK_SERVER = ROOT / "oracle" / "_ref" / "pir_server"
PORT = 1234  # XPIR's server listens on its default port (its -p value is never applied)


def listening(port: int) -> bool:
    """Whether a socket listens on the port (read from /proc, without connecting: a probe
    connection would be taken by the server as a session)."""
    want = f":{port:04X}"
    for table in ("/proc/net/tcp", "/proc/net/tcp6"):
        try:
            for line in open(table).readlines()[1:]:
                f = line.split()
                if f[1].endswith(want) and f[3] == "0A":
                    return True
        except OSError:
            pass
    return False


def loopback(server_exe: Path, tmp_path: Path, reclvl: int, alpha: int, params: str) -> None:
    for exe in (server_exe, CLIENT):
        if not exe.exists():
            pytest.skip(f"{exe.relative_to(ROOT)} is not built (built by __graft_entry__.build() from the XPIR sources)")
    for _ in range(60):  # a previous server's port must be free
        if not listening(PORT):
            break
        time.sleep(1)
    assert not listening(PORT), f"port {PORT} is in use"
    (tmp_path / "db").mkdir()
    (tmp_path / "exp").mkdir()
    (tmp_path / "reception").mkdir()
    rng = np.random.default_rng(100 * reclvl + alpha)
    for i in range(16):
        rng.integers(0, 256, size=12345, dtype=np.uint8).tofile(tmp_path / "db" / f"test{i + 1}")
    first = os.listdir(tmp_path / "db")[0]
    want = (tmp_path / "db" / first).read_bytes()

    server = subprocess.Popen([str(server_exe), "-z"], cwd=tmp_path, stdout=open(tmp_path / "server.out", "w"),
                              stderr=subprocess.STDOUT)
    try:
        for _ in range(300):
            if listening(PORT) or server.poll() is not None:
                break
            time.sleep(0.2)
        assert server.poll() is None and listening(PORT), (tmp_path / "server.out").read_text()[-2000:]
        for run in range(2):
            out = subprocess.run([str(CLIENT), "-r", params, "--reclvl", str(reclvl), "--alpha", str(alpha), "-c"],
                                 cwd=tmp_path, capture_output=True, text=True, timeout=600)
            log = out.stdout[-3000:] + out.stderr[-2000:] + (tmp_path / "server.out").read_text()[-3000:]
            assert out.returncode == 0, log
            got = (tmp_path / "reception" / "0").read_bytes()
            assert got == want, f"run {run}: retrieved file differs from {first}\n{log}"
            (tmp_path / "reception" / "0").unlink()
        text = (tmp_path / "server.out").read_text()
        assert "Already got an imported database available, using it" in text  # the kept database served run 2
    finally:
        server.terminate()
        try:
            server.wait(timeout=30)
        except subprocess.TimeoutExpired:
            server.kill()
            server.wait(timeout=30)


@pytest.mark.gpu
@pytest.mark.parametrize("reclvl,alpha,params", [(1, 1, "LWE:.*:4096:120"), (2, 1, "LWE:.*:4096:120"),
                                                 (1, 2, "LWE:.*:2048:60"), (3, 1, "LWE:.*:4096:180")])
def test_xpir_server_on_gpu_and_client_over_loopback(tmp_path, reclvl, alpha, params):
    loopback(SERVER, tmp_path, reclvl, alpha, params)


def test_stock_xpir_server_and_client_over_loopback(tmp_path):
    loopback(STOCK_SERVER, tmp_path, 2, 1, "LWE:.*:4096:120")
