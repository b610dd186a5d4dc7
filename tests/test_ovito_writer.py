"""The drivers' asynchronous output: the OVITO writer (fmdh::OvitoWriter:
frames copied, formatted in parallel chunks on a writer thread, appended in
order) writes exactly the bytes of the synchronous formatter, for atomistic
and rigid frames, with one and with several formatting threads; restart
saves run as jobs on a writer thread (fmdh::RestartWriter) and write exactly
the synchronous writers' files for all three programs."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "fuller_md_en_b200" / "_lib"
HOST = ROOT / "fuller_md_en_b200" / "host"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if not (LIB / "libfullermd_host.so").exists():
        pytest.fail("libfullermd_host.so is not built (python -m fuller_md_en_b200.build)")
    exe = tmp_path_factory.mktemp("ovito") / "ovito_writer_check"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", str(HOST), "-I", str(ROOT / "include"),
                        "-o", str(exe), str(ROOT / "tests" / "cpp" / "ovito_writer_check.cpp"), f"-L{LIB}",
                        "-lfullermd_host", f"-Wl,-rpath,{LIB}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("threads", [1, 7])
def test_async_writer_matches_sync_formatter(checker, tmp_path, threads):
    a, b = tmp_path / "sync.xyz", tmp_path / "async.xyz"
    r = subprocess.run([str(checker), str(a), str(b), str(threads)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    da, db = a.read_bytes(), b.read_bytes()
    assert len(da) > 10_000_000 and da == db
    assert da.count(b"Lattice=") == 11


def test_restart_writer_matches_sync_writer(tmp_path):
    exe = tmp_path / "restart_writer_check"
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", str(HOST), "-I", str(ROOT / "include"),
                        "-o", str(exe), str(ROOT / "tests" / "cpp" / "restart_writer_check.cpp"), f"-L{LIB}",
                        "-lfullermd_host", f"-Wl,-rpath,{LIB}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    a, b = tmp_path / "sync", tmp_path / "async"
    a.mkdir()
    b.mkdir()
    r = subprocess.run([str(exe), str(a), str(b)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    names = sorted(p.name for p in a.iterdir())
    assert len(names) == 12 and names == sorted(p.name for p in b.iterdir())
    for nm in names:
        assert (a / nm).read_bytes() == (b / nm).read_bytes(), nm
    assert (a / "c40_ai.rst").read_bytes() != (a / "c30_ai.rst").read_bytes()
