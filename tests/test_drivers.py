"""The drop-in programs (fuller_*_gpu) against the reference programs.

The reference programs are built from their own sources into
oracle/_ref/bin (serial and OpenMP builds, exactly as the reference's build
script compiles them) and run here on the CPU as the checker.  Both sides
read the same fullerene library, written by ``write_library`` from this
package's own C60 geometry in the .cc1 layout of
FullereneLib/C60-76/C60-Ih.cc1 (count line, then "C idx x y z flag nbrs...").

Whole runs are compared with the SERIAL reference build: the OpenMP AIREBO
build accumulates REBO forces with `omp atomic` under dynamic scheduling
(AI:284-417), so its trajectories differ from run to run (at cell=1 the
printed E_REBO moves in the 4th decimal by step 10), while the serial build
is deterministic.

CPU tests: help text, banners, topology lines and the restart reader (our
driver reads a restart file the reference wrote).  GPU tests: monitor and
average lines of whole runs, OVITO frames, restart files read back by the
reference, abort.md / stop.md control.
"""
from __future__ import annotations

import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fuller_md_en_b200 import crystal

ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "fuller_md_en_b200" / "_bin"
REFBIN = ROOT / "oracle" / "_ref" / "bin"

OURS = {"lj": "fuller_LJ_npt_md_gpu", "ai": "fuller_airebo_npt_md_gpu", "mm": "fuller_LJ_npt_mmmd_gpu",
        "core": "fuller_LJ_core_gpu"}
REF = {"lj": "fuller_LJ_npt_md", "ai": "fuller_airebo_npt_md", "mm": "fuller_LJ_npt_mmmd", "core": "fuller_LJ_core"}


def ours(prog: str) -> Path:
    p = BIN / OURS[prog]
    if not p.exists():
        pytest.fail(f"{p} is not built (python -m fuller_md_en_b200.build)")
    return p


def ref(prog: str, omp: bool = False) -> Path:
    p = REFBIN / f"{REF[prog]}_{'omp' if omp else 'serial'}"
    if not p.exists():
        pytest.skip(f"reference program {p.name} not built (make -C oracle ref)")
    return p


def write_library(root: Path) -> Path:
    """FullereneLib-shaped directory holding C60-Ih.cc1 from crystal.c60_ih()."""
    coords = crystal.c60_ih()
    bonds = crystal.bonds_from_geometry(coords)
    nbr = [[] for _ in range(len(coords))]
    for i, j in bonds:
        nbr[i].append(j + 1)
        nbr[j].append(i + 1)
    d = root / "FullereneLib" / "C60-76"
    d.mkdir(parents=True, exist_ok=True)
    lines = [f" {len(coords)}"]
    for i, (x, y, z) in enumerate(coords):
        lines.append(f"  C {i + 1:4d} {x:11.6f} {y:11.6f} {z:11.6f}    2" + "".join(f" {b:3d}" for b in nbr[i]))
    (d / "C60-Ih.cc1").write_text("\n".join(lines) + "\n")
    return root / "FullereneLib"


REF_MOLECULES = Path(__file__).resolve().parent / "golden" / "fullerenes.npz"


def cc1_text(xyz, flag, nbr) -> str:
    """A molecule in the .cc1 layout of the reference's FullereneLib, byte
    for byte as the library writes it (count line; "C", index, x y z with six
    decimals, flag, 1-based neighbours)."""
    lines = [f" {len(xyz)}"]
    for i, (p, f, b) in enumerate(zip(xyz, flag, nbr)):
        lines.append(f"  C{i + 1:5d}{p[0]:12.6f}{p[1]:12.6f}{p[2]:12.6f}{f:5d}" + "".join(f"{v:4d}" for v in b if v >= 0))
    return "\n".join(lines) + "\n"


def write_reference_library(root: Path) -> Path:
    """FullereneLib holding the reference library's own molecules recorded in
    tests/golden/fullerenes.npz (C60-Ih, C70-D5h, C72-D6d, C84 No.01-D2 and
    No.24-D6h; tests/golden/gen_fullerenes.py)."""
    z = np.load(REF_MOLECULES)
    for key in sorted({k.split("/")[0] for k in z.files}):
        d = root / "FullereneLib" / str(z[f"{key}/dir"])
        d.mkdir(parents=True, exist_ok=True)
        (d / f"{key}.cc1").write_text(cc1_text(z[f"{key}/xyz"], z[f"{key}/flag"], z[f"{key}/nbr"]))
    return root / "FullereneLib"


def run(exe: Path, args: list[str], cwd: Path, timeout: int = 600, env: dict | None = None):
    e = dict(os.environ)
    e.setdefault("OMP_NUM_THREADS", str(min(16, os.cpu_count() or 1)))
    if env:
        e.update(env)
    return subprocess.run([str(exe), *args], cwd=cwd, capture_output=True, text=True, timeout=timeout, env=e)


@pytest.fixture()
def work(tmp_path):
    lib = write_library(tmp_path)
    a = tmp_path / "ours"
    b = tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    return {"lib": str(lib), "ours": a, "ref": b}


_MODE = re.compile(r"GPU|OpenMP|OpenACC|Serial|CUDA|threads|Active device|GPU devices")


def banner(text: str) -> list[str]:
    """Lines up to the blank line after the banner's closing rule, without
    the lines that name the build mode or device."""
    out = []
    for ln in text.splitlines():
        if ln.strip() == "" and out and out[-1].startswith("===="):
            break
        if not _MODE.search(ln):
            out.append(ln)
    return out


# ---------------------------------------------------------------- CPU tests
@pytest.mark.parametrize("prog", ["lj", "ai", "mm"])
def test_help_matches_reference(prog, work):
    a = run(ours(prog), ["--help"], work["ours"])
    b = run(ref(prog), ["--help"], work["ref"])
    assert a.returncode == 0 and b.returncode == 0
    assert a.stdout == b.stdout


@pytest.mark.parametrize("prog,args", [
    ("lj", ["--cell=2", "--crystal=hcp", "--temp=350"]),
    ("ai", ["--cell=1", "--pres=0.5", "--dt=0.25"]),
    ("mm", ["--cell=1", "--crystal=bcc", "--ff_kb=500"]),
])
def test_banner_matches_reference(prog, args, work):
    args = args + ["--step=4", "--mon=2", f"--libdir={work['lib']}"]
    a = run(ours(prog), args, work["ours"])
    b = run(ref(prog), args, work["ref"])
    assert b.returncode == 0, b.stderr
    ba, bb = banner(a.stdout), banner(b.stdout)
    assert len(bb) > 5
    assert ba == bb


def test_core_banner(work):
    # The reference core program always runs its 1000 steps, so its banner is
    # compared in the GPU run test; here the lines the program fixes.
    a = run(ours("core"), ["--cell=2"], work["ours"])
    lines = banner(a.stdout)
    assert "  FCC cell        : 2x2x2  N=32 molecules" in lines
    assert "  a0=14.17 A  T=300 K  P=0.0 GPa  dt=1.0 fs  steps=1000" in lines
    assert "  MAX_NEIGH=80  VECTOR_LENGTH=128" in lines


@pytest.mark.parametrize("prog", ["lj", "ai", "mm"])
def test_unknown_fullerene_and_missing_library(prog, work):
    a = run(ours(prog), ["--fullerene=C99", f"--libdir={work['lib']}"], work["ours"])
    b = run(ref(prog), ["--fullerene=C99", f"--libdir={work['lib']}"], work["ref"])
    assert a.returncode == b.returncode != 0
    assert a.stderr.strip() == b.stderr.strip()
    a = run(ours(prog), ["--fullerene=C70", f"--libdir={work['lib']}"], work["ours"])
    b = run(ref(prog), ["--fullerene=C70", f"--libdir={work['lib']}"], work["ref"])
    assert a.returncode == b.returncode != 0
    assert a.stderr.strip() == b.stderr.strip()


def test_core_rejects_bad_cell(work):
    a = run(ours("core"), ["9"], work["ours"])
    b = run(ref("core"), ["9"], work["ref"])
    assert a.returncode == b.returncode == 1
    assert a.stdout == b.stdout


@pytest.mark.parametrize("prog,tag,unit", [("lj", "restart_LJ_serial", "mols"),
                                           ("ai", "restart_airebo_serial", "atoms"),
                                           ("mm", "restart_mmmd_serial", "atoms")])
def test_restart_reader_reads_reference_file(prog, tag, unit, work):
    base = ["--cell=1", "--step=4", "--mon=2", f"--libdir={work['lib']}"]
    b = run(ref(prog), base + ["--restart=2"], work["ref"])
    assert b.returncode == 0, b.stderr
    files = sorted(work["ref"].glob("restart_*.rst"))
    assert files, b.stdout
    rst = files[0]
    a = run(ours(prog), base + [f"--resfile={rst}"], work["ours"])
    c = run(ref(prog), base + [f"--resfile={rst}"], work["ref"])
    la = [ln for ln in a.stdout.splitlines() if "Restart" in ln]
    lc = [ln for ln in c.stdout.splitlines() if "Restart" in ln]
    assert len(lc) == 2 and lc[0].endswith(f"{unit})")
    assert la == lc


def test_recorded_molecules_are_the_reference_library():
    """The recorded molecules, written back by cc1_text, are the reference
    library's files byte for byte (checked where the reference checkout is
    present: REF, or "reference" beside this repository)."""
    root = Path(os.environ.get("REF", ROOT.parent / "reference")) / "FullereneLib"
    if not root.exists():
        pytest.skip("reference checkout not present")
    z = np.load(REF_MOLECULES)
    keys = sorted({k.split("/")[0] for k in z.files})
    assert len(keys) == 5
    for key in keys:
        want = (root / str(z[f"{key}/dir"]) / f"{key}.cc1").read_text()
        assert cc1_text(z[f"{key}/xyz"], z[f"{key}/flag"], z[f"{key}/nbr"]) == want, key


# ---------------------------------------------------------------- GPU tests
_NUM = re.compile(r"^-?\d+(\.\d*)?([eE][-+]?\d+)?$")


def monitor_rows(text: str) -> list[list[str]]:
    rows = []
    for ln in text.splitlines():
        tok = ln.split()
        if len(tok) >= 5 and tok[0].isdigit() and all(_NUM.match(t) or t in ("COLD", "WARM", "PROD") for t in tok):
            rows.append(tok)
    return rows


def averages(text: str) -> dict[str, float]:
    for ln in text.splitlines():
        if "Averages (" in ln or ln.startswith("Avg("):
            out = {"n": float(re.search(r"\((\d+)", ln).group(1))}
            for k, v in re.findall(r"(\w+)=(-?[\d.]+)", ln):
                out[k] = float(v)
            return out
    return {}


def close_tok(x: str, y: str, rel: float) -> bool:
    if not _NUM.match(x):
        return x == y
    dec = len(x.split(".")[1]) if "." in x else 0
    a, b = float(x), float(y)
    return abs(a - b) <= 1.01 * 10.0 ** (-dec) + rel * abs(b)


def assert_rows_match(ra, rb, skip_last_col=True, rel=1e-6):
    assert len(ra) == len(rb) and ra, (ra, rb)
    for x, y in zip(ra, rb):
        n = len(y) - (1 if skip_last_col else 0)    # last column: wall time
        assert len(x) == len(y)
        for i in range(n):
            assert close_tok(x[i], y[i], rel), (x, y, i)


def assert_avg_match(a, b, rel=1e-6):
    assert a and a.keys() == b.keys(), (a, b)
    for k in b:
        assert abs(a[k] - b[k]) <= 1.01e-4 + rel * abs(b[k]) if k != "n" else a[k] == b[k], (k, a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("prog,args", [
    ("ai", ["--cell=1", "--step=20", "--mon=5"]),
    ("ai", ["--cell=1", "--coldstart=6", "--warmup=6", "--step=8", "--mon=3", "--warmup_mon=freq"]),
    ("mm", ["--cell=1", "--step=40", "--mon=10"]),
    ("mm", ["--cell=1", "--crystal=hcp", "--coldstart=10", "--warmup=10", "--step=20", "--mon=5"]),
    ("lj", ["--cell=2", "--step=100", "--mon=20"]),
    ("lj", ["--cell=2", "--crystal=bcc", "--coldstart=20", "--warmup=20", "--step=60", "--mon=10"]),
])
def test_driver_run_matches_reference(prog, args, work):
    args = args + [f"--libdir={work['lib']}"]
    a = run(ours(prog), args, work["ours"])
    assert a.returncode == 0, a.stdout + a.stderr
    b = run(ref(prog), args, work["ref"])
    assert b.returncode == 0, b.stderr
    assert_rows_match(monitor_rows(a.stdout), monitor_rows(b.stdout))
    assert_avg_match(averages(a.stdout), averages(b.stdout))
    assert "Done (" in a.stdout


@pytest.mark.gpu
def test_core_driver_matches_reference(work):
    a = run(ours("core"), ["2"], work["ours"])
    assert a.returncode == 0, a.stdout + a.stderr
    b = run(ref("core"), ["2"], work["ref"], timeout=1200)
    assert b.returncode == 0, b.stderr
    assert_rows_match(monitor_rows(a.stdout), monitor_rows(b.stdout))
    assert_avg_match(averages(a.stdout), averages(b.stdout))
    assert re.search(r"^Done \d+\.\ds$", a.stdout, re.M)


def read_xyz(path: Path):
    frames = []
    lines = path.read_text().splitlines()
    i = 0
    while i < len(lines):
        n = int(lines[i])
        head = lines[i + 1]
        body = np.array([[float(v) for v in ln.split()[1:]] for ln in lines[i + 2:i + 2 + n]])
        frames.append((head, body))
        i += 2 + n
    return frames


@pytest.mark.gpu
@pytest.mark.parametrize("prog,ovito", [("ai", "ovito_traj_airebo"), ("mm", "ovito_traj_mmmd"),
                                        ("lj", "ovito_traj_LJ")])
def test_ovito_frames_match_reference(prog, ovito, work):
    args = ["--cell=1", "--step=10", "--mon=5", "--ovito=5", f"--libdir={work['lib']}"]
    a = run(ours(prog), args, work["ours"])
    assert a.returncode == 0, a.stdout + a.stderr
    b = run(ref(prog), args, work["ref"])
    assert b.returncode == 0, b.stderr
    fa = read_xyz(next(work["ours"].glob(f"{ovito}*.xyz")))
    fb = read_xyz(next(work["ref"].glob(f"{ovito}*.xyz")))
    assert len(fa) == len(fb) == 2
    num = re.compile(r"-?\d+\.\d+")
    for (ha, xa), (hb, xb) in zip(fa, fb):
        assert num.sub("#", ha) == num.sub("#", hb)
        np.testing.assert_allclose([float(v) for v in num.findall(ha)], [float(v) for v in num.findall(hb)],
                                   rtol=1e-7, atol=2e-8)
        assert xa.shape == xb.shape
        np.testing.assert_array_equal(xa[:, 3], xb[:, 3])          # molecule index column
        np.testing.assert_allclose(xa, xb, rtol=1e-6, atol=1e-7)


def parse_restart(path: Path) -> dict[str, list[str]]:
    out: dict[str, list[str]] = {}
    for ln in path.read_text().splitlines():
        tok = ln.split()
        if not tok or tok[0].startswith("#"):
            continue
        out.setdefault(tok[0], []).append(" ".join(tok[1:]))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prog,tag", [("ai", "restart_airebo"), ("mm", "restart_mmmd"), ("lj", "restart_LJ")])
def test_restart_written_by_driver_resumes_in_both(prog, tag, work):
    base = ["--cell=1", "--step=20", "--mon=5", f"--libdir={work['lib']}"]
    full = run(ours(prog), base, work["ours"])
    assert full.returncode == 0, full.stdout + full.stderr
    a = run(ours(prog), base + ["--restart=10"], work["ours"])
    assert a.returncode == 0, a.stdout + a.stderr
    # restart_filename: "_<step>" zero-padded to the digits of the total
    # step count, no suffix at the last step (LJ:583-588)
    got = sorted(p.name for p in work["ours"].glob(f"{tag}_gpu*.rst"))
    assert len(got) == 2 and got[1].endswith("_10.rst") and got[0] == got[1][:-7] + ".rst", got
    mid = work["ours"] / got[1]
    # same records and field counts as a restart file of the reference
    b = run(ref(prog), base + ["--restart=10"], work["ref"])
    assert b.returncode == 0, b.stderr
    refmid = sorted(work["ref"].glob(f"{tag}_serial*_10.rst"))
    assert len(refmid) == 1
    assert refmid[0].name.replace("_serial", "_gpu") == mid.name
    ra, rb = parse_restart(mid), parse_restart(refmid[0])
    assert ra.keys() == rb.keys()
    for k in rb:
        assert len(ra[k]) == len(rb[k]), k
        assert [len(x.split()) for x in ra[k]] == [len(x.split()) for x in rb[k]], k
    # resume: ours and the reference from OUR file agree with the uninterrupted run
    ra = run(ours(prog), base + [f"--resfile={mid}"], work["ours"])
    rr = run(ref(prog), base + [f"--resfile={mid}"], work["ref"])
    assert ra.returncode == 0 and rr.returncode == 0
    tail = [r for r in monitor_rows(full.stdout) if int(r[0]) > 10]
    assert_rows_match(monitor_rows(ra.stdout), tail)
    assert_rows_match(monitor_rows(rr.stdout), tail)


@pytest.mark.gpu
@pytest.mark.parametrize("prog", ["ai", "mm", "lj"])
def test_abort_and_stop_control(prog, work):
    base = ["--cell=1", "--step=30", "--mon=5", "--restart=10", f"--libdir={work['lib']}"]
    for d in (work["ours"], work["ref"]):
        (d / "abort.md").mkdir()
    a = run(ours(prog), base, work["ours"])
    b = run(ref(prog), base, work["ref"])
    assert a.returncode == 0 and b.returncode == 0
    msg = [ln for ln in b.stdout.splitlines() if "***" in ln]
    assert msg == ["  *** abort.md detected at step 5 ***"]
    assert [ln for ln in a.stdout.splitlines() if "***" in ln] == msg
    assert len(list(work["ours"].glob("*_05.rst"))) == 1
    for d in (work["ours"], work["ref"]):
        (d / "abort.md").rmdir()
        (d / "stop.md").mkdir()
    a = run(ours(prog), base, work["ours"])
    b = run(ref(prog), base, work["ref"])
    assert a.returncode == 0 and b.returncode == 0
    mb = [ln for ln in b.stdout.splitlines() if "***" in ln]
    ma = [ln for ln in a.stdout.splitlines() if "***" in ln]
    assert len(mb) == 2 and ma == mb
    assert_rows_match(monitor_rows(a.stdout), monitor_rows(b.stdout))


@pytest.mark.gpu
@pytest.mark.parametrize("prog,bits,wrong", [("ai", 2, 1), ("mm", 1, 4), ("lj", 4, 2)])
def test_physics_option(prog, bits, wrong, work):
    """--physics=<bits> (no reference counterpart): the run changes, the
    reference's options and output format do not; a bit the program's force
    field lacks is refused."""
    args = ["--cell=1", "--step=40", "--mon=20", f"--libdir={work['lib']}"]
    a = run(ours(prog), args, work["ours"])
    (work["ours"] / "p").mkdir()
    b = run(ours(prog), args + [f"--physics={bits}"], work["ours"] / "p")
    assert a.returncode == 0 and b.returncode == 0, a.stderr + b.stderr
    ra, rb = monitor_rows(a.stdout), monitor_rows(b.stdout)
    assert len(ra) == len(rb) >= 2
    assert [len(r) for r in ra] == [len(r) for r in rb]
    assert [r[:-1] for r in ra] != [r[:-1] for r in rb]      # all but the elapsed time
    (work["ours"] / "w").mkdir()
    c = run(ours(prog), args + [f"--physics={wrong}"], work["ours"] / "w")
    assert c.returncode != 0


@pytest.fixture()
def reflib(tmp_path):
    lib = write_reference_library(tmp_path)
    a = tmp_path / "ours"
    b = tmp_path / "ref"
    a.mkdir()
    b.mkdir()
    return {"lib": str(lib), "ours": a, "ref": b, "root": tmp_path}


@pytest.mark.gpu
@pytest.mark.parametrize("prog,species,args", [
    ("lj", "C70", ["--cell=2", "--step=60", "--mon=20"]),
    ("lj", "C84:1", ["--cell=2", "--step=60", "--mon=20"]),
    ("ai", "C60", ["--cell=2", "--step=20", "--mon=5"]),
    ("ai", "C70", ["--cell=2", "--step=20", "--mon=5"]),
    ("ai", "C84:24:D6h", ["--cell=2", "--step=20", "--mon=5"]),
    ("mm", "C72", ["--cell=2", "--step=30", "--mon=10"]),
    ("mm", "C84:1", ["--cell=2", "--step=30", "--mon=10"]),
])
def test_reference_molecules_match_reference(prog, species, args, reflib):
    """Whole runs on the reference library's own molecules (resolve_fullerene,
    LJ:210-226; load_cc1, LJ:178-207): the 70-84 atom molecules take the
    cell-grid list path of the atomistic programs (the molecule-wise builder
    covers 32-64 atoms).  Monitor and average lines against the serial
    reference."""
    args = args + [f"--fullerene={species}", f"--libdir={reflib['lib']}"]
    a = run(ours(prog), args, reflib["ours"])
    assert a.returncode == 0, a.stdout + a.stderr
    b = run(ref(prog), args, reflib["ref"])
    assert b.returncode == 0, b.stderr
    assert banner(a.stdout) == banner(b.stdout)
    assert_rows_match(monitor_rows(a.stdout), monitor_rows(b.stdout))
    assert_avg_match(averages(a.stdout), averages(b.stdout))


@pytest.mark.gpu
@pytest.mark.parametrize("prog,args", [("core", []), ("lj", ["--step=200", "--mon=100"]),
                                       ("mm", ["--step=200", "--mon=100"]), ("ai", ["--step=200", "--mon=100"])])
def test_reference_test_script_gpu_rows(prog, args, reflib):
    """The *_gpu rows of the reference's own validation script
    (Test_fuller.sh:211-272; pass rule run_test, :159-183): each program
    with the script's arguments, run from a directory holding FullereneLib
    (the script cd's to the checkout's root), passes when it exits 0 and its
    output contains "Done".  The script itself does not travel with this
    repository; these are its invocations and its pass rule."""
    r = run(ours(prog), args, reflib["root"], timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert "Done" in r.stdout
