"""The heom_scan driver's host side (no GPU): template expansion, key grouping, names.

heom_scan replaces script/IO-scripts/gen_2d_data.sh + script/cpu-script/submit_jobs.sh.
Its template mode must write exactly the key files gen_2d_data.sh writes (same names,
same substitutions), and its directory mode must batch exactly the keys that differ
only in pulse times and end time.
"""
import os
import subprocess
import sys

import pytest

from heomtest import KEYS, PKG_DIR, ROOT, load_pkg

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from make_fixtures import SCAN_ARGS, gen_2d_keys  # noqa: E402

EXE = os.path.join(PKG_DIR, "heom_scan")
TMPL = os.path.join(KEYS, "t_scan.key-tmpl")


def _template_args(key_dir, out_dir):
    a = SCAN_ARGS
    return [EXE, "--template", TMPL, "--key-dir", str(key_dir), "--output-dir", str(out_dir),
            "--t0", str(a["t0"]), "--propagate", str(a["propagate"]), "--tau-step", str(a["tau_step"]),
            "--tau-bound", str(a["tau_bound"]), "--T", ",".join(a["T"])]


@pytest.fixture(scope="module")
def exe():
    if not os.path.exists(EXE):
        pytest.skip("heom_scan not built")
    return EXE


def test_template_mode_writes_gen_2d_data_keys(exe, tmp_path):
    r = subprocess.run(_template_args(tmp_path / "in", tmp_path / "out") + ["--dry-run"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    want = gen_2d_keys(open(TMPL).read(), **SCAN_ARGS)
    got = {f: open(tmp_path / "in" / f).read() for f in os.listdir(tmp_path / "in")}
    assert got == want
    assert "10 key files, 1 scan groups" in r.stdout
    for name in want:
        assert f"{name} -> out{name[3:-4]}.out" in r.stdout
    assert not (tmp_path / "out").exists()  # a dry run propagates nothing


def test_directory_mode_groups_by_system(exe, tmp_path):
    keys = gen_2d_keys(open(TMPL).read(), **SCAN_ARGS)
    d = tmp_path / "in"
    d.mkdir()
    for name, text in keys.items():
        (d / name).write_text(text)
    # a different disorder seed draws different samples: its own group
    other = keys["key_0_0.key"].replace("2 114\n", "2 115\n")
    assert other != keys["key_0_0.key"]
    (d / "key_seed_0.key").write_text(other)
    (d / "notes.txt").write_text("not a key file")
    r = subprocess.run([exe, "--input-dir", str(d), "--output-dir", str(tmp_path / "out"), "--dry-run"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "11 key files, 2 scan groups" in r.stdout
    assert "group 0: 10 points, 2 samples" in r.stdout and "group 1: 1 points, 2 samples" in r.stdout


def test_unreadable_key_is_reported(exe, tmp_path):
    d = tmp_path / "in"
    d.mkdir()
    (d / "key_bad_0.key").write_text("SIZE\n3\n")
    r = subprocess.run([exe, "--input-dir", str(d), "--output-dir", str(tmp_path / "out"), "--dry-run"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "key_bad_0.key" in r.stderr


def test_scan_compatible_api():
    heom = load_pkg()
    keys = gen_2d_keys(open(TMPL).read(), **SCAN_ARGS)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        paths = {}
        for name in ("key_0_0.key", "key_-20_50.key"):
            paths[name] = os.path.join(d, name)
            open(paths[name], "w").write(keys[name])
        p3 = os.path.join(d, "k3.key")
        open(p3, "w").write(keys["key_0_0.key"].replace("0.5308 30 20 12500", "0.6 30 20 12500"))
        a = heom.Problem.from_key(paths["key_0_0.key"])
        b = heom.Problem.from_key(paths["key_-20_50.key"])
        c = heom.Problem.from_key(p3)
        assert a.scan_compatible(b) and b.scan_compatible(a)
        assert not a.scan_compatible(c)  # a different pulse amplitude is a different system
