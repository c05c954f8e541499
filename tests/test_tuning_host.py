"""Host-side checks of the tunable driver parameters (atlas_b200/csrc/tuning.cu,
the role ATLAS's install-time search output plays for the reference:
tune/blas/gemm/gmmsearch.c writes the chosen blockings into generated
headers).  No GPU: the atlb_tune_* entry points only read and write host
state and the tuning file."""
import os
import subprocess
import sys

import atlas_b200 as AB

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INT_MIN = -2 ** 31
NAMES = ["getrf_nb", "potrf_nb", "dgemm_group", "dgemm_splitk", "lookahead", "mixed_tc_min_work_log2",
         "lookahead_reserve_sms", "sgetrf_nb", "qr_nb", "batch_posv_small", "batch_posv_pw",
         "mixed_krylov"]


def _run(code, **env):
    """Runs `code` in a fresh interpreter (the parameters are read once per process)."""
    e = dict(os.environ)
    e.update(env)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=e, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip()


def test_every_parameter_has_a_name(atl):
    n = AB.atlb_tune_count()
    names = [AB.atlb_tune_name(i).decode() for i in range(n)]
    assert names == NAMES
    assert AB.atlb_tune_name(n) is None and AB.atlb_tune_name(-1) is None


def test_unknown_names_are_rejected(atl):
    assert AB.atlb_tune_get("no_such_parameter") == INT_MIN
    assert AB.atlb_tune_set("no_such_parameter", 3) == -1


def test_set_clamps_and_rounds_to_the_step(atl):
    old = AB.atlb_tune_get("getrf_nb")
    try:
        assert AB.atlb_tune_set("getrf_nb", 100) == 96       # multiples of 32
        assert AB.atlb_tune_get("getrf_nb") == 96
        assert AB.atlb_tune_set("getrf_nb", 10000) == 256    # the fused panel's limit
        assert AB.atlb_tune_set("getrf_nb", 1) == 64
        assert AB.atlb_tune_set("lookahead", 7) == 1
    finally:
        AB.atlb_tune_set("getrf_nb", old)


def test_defaults_without_a_file():
    out = _run("import atlas_b200 as AB; AB.lib(); "
               "print(*[AB.atlb_tune_get(n) for n in %r])" % NAMES, ATLAS_B200_TUNE_FILE="none")
    assert [int(v) for v in out.split()] == [256, 256, 8, 1, 1, 31, 0, 256, 128, 64, 16, 1]


def test_file_is_read_on_first_use(tmp_path):
    conf = tmp_path / "t.conf"
    conf.write_text("# a comment line\ngetrf_nb 128   # trailing comment\npotrf_nb 333\nunknown_name 5\n"
                    "lookahead 0\n")
    out = _run("import atlas_b200 as AB; AB.lib(); "
               "print(AB.atlb_tune_get('getrf_nb'), AB.atlb_tune_get('potrf_nb'), AB.atlb_tune_get('lookahead'),"
               " AB.atlb_tune_get('dgemm_group'))", ATLAS_B200_TUNE_FILE=str(conf))
    assert out.split() == ["128", "320", "0", "8"]  # potrf_nb rounds down to a multiple of 64


def test_load_replaces_values(tmp_path, atl):
    conf = tmp_path / "u.conf"
    conf.write_text("dgemm_group 4\nsgetrf_nb 192\n")
    old = (AB.atlb_tune_get("dgemm_group"), AB.atlb_tune_get("sgetrf_nb"))
    try:
        assert AB.atlb_tune_load(str(conf)) == 2
        assert AB.atlb_tune_get("dgemm_group") == 4 and AB.atlb_tune_get("sgetrf_nb") == 192
        assert AB.atlb_tune_load(str(tmp_path / "missing.conf")) == -1
    finally:
        AB.atlb_tune_set("dgemm_group", old[0])
        AB.atlb_tune_set("sgetrf_nb", old[1])


def test_committed_tuning_file_parses():
    path = os.path.join(ROOT, "atlas_b200", "tuning.conf")
    vals = {}
    for line in open(path):
        line = line.split("#", 1)[0].split()
        if len(line) == 2:
            vals[line[0]] = int(line[1])
    assert set(vals) <= set(NAMES) and "getrf_nb" in vals
