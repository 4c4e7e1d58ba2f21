"""CPU: the preprocess command's argument handling (no GPU is touched before
the arguments are checked): the reference's usage text and messages
(src/preprocess_cli.cpp:22-127), which exit 0 as the reference does."""
import os
import subprocess

import pytest

from conftest import GOLDEN, ROOT

PRE = os.path.join(ROOT, "new_fgssjoin_b200", "_lib", "preprocess")
pytestmark = pytest.mark.skipif(not os.path.exists(PRE), reason="preprocess not built")


def _run(*args):
    return subprocess.run([PRE] + list(args), capture_output=True, text=True, timeout=60)


def test_usage_without_arguments():
    p = _run()
    assert p.returncode == 0 and "preprocess selfjoin <only_file> <q_gram>" in p.stdout
    assert "preprocess dualjoin <1st_file> <2nd_file> <q_gram>" in p.stdout


def test_missing_arguments_and_files():
    p = _run("selfjoin", os.path.join(GOLDEN, "small.txt"))
    assert p.returncode == 0 and p.stderr.startswith("Missing arguments.")
    p = _run("selfjoin", "/nonexistent/x.txt", "3")
    assert p.returncode == 0 and 'File "/nonexistent/x.txt" does not exist.' in p.stderr
    p = _run("dualjoin", os.path.join(GOLDEN, "small.txt"), "/nonexistent/y.txt", "3")
    assert 'File "/nonexistent/y.txt" does not exist.' in p.stderr


@pytest.mark.parametrize("q", ["0", "1025", "abc"])
def test_bad_qgram(q):
    p = _run("selfjoin", os.path.join(GOLDEN, "small.txt"), q)
    assert p.returncode == 0 and 'Bad "qgram" value. Must be between 1 and 1024.' in p.stderr
