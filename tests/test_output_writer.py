"""The output-file formatter and background writer used by the drop-in
DVMBase (dvmpp_b200/host/OutputWriter.*): byte-identical to the reference's
std::ostream formatting over ~2.2 M values (incl. specials and rounding
boundaries), multi-threaded row formatting equal to a plain ostream loop,
ordered appends, and errors surfacing on flush.  CPU only: the checker is
compiled here with g++."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "dvmpp_b200", "host")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_formatter_and_writer(tmp_path):
    exe = str(tmp_path / "check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + HOST,
                    os.path.join(ROOT, "tests", "cpu_cpp", "output_format_check.cpp"),
                    os.path.join(HOST, "OutputWriter.cpp"), "-o", exe], check=True,
                   capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
