"""The C++ drop-in layer compiles against include/ and reports bad ingest
arguments as exceptions (no GPU needed: every call fails its argument checks
before touching the device)."""
import subprocess
from pathlib import Path

from golap_public_b200._lib import LIB_PATH

ROOT = Path(__file__).resolve().parent.parent


def test_compat_header_errors_without_gpu(tmp_path):
    out = tmp_path / "errors_host"
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), str(ROOT / "tests" / "compat" / "errors_host.cu"), "-o", str(out),
           "-L", str(LIB_PATH.parent), "-lgx", f"-Xlinker=-rpath,{LIB_PATH.parent}"]
    subprocess.run(cmd, check=True)
    r = subprocess.run([str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("threw") == 4
