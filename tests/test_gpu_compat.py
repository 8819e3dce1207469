"""The C++ drop-in layer (include/golap_compat/golap_compat.cuh): a pipeline in
the reference's per-chunk style (ChunkDecompressor steps + a kernel calling
HashMap::probe) must give the oracle's Q1 result and agree with the fused
gx_scan on the same compressed chunks."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from golap_public_b200 import datagen
from golap_public_b200._lib import LIB_PATH
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    out = tmp_path_factory.mktemp("compat") / "q1_pipeline"
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), str(ROOT / "tests" / "compat" / "q1_pipeline.cu"), "-o", str(out),
           "-L", str(LIB_PATH.parent), "-lgx", f"-Xlinker=-rpath,{LIB_PATH.parent}"]
    subprocess.run(cmd, check=True)
    return out


@pytest.mark.parametrize("month,disc,qty", [(199401, (4, 6), (26, 35)), (199512, (1, 3), (1, 24))])
def test_reference_style_pipeline(binary, tmp_path, month, disc, qty):
    f = datagen.fact_q1(8_500_000, True, seed=77)
    dd = datagen.date_dim()
    for k, v in f.items():
        v.astype(np.int32).tofile(tmp_path / f"{k}.bin")
    ok = (dd["d_yearmonthnum"] == month).astype(np.int32)
    dd["d_key"].tofile(tmp_path / "d_key.bin")
    ok.tofile(tmp_path / "d_ok.bin")
    lo, hi = int(dd["d_key"][ok == 1].min()), int(dd["d_key"][ok == 1].max())
    r = subprocess.run([str(binary), str(tmp_path), str(tmp_path / "d_key.bin"), str(tmp_path / "d_ok.bin"), str(lo),
                        str(hi), *map(str, disc), *map(str, qty)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    fields = dict(x.split("=") for x in r.stdout.split())
    want = O.q1(f["date_key"], f["discount"], f["quantity"], f["extended_price"], dd["d_key"], ok, *disc, *qty)
    assert int(fields["pipeline"]) == want and int(fields["fused"]) == want
    kept, total = map(int, fields["chunks"].split("/"))
    assert total == 9 and 1 <= kept <= 2
