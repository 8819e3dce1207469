"""The C++ drop-in layer (include/golap_compat/golap_compat.cuh): pipelines in
the reference's per-chunk style must give the oracle's results and agree with
the fused gx_scan on the same compressed chunks.
  q1_pipeline.cu  ChunkDecompressor steps + a kernel calling HashMap::probe
                  (usecases/ssb/queries/01.hpp:350-424, 01.cuh:27-54)
  q3_pipeline.cu  the query3 driver's shape (03.hpp:249-547): customer table
                  from compressed customer chunks, hash_map_build_pred_other
                  launches, HashAggregate<group struct> with SumAgg,
                  MinMaxMeta(chunk_num, max_tuples) + init_chunk, MetaChecker
                  on a std::any, Aggregate over the group sums"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from golap_public_b200 import datagen
from golap_public_b200._lib import LIB_PATH
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def _compile(tmp_path_factory, name):
    out = tmp_path_factory.mktemp("compat") / name
    cmd = ["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), str(ROOT / "tests" / "compat" / f"{name}.cu"), "-o", str(out),
           "-L", str(LIB_PATH.parent), "-lgx", f"-Xlinker=-rpath,{LIB_PATH.parent}"]
    subprocess.run(cmd, check=True)
    return out


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    return _compile(tmp_path_factory, "q1_pipeline")


@pytest.fixture(scope="module")
def binary_q3(tmp_path_factory):
    return _compile(tmp_path_factory, "q3_pipeline")


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


@pytest.mark.parametrize("region,ylo,yhi", [(2, 1992, 1997), (4, 1994, 1995)])
def test_reference_style_q3_pipeline(binary_q3, tmp_path, region, ylo, yhi):
    n_cust, n_supp = 250_000, 20_000
    g = datagen.fact_q3(6_300_000, True, seed=91, n_customer=n_cust, n_supplier=n_supp)
    cust = datagen.dim_geo(n_cust, 91, 21)
    supp = datagen.dim_geo(n_supp, 91, 22)
    dd = datagen.date_dim()
    files = {"date_key": g["date_key"], "cust_key": g["cust_key"], "supp_key": g["supp_key"],
             "revenue": g["revenue"], "c_key": cust["key"], "c_nation": cust["nation"], "c_region": cust["region"],
             "s_key": supp["key"], "s_nation": supp["nation"], "s_region": supp["region"], "d_key": dd["d_key"],
             "d_year": dd["d_year"]}
    for k, v in files.items():
        np.ascontiguousarray(v, np.int32).tofile(tmp_path / f"{k}.bin")
    r = subprocess.run([str(binary_q3), str(tmp_path), str(region), str(ylo), str(yhi), "100000"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    lines = r.stdout.split("\n")
    got = {}
    for ln in lines:
        if ln.startswith("g "):
            c, s, y, v = map(int, ln.split()[1:])
            got[(c, s, y)] = v
    summary = dict(x.split("=") for x in next(ln for ln in lines if ln.startswith("groups=")).split())
    sums, counts = O.q3(g["cust_key"], g["supp_key"], g["date_key"], g["revenue"], cust["key"], cust["nation"],
                        cust["region"] == region, supp["key"], supp["nation"], supp["region"] == region,
                        dd["d_key"], dd["d_year"], (dd["d_year"] >= ylo) & (dd["d_year"] <= yhi), 0, 25, 0, 25,
                        ylo, yhi - ylo + 1)
    want = {(c, s, ylo + y): int(sums[c, s, y]) for c, s, y in zip(*np.nonzero(counts))}
    assert got == want
    assert int(summary["total"]) == sum(want.values()) == int(summary["fused_total"]) == int(summary["agg_total"])
    assert summary["minmax_ok"] == "1"
    kept, total = map(int, summary["chunks"].split("/"))
    assert total == 7 and kept == sum(1 for c in range(7) if
                                       g["date_key"][c * 1_000_000:(c + 1) * 1_000_000].min() <= yhi * 10000 + 1231
                                       and g["date_key"][c * 1_000_000:(c + 1) * 1_000_000].max() >= ylo * 10000 + 101)
