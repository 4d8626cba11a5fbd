"""The SYRK / TRSM / GEMM component benchmarks write the reference's CSV
schema (src/utils/benchmark/benchmark_printer.cpp:26-68) and their methods
compute the right thing (forward error against an FP64 product, sampled FP64
residual)."""
import csv

import pytest

pytestmark = pytest.mark.gpu

COLUMNS = ["benchmark", "method", "parameters", "iteration", "time_ms", "mean_ms", "median_ms",
           "stddev_ms", "min_ms", "max_ms", "gflops", "speedup", "forward_error",
           "residual_metric", "residual_value"]


@pytest.mark.parametrize("argv,fwd_bound", [
    (["syrk", "1024", "384", "3", "--nb", "256", "--k-tile", "128"], 1e-5),
    (["trsm", "1024", "512", "3", "--nb", "128", "--double-nb", "256", "--b", "64"], 1e-5),
    (["gemm", "--shape", "1000", "700", "300", "--m-tile", "256", "--error-mode", "3"], 1e-5),
])
def test_component_csv(hd, torch_cuda, tmp_path, monkeypatch, argv, fwd_bound):
    from hygondoubleblockedfactorizations_b200 import component_bench
    path = tmp_path / "bench.csv"
    monkeypatch.setenv("BENCHMARK_CSV_PATH", str(path))
    monkeypatch.setenv("BENCHMARK_WARMUP_ITERS", "1")
    monkeypatch.setenv("BENCHMARK_PROFILE_ITERS", "2")
    res = component_bench.main(argv)
    rows = list(csv.reader(open(path)))
    assert rows[0] == COLUMNS
    assert len(rows) - 1 == 2 * len(res)
    for r in res:
        bound = 5e-2 if "Mixed" in r["method"] else fwd_bound  # FP16 operands
        assert 0 <= r["forward_error"] <= bound, r
        assert 0 <= r["residual_value"] <= bound, r
        assert r["gflops"] > 0
