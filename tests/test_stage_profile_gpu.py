"""Stage profiles (the reference's STAGE_SAMPLE tables and stage spread):
every launch of the double-blocked drivers is attributed to one of the
reference's stage names, and the stage times add up to the kernel-class times
of the same interval."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("argv,want", [
    (["--op", "potrf", "--n", "2048", "--outer", "512", "--inner", "128"],
     {"POTRF", "TRSM", "Inner GEMM", "Outer GEMM"}),  # SYRK inside the outer GEMM launch
    (["--op", "potrf", "--n", "2048", "--outer", "512", "--inner", "128", "--syrk-k-tile", "256"],
     {"POTRF", "TRSM", "Inner GEMM", "Outer SYRK", "Outer GEMM"}),
    (["--op", "getrf", "--n", "2048", "--outer", "1024", "--inner", "256", "--batched",
      "--trsm-block", "256"],
     {"Panel GETRF", "Inner pivot batch", "Inner TRSM", "Inner GEMM", "Outer pivot batch",
      "Outer TRSM block", "Outer TRSM GEMM", "Outer GEMM"}),
    (["--op", "getrf", "--n", "2048", "--outer", "1024", "--inner", "256"],
     {"Panel GETRF", "Pivot propagation", "Inner TRSM", "Inner GEMM", "Outer TRSM direct",
      "Outer GEMM"}),
])
def test_stage_samples(hd, torch_cuda, capsys, argv, want):
    from hygondoubleblockedfactorizations_b200 import stage_profile
    out = stage_profile.main(argv + ["--reps", "3", "--stage-samples"])
    text = capsys.readouterr().out
    assert text.count("STAGE_SAMPLE") == 3
    spread = out["stage_spread"]
    assert set(spread) - {"Total"} == want
    total_classes = sum(v["ms"] for v in out["stages"].values())  # one profiled call, by class
    assert spread["Total"]["mean_ms"] == pytest.approx(total_classes, rel=0.25)
    for name, st in spread.items():
        assert st["min_ms"] <= st["mean_ms"] <= st["max_ms"]
