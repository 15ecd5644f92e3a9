"""The launch-shape autotuner (zqd_autotune): it measures the shapes the kernels accept for a
(dims, points, states, precision) key, records the fastest, and jobs created afterwards use it.
Results with a tuned shape stay within the parity bars against the oracle (FP64: populations
1e-12, relative L2 of the wavefunction 1e-10; FP32: populations 1e-5), and the table survives a
save / clear / load round trip."""
import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import quantum_dynamics as qd

from test_gpu_parity import FP32_POP_TOL, compare, tully

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fresh_table():
    qd.tune_clear()
    yield
    qd.tune_clear()


def test_tuned_1d_shape_keeps_parity():
    e = qd.autotune(1, 1024, 2, "fp64")
    assert e["candidates"] >= 2 and e["us_per_step"] <= e["default_us_per_step"] * 1.0001
    opt = tully("tully_1", True, npoint=1024, iters=400)
    gpu, _, _ = compare(opt)
    job = qd.Job(opt)
    if e["cluster_ctas"]:
        assert job.info()["cluster_ctas"] == e["cluster_ctas"]
    job.close()


def test_tuned_2d_shape_keeps_parity_fp64_and_fp32():
    from test_gpu_nd import coupled_harmonic_2d

    for prec in ("fp64", "fp32"):
        e = qd.autotune(2, 64, 3, prec)
        assert e["candidates"] >= 2
    opt = coupled_harmonic_2d(npoint=64, iters=100)
    compare(opt)
    compare(opt, precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4)


def test_table_save_clear_load(tmp_path):
    e = qd.autotune(1, 256, 1, "fp32")
    path = tmp_path / "tune.txt"
    qd.tune_save(path)
    lines = [ln for ln in open(path) if not ln.startswith("#")]
    qd.tune_clear()
    qd.tune_load(path)
    qd.tune_save(tmp_path / "again.txt")
    assert lines == [ln for ln in open(tmp_path / "again.txt") if not ln.startswith("#")]
    if e["cluster_ctas"]:
        assert lines == [f"1 256 1 1 {e['cluster_ctas']} {e['radix_log2']} 0 0 0 0\n"]


def test_tuned_nd_shape_round_trips_with_the_tma_fields(tmp_path):
    e = qd.autotune(3, 32, 1, "fp64")
    assert e["candidates"] >= 2 and e["us_per_step"] <= e["default_us_per_step"] * 1.0001
    path = tmp_path / "tune.txt"
    qd.tune_save(path)
    lines = [ln.split() for ln in open(path) if not ln.startswith("#")]
    if lines:  # a tuned shape beat the rules: all ten fields, the TMA pair as measured
        assert len(lines) == 1 and len(lines[0]) == 10
        assert [int(x) for x in lines[0][8:]] == [e["tma_row_block"], e["tma_tile_lines"]]
    # an eight-field table (written before the TMA-staged passes) still loads
    old = tmp_path / "old.txt"
    old.write_text("2 64 1 0 0 0 2 4\n")
    qd.tune_clear()
    qd.tune_load(old)
    qd.tune_save(tmp_path / "again.txt")
    assert [ln for ln in open(tmp_path / "again.txt") if not ln.startswith("#")] == ["2 64 1 0 0 0 2 4 0 0\n"]
