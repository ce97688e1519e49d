"""CPU checks of bench.py's accounting: per-class algorithmic bytes count only
the launches that did work, and the roofline figures follow from them."""
import bench


def test_work_launches_per_class():
    w = bench.work_launches(inner=60, outer=5)
    assert w["jline"] == 8 * 60  # two MSOLVEs of two red/black passes each per iteration
    assert w["outer_step"] == 5
    assert all(w[k] == 60 for k in ("p_update", "matvec_alpha", "s_update", "matvec_omega", "xr_update"))


def test_class_table_ignores_idle_launches():
    cells = 1_000_000
    # 10 launches of which 8 did work, 1 ms in all
    kt = {"jline": (1.0, 10), "outer_step": (0.5, 10)}
    t = bench.class_table(kt, cells, True, 1000.0, {"jline": 8, "outer_step": 2})
    j = t["jline"]
    assert j["launches"] == 10 and j["work_launches"] == 8
    assert abs(j["us_per_launch"] - 125.0) < 1e-9
    assert abs(j["gbs"] - 20 * cells * 8 / 1e-3 / 1e9) < 1e-6  # 20 B per cell per FP32 half-sweep
    assert abs(j["frac"] - j["gbs"] / 1000.0) < 1e-3
    # a work count above the launches seen is capped
    t = bench.class_table({"p_update": (1.0, 4)}, cells, False, 1000.0, {"p_update": 9})
    assert t["p_update"]["work_launches"] == 4


def test_cg_bytes_model():
    # 40 words per cell per FP64 CG iteration: MSOLVE 20, matvec 9, rho 2, P 3, X/R 6
    assert bench.BYTES_CG_ITER == 8 * 40
