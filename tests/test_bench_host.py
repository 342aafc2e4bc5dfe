"""Host-side pieces of bench.py's JSON line (no GPU): the kernel named in
`roofline`, the DRAM traffic read from the ncu summary table under profiles/,
the algorithmic-bytes numerator and the run defaults."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def shape(variant, knob, vector, schedule="levels", streams=2):
    return {"schedule": schedule, "variant": variant, "knob": knob, "vector": vector, "streams": streams}


def test_kernel_names_of_the_default_shapes():
    assert bench.kernel_name(shape("compact", -180, 4), True) == "sweep_direct_slot_kernel<4,64,compact,12>"
    assert bench.kernel_name(shape("compact", -172, 4), True) == "sweep_direct_slot_kernel<4,64,compact,14>"
    assert bench.kernel_name(shape("direct", -196, 2), True) == "sweep_direct_slot_kernel<2,64,full,10>"
    assert bench.kernel_name(shape("compact", -96, 2), False) == "sweep_direct_level_kernel<double,2,-96,compact>"
    assert bench.kernel_name(shape("records", 16, 4, "persist", 1), True) == "sweep_record_persist_kernel<float,16,4>"


def test_traffic_rows_of_the_profile_table():
    # the compact rows of profiles/sweep_traffic.md (FP32 slotted, FP64 capped)
    fam32 = bench.traffic_family(shape("compact", -180, 4), True)
    fam64 = bench.traffic_family(shape("compact", -96, 2), False)
    assert fam32 == "compact float vg4" and fam64 == "compact double vg2"
    t32 = bench.profiled_traffic("kuhn32_s8_g8", fam32)
    t64 = bench.profiled_traffic("kuhn32_s8_g8", fam64)
    assert t32 == pytest.approx(4.361e9) and t64 == pytest.approx(8.357e9)
    # the sweep reads less from DRAM than its algorithmic bytes (8.12 / 16.10 GB):
    # upwind rows are L2 hits
    assert t32 < 8.12e9 and t64 < 16.10e9
    assert "sweep_traffic.md" in bench.TRAFFIC_SOURCE
    assert bench.profiled_traffic("kuhn32_s8_g8", "compact float vg1") is None
    assert bench.profiled_traffic("kuhn64_s8_g16", fam32) is None


def test_algorithmic_bytes():
    # one cell, one angle, one group, no upwind face: psi write (4 values),
    # FP64 phi in and out (4 x 16 B), 208 B of per-cell tables
    assert bench.algorithmic_bytes(1, 1, 1, 0, 4) == 4 * 4 + 64 + 208
    assert bench.algorithmic_bytes(1, 1, 1, 0, 8) == 8 * 4 + 64 + 208
    # each upwind face adds three values per group
    nc, A, G, n_in = 10, 8, 4, 50
    assert (bench.algorithmic_bytes(nc, A, G, n_in, 4) - bench.algorithmic_bytes(nc, A, G, 0, 4)
            == 4 * G * 3 * n_in)


def test_defaults_keep_the_timing_rules(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
    assert a.impl == "b200" and a.workload == "kuhn32_s8_g8" and a.shape == "default"


def test_reference_inputs_are_written_without_the_product(tmp_path):
    """The reference arm's mesh and inputs (oracle/kuhn_problem.py) equal the
    product's byte for byte: the same .smesh, sigma_t, sigma_s and q."""
    import numpy as np
    import tycho2_b200 as ty
    from oracle import kuhn_problem as kp
    for n, jitter, seed in ((3, 0.05, 7), (4, 0.0, 0), (5, 0.05, 1234)):
        a, b = str(tmp_path / "a.smesh"), str(tmp_path / "b.smesh")
        kp.write_smesh(a, kp.kuhn_cube(n, jitter, seed))
        ty.TychoMesh.kuhn_cube(n, jitter, seed, 1.0).write_smesh(b)
        assert open(a, "rb").read() == open(b, "rb").read()
    for p in ty.problems.batch_instances(4, seed=4321) + [ty.problems.WORKLOADS["kuhn8_s4_g1"]]:
        ours, theirs = kp.make_problem(**p)[1:], ty.problems.make_problem(**p)[1:]
        for x, y in zip(ours, theirs):
            assert (x is None and y is None) or np.array_equal(x, y)


def test_psi_hash_is_the_weighted_word_sum():
    import numpy as np
    rng = np.random.default_rng(3)
    psi = rng.normal(size=1000)
    words = [int(x) for x in psi.view(np.uint64)]
    want = sum(x * (2 * i + 1) for i, x in enumerate(words)) % (1 << 64)
    assert bench.psi_hash(psi) == "%016x" % want
    assert bench.psi_hash(psi, chunk=7) == "%016x" % want
