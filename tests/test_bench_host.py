"""bench.py's host-side arithmetic (no GPU): the byte models at the 3,145,728-tet channel give the
figures the roofline fractions and profiles quote, the measured-traffic table stays within 10 % of
the algorithmic bytes, and the L2 note says which workloads are L2-warm."""
import bench

N, F, NB, NODES = 3145728, 6332416, 81920, 545025  # bump channel 128 x 64 x 64 hexes


def test_step_byte_model():
    assert round(bench.model_bytes_per_cell_stage(N, F), 1) == 523.7


def test_algorithmic_bytes_per_launch():
    fp64 = bench.algorithmic_bytes(N, F, NB, NODES, "fp64", True)
    mixed = bench.algorithmic_bytes(N, F, NB, NODES, "mixed", True)
    assert round(fp64["gradient"] / 1e6, 1) == 796.7 and round(fp64["flux"] / 1e6, 1) == 1157.4
    assert round(mixed["gradient"] / 1e6, 1) == 527.9 and round(mixed["flux"] / 1e6, 1) == 1054.7


def test_measured_traffic_is_close_to_the_algorithmic_bytes():
    for (prec, kern), per_cell in bench.MEASURED_DRAM_BYTES_PER_CELL.items():
        alg = bench.algorithmic_bytes(N, F, NB, NODES, prec, True)[kern]
        assert 0.9 <= per_cell * N / alg <= 1.1, (prec, kern)


def test_l2_note():
    assert "no flush needed" in bench.l2_note(523.7 * N)
    assert "L2-warm" in bench.l2_note(526.7 * 48000)
