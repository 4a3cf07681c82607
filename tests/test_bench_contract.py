"""bench.py helpers that need no GPU: the DRAM traffic figures it reports beside the roofline
come from the committed ncu summaries and must parse as whole byte counts."""
import bench


def test_traffic_figures_parse_from_profiles():
    plain = bench.read_traffic()
    assert plain is not None and 1e8 < plain < 1e9          # one 512x128x128 FP32 step launch
    step = bench.read_traffic("fslbm_step2_batch_kernel_ensemble64.md",
                              "dram_bytes_per_step_full_size")
    assert step is not None and 1e9 < step < 1e10             # one step of the 64-pipe ensemble
    launch = bench.read_traffic("fslbm_step2_batch_kernel_ensemble64.md")
    assert launch is not None and abs(launch / 16 - step) < 1.0


def test_missing_summary_gives_none():
    assert bench.read_traffic("no_such_summary.md") is None
