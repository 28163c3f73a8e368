"""Host-side pieces of bench.py that its JSON lines depend on (no GPU):
the DRAM traffic each roofline line takes from the committed ncu summaries,
and the zero-padded byte model the Toeplitz lines are quoted on."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_profile_traffic_lines_parse():
    """Every roofline line that quotes a captured traffic finds a positive figure
    in its profile, and the figures are the sums written in those files."""
    nudft = bench.ncu_traffic()
    c5 = bench.ncu_traffic("toeplitz_apply_warm512.md", "traffic_bytes_per_apply:")
    c3 = bench.ncu_traffic("toeplitz_apply_toep3d_256x256x32.md", "traffic_bytes_per_apply:")
    assert nudft and nudft > 0
    assert c5 == 583523328.0
    assert c3 == 12562472448.0
    assert bench.ncu_traffic("no_such_profile.md") is None


def test_toeplitz_byte_model():
    """The byte model of one A^H A application: 1.556 GB for the warm-start
    configuration (512x512, 32 coils, one segment) and 25.5 GB for the 3-D
    configuration (256x256x32, 4 coils, 9 segments)."""
    n2 = 512 * 512
    assert bench.toep_model_bytes(n2, 4 * n2, 32, 1) == 1556086784
    n3 = 256 * 256 * 32
    assert bench.toep_model_bytes(n3, 8 * n3, 4, 9) == 25534922752
